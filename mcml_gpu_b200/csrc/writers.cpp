// writers.cpp -- the reference's output files, byte for byte.
//
// Names, open modes and value formatting follow io.cpp:11-33 and 281-469:
// iostream default formatting (6 significant digits) for text, float32
// for binary, fixed file names in the working directory except the
// caller-named reflectance file.  The value written for reflectance and
// absorbance is computed with the reference's expressions
// (weight / (0xFFFFFFFF*N), and / (scale*2*PI*(r+0.5)*dr*dr*dz)).
#include <algorithm>
#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>
#include <thread>
#include <vector>

#include "internal.h"

namespace mcml {

namespace {

constexpr float kPIf = 3.141592654f;

std::string join(const std::string &dir, const std::string &name) {
  if (dir.empty()) return name;
  if (dir.back() == '/') return dir + name;
  return dir + "/" + name;
}

std::string numbered(const char *prefix, int sds1, const char *postfix) {
  return std::string(prefix) + std::to_string(sds1) + postfix;
}

// Text of lines [0, n) appended to fp.  line(i, p) writes line i at p (at
// most max_line bytes) and returns its end.  Lines go out in rounds: all
// host threads format a round's blocks into one of two buffer sets while a
// writer thread appends the previous round from the other set, so the file
// output overlaps the formatting and the lines stay in order.  The
// reference's per-line `<< endl` flushes only cost time; the bytes are the
// same.
template <class Line>
bool append_lines(FILE *fp, size_t n, size_t max_line, Line line) {
  const size_t threads = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
  const size_t block = std::max<size_t>(1, (size_t(4) << 20) / max_line);
  std::vector<std::string> buf[2] = {std::vector<std::string>(threads),
                                     std::vector<std::string>(threads)};
  std::vector<size_t> used[2] = {std::vector<size_t>(threads), std::vector<size_t>(threads)};
  bool ok = true;  // set by the writer thread, read only after joining it
  std::thread writer;
  size_t round = 0;
  for (size_t base = 0; base < n; base += threads * block, ++round) {
    const int k = (int)(round & 1);
    auto work = [&](size_t t) {
      const size_t i0 = base + t * block, i1 = std::min(n, i0 + block);
      used[k][t] = 0;
      if (i0 >= i1) return;
      buf[k][t].resize((i1 - i0) * max_line);
      char *p = &buf[k][t][0];
      for (size_t i = i0; i < i1; ++i) p = line(i, p);
      used[k][t] = (size_t)(p - &buf[k][t][0]);
    };
    const size_t active = std::min(threads, (n - base + block - 1) / block);
    std::vector<std::thread> pool;
    for (size_t t = 1; t < active; ++t) pool.emplace_back(work, t);
    work(0);
    for (auto &th : pool) th.join();
    if (writer.joinable()) writer.join();  // the previous round is in the file
    if (!ok) break;
    writer = std::thread([&, k, active] {
      for (size_t t = 0; t < active; ++t)
        if (used[k][t] && std::fwrite(buf[k][t].data(), 1, used[k][t], fp) != used[k][t]) {
          ok = false;
          return;
        }
    });
  }
  if (writer.joinable()) writer.join();
  return ok;
}

}  // namespace

char *put_g6(char *p, double v) {
  return std::to_chars(p, p + kG6Max, v, std::chars_format::general, 6).ptr;
}

char *put_row_text(char *p, const float *row, int row_len) {
  for (int j = 0; j < row_len; ++j) {
    p = put_g6(p, row[j]);
    *p++ = '\t';
  }
  *p++ = '\n';
  return p;
}

// transport.cu:274-297
void average_pathlength(const HostOutputs &o, std::vector<double> &out) {
  const int S = (int)o.sim->num_sds;
  const int L = (int)o.sim->num_layers;
  out.assign((size_t)S * L, 0.0);
  const double inverse_start_weight = double(1 / o.der->start_weight);
  for (int s = 0; s < S; s++) {
    const std::vector<float> &rows = o.rows[s];
    const size_t n = rows.size() / (size_t)(L + 2);
    for (int l = 1; l <= L; l++) {
      double sum_photon_reflectance = 0;
      double sum_photon_change_reflectance = 0;
      const double changed_mua = 0.001 * o.sim->mua[l - 1];
      for (size_t i = 0; i < n; i++) {
        const float *row = &rows[i * (L + 2)];
        double photon_energy = row[0] * inverse_start_weight;
        sum_photon_reflectance += photon_energy;
        photon_energy *= std::exp(-1 * changed_mua * row[l]);
        sum_photon_change_reflectance += photon_energy;
      }
      out[(size_t)s * L + l - 1] =
          std::log(sum_photon_reflectance / sum_photon_change_reflectance) / changed_mua;
    }
  }
}

// io.cpp:11-33
int write_output_txt(const HostOutputs &o, const std::string &path) {
  std::ofstream f(path, std::ios::app);
  if (!f) return set_error(MCML_E_IO, "cannot open " + path);
  const double scale1 = (double)0xFFFFFFFF * (double)o.sim->number_photons;
  for (unsigned i = 0; i < o.sim->num_sds; i++) f << double(o.weight_sum[i] / scale1) << " ";
  f << std::endl;
  return f ? MCML_OK : set_error(MCML_E_IO, "write failed: " + path);
}

// io.cpp:345-381
int write_summary(const HostOutputs &o, const std::string &path, double sim_s, double replay_s) {
  std::ofstream f(path, std::ios::app);
  if (!f) return set_error(MCML_E_IO, "cannot open " + path);
  const double N = (double)o.sim->number_photons;
  const double scale1 = (double)0xFFFFFFFF * N;
  f << "{\n";
  f << "\"MCML_version_K\": " << "3.02" << ",\n";
  f << "\"num_photon\": " << o.sim->number_photons << ",\n";
  f << "\"sim_time\": " << sim_s << ",\n";
  double sim_speed;
  if (o.replayed) {
    f << "\"replay_time\": " << replay_s << ",\n";
    sim_speed = N / (sim_s + replay_s);
  } else {
    sim_speed = N / sim_s;
  }
  f << "\"sim_speed(photons/s)\": " << sim_speed << ",\n";
  f << "\"sim_GPU\": \"" << o.gpu_name << "\",\n";
  f << "\"each_photon_weight\": " << scale1 << ",\n";
  f << "\"number_layers\": " << o.sim->num_layers << ",\n";
  f << "\"detect_mode\": ";
  f << (o.sim->source_probe_oblique ? "\"fiber\"" : "\"ring\"");
  f << ",\n";
  f << "\"num_SDS\": " << o.sim->num_sds << ",\n";
  f << "\"SDS_detected_number\": [";
  const unsigned S = o.sim->num_sds;
  for (unsigned d = 0; d + 1 < S; d++) f << " " << o.detected[d] << " ,";
  f << " " << o.detected[S - 1] << " ]\n";
  f << "}";
  return f ? MCML_OK : set_error(MCML_E_IO, "write failed: " + path);
}

// io.cpp:281-329
int write_pathlength(const HostOutputs &o, const std::string &dir, bool binary) {
  const int L = (int)o.sim->num_layers;
  for (unsigned s = 0; s < o.sim->num_sds; s++) {
    const std::vector<float> &rows = o.rows[s];
    if (binary) {
      const std::string name = join(dir, numbered("pathlength_SDS_", s + 1, ".bin"));
      FILE *fp = std::fopen(name.c_str(), "wb");
      if (!fp) return set_error(MCML_E_IO, "cannot open " + name);
      const size_t n = rows.size();
      const bool ok = n == 0 || std::fwrite(rows.data(), sizeof(float), n, fp) == n;
      std::fclose(fp);
      if (!ok) return set_error(MCML_E_IO, "write failed: " + name);
    } else {
      const std::string name = join(dir, numbered("pathlength_SDS_", s + 1, ".txt"));
      FILE *fp = std::fopen(name.c_str(), "ab");
      if (!fp) return set_error(MCML_E_IO, "cannot open " + name);
      const int rl = L + 2;
      const size_t n = rows.size() / (size_t)rl;
      const bool ok = append_lines(fp, n, (size_t)rl * (kG6Max + 1) + 1, [&](size_t i, char *p) {
        return put_row_text(p, &rows[i * rl], rl);
      });
      const bool closed = std::fclose(fp) == 0;
      if (!ok || !closed) return set_error(MCML_E_IO, "write failed: " + name);
    }
  }
  return MCML_OK;
}

// io.cpp:331-343
int write_average_pathlength(const HostOutputs &o, const std::string &path) {
  std::vector<double> avg;
  average_pathlength(o, avg);
  std::ofstream f(path, std::ios::app);
  if (!f) return set_error(MCML_E_IO, "cannot open " + path);
  const unsigned L = o.sim->num_layers;
  for (unsigned s = 0; s < o.sim->num_sds; s++)
    for (unsigned l = 0; l < L; l++) f << avg[(size_t)s * L + l] << '\t';
  f << std::endl;
  return f ? MCML_OK : set_error(MCML_E_IO, "write failed: " + path);
}

// io.cpp:383-434
int write_A_rz(const HostOutputs &o, const std::string &dir, bool binary) {
  const double scale1 = (double)0xFFFFFFFF * (double)o.sim->number_photons;
  const uint32_t nr = o.nr, nz = o.nz;
  const float dr = o.dr, dz = o.dz;
  std::vector<double> scale2(nr);
  for (uint32_t r = 0; r < nr; r++) scale2[r] = scale1 * 2 * kPIf * (r + 0.5) * dr * dr * dz;
  for (unsigned s = 0; s < o.sim->num_sds; s++) {
    const uint64_t *data = o.A_rz + (size_t)s * nr * nz;
    if (binary) {
      const std::string name = join(dir, numbered("A_rz_SDS_", s + 1, ".bin"));
      FILE *fp = std::fopen(name.c_str(), "wb");
      if (!fp) return set_error(MCML_E_IO, "cannot open " + name);
      std::vector<float> buf((size_t)nr * nz);
      for (uint32_t z = 0; z < nz; z++)
        for (uint32_t r = 0; r < nr; r++)
          buf[(size_t)z * nr + r] = float(double(data[(size_t)z * nr + r] / scale2[r]));
      const bool ok = std::fwrite(buf.data(), sizeof(float), buf.size(), fp) == buf.size();
      std::fclose(fp);
      if (!ok) return set_error(MCML_E_IO, "write failed: " + name);
    } else {
      const std::string name = join(dir, numbered("A_rz_SDS_", s + 1, ".txt"));
      FILE *fp = std::fopen(name.c_str(), "ab");
      if (!fp) return set_error(MCML_E_IO, "cannot open " + name);
      const bool ok = append_lines(fp, nz, (size_t)nr * (kG6Max + 1) + 1, [&](size_t z, char *p) {
        for (uint32_t r = 0; r < nr; r++) {
          p = put_g6(p, double(data[z * nr + r] / scale2[r]));
          *p++ = '\t';
        }
        *p++ = '\n';
        return p;
      });
      const bool closed = std::fclose(fp) == 0;
      if (!ok || !closed) return set_error(MCML_E_IO, "write failed: " + name);
    }
  }
  return MCML_OK;
}

// io.cpp:436-469
int write_A0_z(const HostOutputs &o, const std::string &dir, bool binary) {
  const double scale1 = (double)0xFFFFFFFF * (double)o.sim->number_photons;
  const double scale2 = scale1 * 2 * kPIf * (0 + 0.5) * o.dr * o.dr * o.dz;
  const uint32_t nz = o.nz;
  for (unsigned s = 0; s < o.sim->num_sds; s++) {
    const uint64_t *data = o.A0_z + (size_t)s * nz;
    if (binary) {
      const std::string name = join(dir, numbered("A0_z_SDS_", s + 1, ".bin"));
      FILE *fp = std::fopen(name.c_str(), "wb");
      if (!fp) return set_error(MCML_E_IO, "cannot open " + name);
      std::vector<float> buf(nz);
      for (uint32_t z = 0; z < nz; z++) buf[z] = float(double(data[z] / scale2));
      const bool ok = std::fwrite(buf.data(), sizeof(float), nz, fp) == nz;
      std::fclose(fp);
      if (!ok) return set_error(MCML_E_IO, "write failed: " + name);
    } else {
      const std::string name = join(dir, numbered("A0_z_SDS_", s + 1, ".txt"));
      FILE *fp = std::fopen(name.c_str(), "ab");
      if (!fp) return set_error(MCML_E_IO, "cannot open " + name);
      const bool ok = append_lines(fp, nz, kG6Max + 2, [&](size_t z, char *p) {
        p = put_g6(p, double(data[z] / scale2));
        *p++ = '\n';
        return p;
      });
      const bool closed = std::fclose(fp) == 0;
      if (!ok || !closed) return set_error(MCML_E_IO, "write failed: " + name);
    }
  }
  return MCML_OK;
}

int write_files(const HostOutputs &o, const std::string &d, const char *output_txt,
                uint32_t flags, double sim_s, double replay_s) {
  const bool replay = (flags & MCML_OUT_REPLAY) != 0;
  const bool bin = (flags & MCML_OUT_BINARY) != 0;
  int rc;
  if (replay) {
    if (flags & MCML_OUT_PATHLENGTH) {
      rc = write_pathlength(o, d, bin);
      if (rc) return rc;
    }
    if (flags & MCML_OUT_AVERAGE_PL) {
      rc = write_average_pathlength(o, join(d, "average_pathlength.txt"));
      if (rc) return rc;
    }
  }
  rc = write_output_txt(o, output_txt);
  if (rc) return rc;
  if (replay && (flags & MCML_OUT_ABSORBANCE)) {
    rc = write_A_rz(o, d, bin);
    if (rc) return rc;
    rc = write_A0_z(o, d, bin);
    if (rc) return rc;
  }
  return write_summary(o, join(d, "summary.json"), sim_s, replay_s);
}

}  // namespace mcml

using namespace mcml;

extern "C" int mcml_format_rows_text(const float *rows, uint64_t n_rows, uint32_t row_len,
                                     char *out, uint64_t capacity, uint64_t *written) {
  clear_error();
  if ((!rows && n_rows) || !written || row_len == 0)
    return set_error(MCML_E_INVALID, "bad argument");
  char line[64 * (kG6Max + 1)];
  if (row_len > 63) return set_error(MCML_E_INVALID, "row_len above 63");
  uint64_t total = 0;
  for (uint64_t i = 0; i < n_rows; ++i) {
    const size_t len = (size_t)(put_row_text(line, rows + i * row_len, (int)row_len) - line);
    if (out && total + len <= capacity) std::memcpy(out + total, line, len);
    total += len;
  }
  *written = total;
  return (!out || total <= capacity) ? MCML_OK
                                     : set_error(MCML_E_INVALID, "output buffer too small");
}

extern "C" int mcml_write_host_outputs(const mcml_sim *sim, const mcml_host_data *d,
                                       const char *dir, const char *output_txt, uint32_t flags,
                                       double sim_s, double replay_s) {
  clear_error();
  if (!sim || !d || !output_txt || !d->detected || !d->weight_sum)
    return set_error(MCML_E_INVALID, "null argument");
  const bool replay = (flags & MCML_OUT_REPLAY) != 0;
  if (replay && !d->rows) return set_error(MCML_E_INVALID, "replay outputs need rows");
  if (replay && (flags & MCML_OUT_ABSORBANCE) && (!d->A_rz || !d->A0_z))
    return set_error(MCML_E_INVALID, "absorbance outputs need A_rz and A0_z");
  int rc = validate_sim(sim);
  if (rc) return rc;
  mcml_sim s = *sim;
  s.number_photons = d->photons;
  mcml_derived der;
  rc = derive(&s, &der);
  if (rc) return rc;
  HostOutputs o;
  o.sim = &s;
  o.der = &der;
  o.gpu_name = d->gpu_name ? d->gpu_name : "";
  o.replayed = replay;
  const unsigned S = s.num_sds;
  const int L = (int)s.num_layers;
  o.weight_sum.assign(d->weight_sum, d->weight_sum + S);
  o.detected.assign(d->detected, d->detected + S);
  o.rows.assign(S, {});
  if (replay)
    for (unsigned k = 0; k < S; ++k) {
      if (d->detected[k] && !d->rows[k]) return set_error(MCML_E_INVALID, "missing rows");
      o.rows[k].assign(d->rows[k], d->rows[k] + d->detected[k] * (uint64_t)(L + 2));
    }
  o.nr = d->grid_nr ? d->grid_nr : MCML_REF_GRID_NR;
  o.nz = d->grid_nz ? d->grid_nz : MCML_REF_GRID_NZ;
  o.dr = d->grid_dr > 0 ? d->grid_dr : MCML_REF_GRID_D;
  o.dz = d->grid_dz > 0 ? d->grid_dz : MCML_REF_GRID_D;
  o.A_rz = d->A_rz;
  o.A0_z = d->A0_z;
  return write_files(o, dir ? dir : "", output_txt, flags, sim_s, replay_s);
}
