// config.cpp -- sim_set.json / input.txt reader and derived constants.
//
// Follows read_mua_mus (io.cpp:35-256): the same keys, the same checks in
// the same order with the same messages, and the same float conversions
// (JSON numbers are read as double and narrowed to float where the
// reference stores float; input.txt values are read as float).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/mcml_b200.h"
#include "internal.h"
#include "json_min.h"

namespace mcml {

namespace {

const json::Value *path(const json::Value &root, std::initializer_list<const char *> keys) {
  const json::Value *v = &root;
  for (const char *k : keys) {
    if (v->kind != json::Value::Object) return nullptr;
    v = v->find(k);
    if (!v) return nullptr;
  }
  return v;
}

bool number_at(const json::Value &root, std::initializer_list<const char *> keys, double *out,
               std::string *err) {
  const json::Value *v = path(root, keys);
  if (!v || v->kind != json::Value::Number) {
    std::string name;
    for (const char *k : keys) name += std::string(name.empty() ? "" : ".") + k;
    *err = "sim_set.json: missing or non-numeric key \"" + name + "\"";
    return false;
  }
  *out = v->num;
  return true;
}

// operator>>(float&) on a whitespace-separated stream: a failed read leaves
// the target 0 and every later read fails too.
class FloatStream {
 public:
  explicit FloatStream(std::istream &in) : in_(in) {}
  FloatStream &operator>>(float &f) {
    if (failed_) return *this;
    std::string tok;
    if (!(in_ >> tok)) {
      failed_ = true;
      f = 0.0f;
      return *this;
    }
    char *end = nullptr;
    const float v = std::strtof(tok.c_str(), &end);
    if (end == tok.c_str()) {
      failed_ = true;
      f = 0.0f;
      return *this;
    }
    f = v;
    if (*end != '\0') failed_ = true;  // trailing junk stops the stream after this value
    return *this;
  }

 private:
  std::istream &in_;
  bool failed_ = false;
};

std::string fmt_float(float v) {
  std::ostringstream os;
  os << v;
  return os.str();
}

}  // namespace

int parse_config(const char *sim_json_path, const char *input_txt_path, mcml_sim *sims,
                 int max_sims, int *num_sims) {
  if (!sim_json_path || !input_txt_path || !num_sims)
    return set_error(MCML_E_INVALID, "mcml_parse_config: null argument");
  *num_sims = 0;

  std::ifstream jf(sim_json_path);
  if (!jf) return set_error(MCML_E_PARSE, std::string("cannot open ") + sim_json_path);
  std::stringstream ss;
  ss << jf.rdbuf();
  json::Value root;
  try {
    root = json::Parser(ss.str()).parse();
  } catch (const std::exception &e) {
    return set_error(MCML_E_PARSE, std::string(sim_json_path) + ": " + e.what());
  }
  std::string err;
  double d_photons, d_nsim, d_refl, d_layers, d_upper, d_lower, d_nsds;
  if (!number_at(root, {"number_photons"}, &d_photons, &err) ||
      !number_at(root, {"number_simulation"}, &d_nsim, &err))
    return set_error(MCML_E_PARSE, err);

  const json::Value *np = path(root, {"number_photons"});
  uint64_t number_of_photons;
  if (np->is_integer && np->text[0] != '-')
    number_of_photons = std::strtoull(np->text.c_str(), nullptr, 10);
  else
    number_of_photons = d_photons > 0 ? (uint64_t)d_photons : 0;
  const int n_simulations = (int)d_nsim;

  int oblique[2];
  const char *okeys[2] = {"source_probe_oblique", "detector_probe_oblique"};
  for (int k = 0; k < 2; ++k) {
    const json::Value *v = path(root, {okeys[k]});
    if (v && v->kind == json::Value::Number && v->num == 1.0) {
      oblique[k] = 1;
    } else if (v && v->kind == json::Value::Number && v->num == 0.0) {
      oblique[k] = 0;
    } else {
      return set_error(MCML_E_PARSE, std::string(okeys[k]) + ": " + (v ? v->repr() : "null") +
                                         "is not 1 or 0!");
    }
  }

  if (!number_at(root, {"detector_reflectance"}, &d_refl, &err))
    return set_error(MCML_E_PARSE, err);
  if (d_refl < 0 || d_refl > 1) {
    std::ostringstream os;
    os << "Detector reflectance: " << d_refl << " is out of range !";
    return set_error(MCML_E_PARSE, os.str());
  }
  if (!number_at(root, {"number_layers"}, &d_layers, &err)) return set_error(MCML_E_PARSE, err);
  const int n_layers = (int)d_layers;
  if (n_layers > MCML_MAX_LAYERS) {
    std::ostringstream os;
    os << "Number of layer is too large!\nThis program only allow number lower than "
       << MCML_MAX_LAYERS << " !";
    return set_error(MCML_E_PARSE, os.str());
  }
  if (n_layers < 1) return set_error(MCML_E_PARSE, "number_layers must be at least 1");
  if (!number_at(root, {"upper_n"}, &d_upper, &err) ||
      !number_at(root, {"lower_n"}, &d_lower, &err) ||
      !number_at(root, {"probes", "num_SDS"}, &d_nsds, &err))
    return set_error(MCML_E_PARSE, err);
  const float upper_n = (float)d_upper;
  const float lower_n = (float)d_lower;
  const int num_detector = (int)d_nsds;
  if (num_detector > MCML_MAX_SDS) {
    std::ostringstream os;
    os << "Number of SDS is too large!\nThis program only allow number lower than "
       << MCML_MAX_SDS << " !";
    return set_error(MCML_E_PARSE, os.str());
  }
  const json::Value *dets = path(root, {"probes", "detectors"});
  const size_t dets_size = (dets && dets->kind == json::Value::Array) ? dets->arr.size() : 0;
  if ((size_t)num_detector != dets_size || num_detector < 0) {
    std::ostringstream os;
    os << "Number of SDS : " << num_detector << " not match the probe setting : " << dets_size
       << " !";
    return set_error(MCML_E_PARSE, os.str());
  }
  if (num_detector < 1) return set_error(MCML_E_PARSE, "probes.num_SDS must be at least 1");
  double s_na, s_r, s_a;
  if (!number_at(root, {"probes", "source", "NA"}, &s_na, &err) ||
      !number_at(root, {"probes", "source", "radius"}, &s_r, &err) ||
      !number_at(root, {"probes", "source", "angle"}, &s_a, &err))
    return set_error(MCML_E_PARSE, err);
  std::vector<double> dpos(num_detector), dna(num_detector), drad(num_detector),
      dang(num_detector);
  for (int d = 0; d < num_detector; ++d) {
    const json::Value &o = dets->arr[d];
    if (!number_at(o, {"NA"}, &dna[d], &err) || !number_at(o, {"radius"}, &drad[d], &err) ||
        !number_at(o, {"pos"}, &dpos[d], &err) || !number_at(o, {"angle"}, &dang[d], &err))
      return set_error(MCML_E_PARSE, "probes.detectors[" + std::to_string(d) + "]: " + err);
  }
  if (n_simulations < 1) return set_error(MCML_E_PARSE, "number_simulation must be at least 1");
  if (sims && n_simulations > max_sims) {
    return set_error(MCML_E_INVALID, "number_simulation " + std::to_string(n_simulations) +
                                         " exceeds the caller's capacity " +
                                         std::to_string(max_sims));
  }

  // input.txt: per simulation (h mua mus n g) x (L-1) then (mua mus n g).
  std::ifstream tf(input_txt_path);
  if (!tf) return set_error(MCML_E_PARSE, std::string("cannot open ") + input_txt_path);
  FloatStream fs(tf);
  std::vector<mcml_sim> parsed(n_simulations);
  for (int i = 0; i < n_simulations; ++i) {
    mcml_sim &s = parsed[i];
    std::memset(&s, 0, sizeof(s));
    int j = 0;
    while (j < n_layers - 1) {
      fs >> s.height[j] >> s.mua[j] >> s.mus[j] >> s.n[j] >> s.g[j];
      j++;
    }
    fs >> s.mua[j] >> s.mus[j] >> s.n[j] >> s.g[j];
    if (s.mus[j] <= 0)
      return set_error(MCML_E_PARSE, "Mus for simulation " + std::to_string(i) + " layer " +
                                         std::to_string(j) + " Error with value " +
                                         fmt_float(s.mus[j]) + " !");
    if (s.n[j] <= 1)
      return set_error(MCML_E_PARSE, "n for simulation " + std::to_string(i) + " layer " +
                                         std::to_string(j) + " Error with value " +
                                         fmt_float(s.n[j]) + " !");
    if (s.g[j] > 1)
      return set_error(MCML_E_PARSE, "g for simulation " + std::to_string(i) + " layer " +
                                         std::to_string(j) + " Error with value " +
                                         fmt_float(s.g[j]) + " !");
    s.number_photons = number_of_photons;
    s.num_layers = (uint32_t)n_layers;
    s.num_sds = (uint32_t)num_detector;
    s.upper_n = upper_n;
    s.lower_n = lower_n;
    s.detector_reflectance = (float)d_refl;
    s.source_probe_oblique = oblique[0];
    s.detector_probe_oblique = oblique[1];
    s.source_NA = (float)s_na;
    s.source_radius = (float)s_r;
    s.source_angle_deg = (float)s_a;
    for (int d = 0; d < num_detector; ++d) {
      s.det_NA[d] = (float)dna[d];
      s.det_radius[d] = (float)drad[d];
      s.det_pos[d] = (float)dpos[d];
      s.det_angle_deg[d] = (float)dang[d];
    }
  }
  if (sims)
    for (int i = 0; i < n_simulations; ++i) sims[i] = parsed[i];
  *num_sims = n_simulations;
  return MCML_OK;
}

int validate_sim(const mcml_sim *s) {
  if (!s) return set_error(MCML_E_INVALID, "null mcml_sim");
  if (s->num_layers < 1 || s->num_layers > MCML_MAX_LAYERS)
    return set_error(MCML_E_INVALID, "num_layers must be in [1, 10]");
  if (s->num_sds < 1 || s->num_sds > MCML_MAX_SDS)
    return set_error(MCML_E_INVALID, "num_sds must be in [1, 30]");
  if (s->number_photons == 0) return set_error(MCML_E_INVALID, "number_photons must be > 0");
  if (!(s->detector_reflectance >= 0.0f && s->detector_reflectance <= 1.0f))
    return set_error(MCML_E_INVALID, "detector_reflectance must be in [0,1]");
  if ((s->source_probe_oblique != 0 && s->source_probe_oblique != 1) ||
      (s->detector_probe_oblique != 0 && s->detector_probe_oblique != 1))
    return set_error(MCML_E_INVALID, "oblique flags must be 0 or 1");
  const unsigned j = s->num_layers - 1;
  if (!(s->mus[j] > 0)) return set_error(MCML_E_INVALID, "last layer mus must be > 0");
  if (!(s->n[j] > 1)) return set_error(MCML_E_INVALID, "last layer n must be > 1");
  if (s->g[j] > 1) return set_error(MCML_E_INVALID, "last layer g must be <= 1");
  return MCML_OK;
}

// Derived constants, io.cpp:168-238.
int derive(const mcml_sim *s, mcml_derived *out) {
  const int rc = validate_sim(s);
  if (rc) return rc;
  std::memset(out, 0, sizeof(*out));
  const int L = (int)s->num_layers;
  const float PI = 3.141592654f;
  out->det_angle_rad[0] = s->source_angle_deg * PI / 180;
  for (unsigned d = 0; d < s->num_sds; ++d) {
    out->det_angle_rad[d + 1] = s->det_angle_deg[d] * PI / 180;
    out->critical_angle[d + 1] = std::asin(s->det_NA[d] / s->upper_n);
  }
  float z_min_cumulate = 0;
  float z_max_cumulate = 0;
  for (int l = 1; l <= L; l++) {
    const float thickness = (l < L) ? s->height[l - 1] : 0.0f;
    z_max_cumulate += thickness;
    out->z_min[l] = z_min_cumulate;
    out->z_max[l] = z_max_cumulate;
    out->mutr[l] = 1.0f / (s->mua[l - 1] + s->mus[l - 1]);
    z_min_cumulate += thickness;
  }
  const float lower_thickness = 10.0;
  if (out->z_max[L] < lower_thickness) out->z_max[L] = lower_thickness;
  const double n1 = s->upper_n;
  const double n2 = s->n[0];
  double r = (n1 - n2) / (n1 + n2);
  r = r * r;
  out->start_weight = (unsigned int)((double)0xffffffff * (1 - r));
  return MCML_OK;
}

}  // namespace mcml

extern "C" int mcml_parse_config(const char *sim_json_path, const char *input_txt_path,
                                 mcml_sim *sims, int max_sims, int *num_sims) {
  return mcml::parse_config(sim_json_path, input_txt_path, sims, max_sims, num_sims);
}

extern "C" int mcml_derive(const mcml_sim *sim, mcml_derived *out) {
  if (!out) return mcml::set_error(MCML_E_INVALID, "mcml_derive: null output");
  return mcml::derive(sim, out);
}
