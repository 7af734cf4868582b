// internal.h -- helpers shared by the library's host translation units.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/mcml_b200.h"

namespace mcml {

// Records `msg` as this thread's last error and returns `code`.
int set_error(int code, const std::string &msg);
void clear_error();

int parse_config(const char *sim_json_path, const char *input_txt_path, mcml_sim *sims,
                 int max_sims, int *num_sims);
int validate_sim(const mcml_sim *s);
int derive(const mcml_sim *s, mcml_derived *out);

// Everything the file writers need, on the host, in output order.
struct HostOutputs {
  const mcml_sim *sim;
  const mcml_derived *der;
  std::string gpu_name;
  bool replayed;
  // per SDS (0-based): detected weights' FP64 sums and counts
  std::vector<double> weight_sum;
  std::vector<uint64_t> detected;
  // replay rows per SDS, (L+2) floats each, photon order
  std::vector<std::vector<float>> rows;
  // tallies (u64 quanta)
  const uint64_t *A_rz = nullptr;
  const uint64_t *A0_z = nullptr;
  uint32_t nr = 1000, nz = 500;
  float dr = 0.01f, dz = 0.01f;
};

// iostream's default text for a value (printf "%g": 6 significant digits,
// C locale); at most kG6Max bytes.  put_row_text: the values of one
// pathlength row, each followed by a tab, then a newline (io.cpp:313-323).
constexpr int kG6Max = 16;
char *put_g6(char *p, double v);
char *put_row_text(char *p, const float *row, int row_len);

// calculate_average_pathlength (transport.cu:274-297); out has S*L entries.
void average_pathlength(const HostOutputs &o, std::vector<double> &out);

// Writers (io.cpp:11-33, 281-469).  Return MCML_OK or MCML_E_IO.
int write_output_txt(const HostOutputs &o, const std::string &path);
int write_summary(const HostOutputs &o, const std::string &path, double sim_s, double replay_s);
int write_pathlength(const HostOutputs &o, const std::string &dir, bool binary);
int write_average_pathlength(const HostOutputs &o, const std::string &path);
int write_A_rz(const HostOutputs &o, const std::string &dir, bool binary);
int write_A0_z(const HostOutputs &o, const std::string &dir, bool binary);

// The files of one simulation as mcml_write_outputs writes them (flags:
// MCML_OUT_*; pathlength, average pathlength and absorbance only with
// MCML_OUT_REPLAY, io.cpp:281-469 and main.cu:108-141).
int write_files(const HostOutputs &o, const std::string &dir, const char *output_txt,
                uint32_t flags, double sim_s, double replay_s);

// Checkpoint file of a chunked first pass (checkpoint.cpp); the layout is
// the one documented beside mcml_run_checkpointed.
constexpr uint64_t kFnvBasis = 14695981039346656037ull;
constexpr uint32_t kRecordBytes = 40;
struct CkptHeader {
  char magic[8];
  uint32_t version;
  uint32_t record_bytes;
  uint64_t run_digest;
  uint64_t seed, slot_begin, photons, slots;
  uint64_t slots_done;
  uint64_t records;
  uint64_t steps;
  uint64_t launches;
  uint64_t records_digest;
  uint64_t header_digest;
  uint64_t zero[3];
};
uint64_t fnv1a(const void *p, size_t n, uint64_t h);
uint64_t run_digest(const mcml_sim &s, uint64_t seed, uint64_t slot_begin, uint64_t slots);
void ckpt_init(CkptHeader &h);
// exists=false and MCML_OK when the file is absent.
int ckpt_read_header(const std::string &path, CkptHeader &h, bool &exists);
int ckpt_read_records(const std::string &path, const CkptHeader &h, void *dst);
// Writes h (with a fresh header digest) as the whole file's header.
int ckpt_write_header(const std::string &path, CkptHeader &h);
// Appends n records after the ones h counts, then the header that counts them.
int ckpt_append(const std::string &path, CkptHeader &h, const void *recs, uint64_t n,
                uint64_t slots_done, uint64_t steps);

}  // namespace mcml
