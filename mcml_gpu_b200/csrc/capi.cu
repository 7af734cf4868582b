// capi.cu -- implementation of the C ABI declared in include/mcml_b200.h.
//
// A context owns one parameter block (DevParams, the reference's
// __constant__ tables made per-context), a stream, and the device buffers
// of one simulation: slot states, detection records, replay rows and the
// absorbance tallies.  Work is enqueued on the context's stream; blocking
// entry points synchronise only that stream.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/mcml_b200.h"
#include "internal.h"
#include "kernels.h"
#include "params.h"

namespace mcml {

namespace {
thread_local std::string g_last_error;
}

int set_error(int code, const std::string &msg) {
  g_last_error = msg;
  return code;
}
void clear_error() { g_last_error.clear(); }

}  // namespace mcml

using namespace mcml;

#define CUDA_TRY(expr)                                                                  \
  do {                                                                                  \
    cudaError_t e_ = (expr);                                                            \
    if (e_ != cudaSuccess)                                                              \
      return set_error(MCML_E_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
  } while (0)

namespace {

struct DeviceGuard {
  int prev = -1;
  bool changed = false;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) == cudaSuccess && prev != dev) {
      changed = cudaSetDevice(dev) == cudaSuccess;
    }
  }
  ~DeviceGuard() {
    if (changed) cudaSetDevice(prev);
  }
};

template <class T>
void dfree(T *&p) {
  if (p) cudaFree(p);
  p = nullptr;
}

constexpr uint64_t kDefaultBudget = 1ull << 26;
// Automatic slot count for N above the reference's thread count: about
// this many photons per slot keeps the end-of-launch tail (one slot of
// work) small against each lane's share, at one skipahead per slot.
constexpr uint64_t kPhotonsPerSlot = 4;
constexpr uint64_t kMaxAutoSlots = 1ull << 26;

}  // namespace

struct mcml_ctx {
  mcml_sim sim{};
  mcml_opts opts{};
  mcml_derived der{};
  DevParams P{};
  int device = 0;
  int sm_count = 0;
  int max_thr_sm = 0;
  std::string gpu_name;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  uint64_t N = 0, S = 0;
  uint64_t slot_cap = 0;
  uint2 *d_slot_state = nullptr;
  unsigned long long *d_counters = nullptr;
  DetRecord *d_records = nullptr;
  uint64_t rec_cap = 0;
  unsigned long long *d_sums = nullptr;  // det_count[32] | wsum[32] | wsq[32]
  float *d_rows = nullptr;
  uint32_t *d_inter = nullptr;
  uint64_t rows_cap = 0;
  int rows_L = 0;
  unsigned long long *d_Arz = nullptr;
  unsigned long long *d_A0z = nullptr;
  size_t arz_n = 0, a0z_n = 0;
  void *d_order = nullptr;  // record-ordering scratch (fetch_host)
  size_t order_bytes = 0;
  // [0] first pass start, [4] walk start, [1] walk end, [2]/[3] replay
  cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  int walk_block = 128;
  int walk_min_blocks = 8;
  int walk_grid = 0;
  int replay_grid = 0;
  bool ran = false, replayed = false;
  bool host_valid = false;
  std::vector<DetRecord> h_rec;
  std::vector<float> h_rows;
  std::vector<uint32_t> h_inter;
  std::vector<std::vector<uint32_t>> order;  // per SDS, record indices by photon

  ~mcml_ctx() {
    DeviceGuard g(device);
    if (stream) cudaStreamSynchronize(stream);
    dfree(d_slot_state);
    dfree(d_counters);
    dfree(d_records);
    dfree(d_sums);
    dfree(d_rows);
    dfree(d_inter);
    dfree(d_Arz);
    dfree(d_A0z);
    dfree(d_order);
    for (auto &e : ev)
      if (e) cudaEventDestroy(e);
    if (own_stream && stream) cudaStreamDestroy(stream);
  }
};

namespace {

uint32_t grid_nr(const mcml_ctx *c) { return c->opts.grid_nr ? c->opts.grid_nr : 1000u; }
uint32_t grid_nz(const mcml_ctx *c) { return c->opts.grid_nz ? c->opts.grid_nz : 500u; }
float grid_dr(const mcml_ctx *c) { return c->opts.grid_dr > 0 ? c->opts.grid_dr : 0.01f; }
float grid_dz(const mcml_ctx *c) { return c->opts.grid_dz > 0 ? c->opts.grid_dz : 0.01f; }
bool ref_grid(const mcml_ctx *c) {
  return grid_nr(c) == 1000u && grid_nz(c) == 500u && grid_dr(c) == 0.01f && grid_dz(c) == 0.01f;
}

int build_params(mcml_ctx *c) {
  fill_dev_params(c->sim, c->der, c->N, c->S, c->P);
  c->P.grid_nr = grid_nr(c);
  c->P.grid_nz = grid_nz(c);
  c->P.grid_dr = grid_dr(c);
  c->P.grid_dz = grid_dz(c);
  return MCML_OK;
}

// Checks the simulation and sizes the slot states before anything of the
// context changes: a rejected simulation leaves the previous one in place,
// and a failed allocation leaves no simulation that launch_run accepts.
int set_sim(mcml_ctx *c, const mcml_sim *sim) {
  mcml_derived der{};
  int rc = derive(sim, &der);
  if (rc) return rc;
  const uint64_t N = sim->number_photons;
  const uint64_t ref_threads = (uint64_t)c->sm_count * (uint64_t)c->max_thr_sm;
  uint64_t S;
  if (c->opts.slots) {
    S = c->opts.slots;
  } else if (N <= ref_threads) {
    S = N;  // the reference's layout: photon t is thread t's first photon
  } else {
    S = (N + kPhotonsPerSlot - 1) / kPhotonsPerSlot;
    S = std::max(S, ref_threads);
    S = std::min(S, std::max(kMaxAutoSlots, ref_threads));
  }
  if (S > N) S = N;
  if (N / S >= 0xFFFFFFFFull)
    return set_error(MCML_E_INVALID, "too many photons per slot; raise mcml_opts.slots");
  if (S >= 0xFFFFFFFFull) return set_error(MCML_E_INVALID, "slots must be below 2^32");
  if (N >= (1ull << 44)) return set_error(MCML_E_INVALID, "number_photons must be below 2^44");
  const uint64_t nz = grid_nz(c), nr = grid_nr(c);
  if (nr == 0 || nz == 0 || (uint64_t)sim->num_sds * nz * nr >= (1ull << 31))
    return set_error(MCML_E_INVALID, "absorbance grid too large");
  DeviceGuard g(c->device);
  if (S > c->slot_cap) {
    dfree(c->d_slot_state);
    c->slot_cap = 0;
    CUDA_TRY(cudaMalloc(&c->d_slot_state, S * 3 * sizeof(uint2)));
    c->slot_cap = S;
  }
  c->der = der;
  c->sim = *sim;
  c->N = N;
  c->S = S;
  build_params(c);
  c->ran = c->replayed = c->host_valid = false;
  return MCML_OK;
}

int ensure_records(mcml_ctx *c, uint64_t cap) {
  if (cap <= c->rec_cap) return MCML_OK;
  DeviceGuard g(c->device);
  dfree(c->d_records);
  c->rec_cap = 0;
  CUDA_TRY(cudaMalloc(&c->d_records, cap * sizeof(DetRecord)));
  c->rec_cap = cap;
  return MCML_OK;
}

// -1 when either event was never recorded; the failed query's error is
// taken off the thread's last-error slot so a later launch check does not
// report it.
float elapsed(cudaEvent_t a, cudaEvent_t b) {
  float ms = 0.0f;
  if (cudaEventElapsedTime(&ms, a, b) != cudaSuccess) {
    cudaGetLastError();
    ms = -1.0f;
  }
  return ms;
}

int fill_result(mcml_ctx *c, mcml_result *r) {
  unsigned long long cnt[kCntWords];
  unsigned long long sums[96];
  CUDA_TRY(cudaMemcpyAsync(cnt, c->d_counters, sizeof(cnt), cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(cudaMemcpyAsync(sums, c->d_sums, sizeof(sums), cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  if (cnt[kCntRecords] > c->rec_cap) {
    return set_error(MCML_E_OVERFLOW, "detection records " + std::to_string(cnt[kCntRecords]) +
                                          " exceed capacity " + std::to_string(c->rec_cap));
  }
  if (!r) return MCML_OK;
  std::memset(r, 0, sizeof(*r));
  const double *wsum = reinterpret_cast<const double *>(sums + 32);
  const double *wsq = reinterpret_cast<const double *>(sums + 64);
  r->num_sds = c->sim.num_sds;
  r->photons = c->N;
  r->slots = c->S;
  r->steps = cnt[kCntSteps];
  const double Nd = (double)c->N;
  const double scale1 = (double)0xFFFFFFFF * Nd;
  for (unsigned s = 0; s < c->sim.num_sds; ++s) {
    r->detected[s] = sums[s];
    r->weight_sum[s] = wsum[s];
    r->weight_sumsq[s] = wsq[s];
    r->reflectance[s] = wsum[s] / scale1;
    const double mean = wsum[s] / Nd;
    double var = wsq[s] / Nd - mean * mean;
    if (var < 0) var = 0;
    r->std_error[s] = Nd > 1 ? std::sqrt(var / (Nd - 1)) / (double)0xFFFFFFFF : 0.0;
  }
  r->seed_ms = elapsed(c->ev[0], c->ev[4]);
  r->walk_ms = elapsed(c->ev[4], c->ev[1]);
  r->replay_ms = c->replayed ? elapsed(c->ev[2], c->ev[3]) : 0.0f;
  return MCML_OK;
}

// Records (and, after a replay, rows and interaction counts) to the host
// in file order: by SDS, then photon index -- sorted on the device.
// The records (and, after a replay, rows and interaction counts) of the
// last run put in file order on the device: SDS-major, photon order within
// an SDS.  *D gets the record count; o points into the context's ordering
// scratch (valid until the next ordering).  The caller holds the device.
int order_on_device(mcml_ctx *c, uint64_t *D_out, OrderedOutput *o) {
  if (!c->ran) return set_error(MCML_E_STATE, "mcml_run has not been called");
  unsigned long long cnt[kCntWords];
  CUDA_TRY(cudaMemcpyAsync(cnt, c->d_counters, sizeof(cnt), cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  if (cnt[kCntRecords] > c->rec_cap)
    return set_error(MCML_E_OVERFLOW, "detection records exceed capacity");
  if (c->replayed && ((int)cnt[kCntStatus] & kStatusBudget))
    return set_error(MCML_E_BUDGET, "a replayed photon exceeded the step budget");
  const uint64_t D = cnt[kCntRecords];
  const int L = (int)c->sim.num_layers;
  const bool rows = c->replayed;
  *D_out = D;
  *o = OrderedOutput{};
  if (D) {
    // Ordering scratch: kept by the context and grown, never shrunk.
    const size_t need = order_scratch_bytes(D, L, rows);
    if (need > c->order_bytes) {
      dfree(c->d_order);
      c->order_bytes = 0;
      CUDA_TRY(cudaMalloc(&c->d_order, need));
      c->order_bytes = need;
    }
    CUDA_TRY(sort_records_for_output(c->d_records, D, rows ? c->d_rows : nullptr, c->d_inter, L,
                                     c->d_order, c->order_bytes, o, c->sm_count, c->stream));
  }
  return MCML_OK;
}

int fetch_host(mcml_ctx *c) {
  if (c->host_valid) return MCML_OK;
  if (!c->ran) return set_error(MCML_E_STATE, "mcml_run has not been called");
  DeviceGuard g(c->device);
  uint64_t D = 0;
  OrderedOutput o;
  int rc = order_on_device(c, &D, &o);
  if (rc) return rc;
  const int L = (int)c->sim.num_layers;
  const bool rows = c->replayed;
  c->h_rec.resize(D);
  c->h_rows.resize(rows ? D * (L + 2) : 0);
  c->h_inter.resize(rows ? D * L : 0);
  if (D) {
    CUDA_TRY(cudaMemcpyAsync(c->h_rec.data(), o.records, D * sizeof(DetRecord),
                             cudaMemcpyDeviceToHost, c->stream));
    if (rows) {
      CUDA_TRY(cudaMemcpyAsync(c->h_rows.data(), o.rows, D * (L + 2) * sizeof(float),
                               cudaMemcpyDeviceToHost, c->stream));
      CUDA_TRY(cudaMemcpyAsync(c->h_inter.data(), o.interactions, D * L * sizeof(uint32_t),
                               cudaMemcpyDeviceToHost, c->stream));
    }
    CUDA_TRY(cudaStreamSynchronize(c->stream));
  }
  c->order.assign(c->sim.num_sds, {});
  for (uint64_t i = 0; i < D; ++i) {
    const uint32_t s = c->h_rec[i].sds;
    if (s >= 1 && s <= c->sim.num_sds) c->order[s - 1].push_back((uint32_t)i);
  }
  c->host_valid = true;
  return MCML_OK;
}

int launch_run(mcml_ctx *c) {
  if (!c->d_slot_state || c->S > c->slot_cap)
    return set_error(MCML_E_STATE, "no simulation set: the last mcml_set_sim failed");
  DeviceGuard g(c->device);
  CUDA_TRY(cudaMemsetAsync(c->d_counters, 0, kCntWords * sizeof(unsigned long long), c->stream));
  CUDA_TRY(cudaMemsetAsync(c->d_sums, 0, 96 * sizeof(unsigned long long), c->stream));
  CUDA_TRY(cudaEventRecord(c->ev[0], c->stream));
  CUDA_TRY(launch_seed_slots(c->opts.seed, c->opts.slot_begin, c->S, c->d_slot_state,
                             c->sm_count, c->stream));
  CUDA_TRY(cudaEventRecord(c->ev[4], c->stream));
  WalkArgs A;
  A.slot_state = c->d_slot_state;
  A.counters = c->d_counters;
  A.records = c->d_records;
  A.rec_cap = c->rec_cap;
  A.slot_end = c->S;
  CUDA_TRY(launch_walk(c->P, A, c->sim.source_probe_oblique != 0,
                       c->sim.detector_probe_oblique != 0, c->walk_block, c->walk_min_blocks,
                       c->walk_grid, c->stream));
  CUDA_TRY(cudaEventRecord(c->ev[1], c->stream));
  CUDA_TRY(launch_reduce_records(c->d_records, c->d_counters + kCntRecords, c->rec_cap,
                                 c->sim.num_sds, c->d_sums,
                                 reinterpret_cast<double *>(c->d_sums + 32),
                                 reinterpret_cast<double *>(c->d_sums + 64), c->sm_count,
                                 c->stream));
  c->ran = true;
  c->replayed = false;
  c->host_valid = false;
  return MCML_OK;
}

int launch_replay(mcml_ctx *c) {
  if (!c->ran) return set_error(MCML_E_STATE, "mcml_run has not been called");
  DeviceGuard g(c->device);
  const int L = (int)c->sim.num_layers;
  if (c->rows_cap < c->rec_cap || c->rows_L != L) {
    dfree(c->d_rows);
    dfree(c->d_inter);
    c->rows_cap = 0;
    CUDA_TRY(cudaMalloc(&c->d_rows, c->rec_cap * (L + 2) * sizeof(float)));
    CUDA_TRY(cudaMalloc(&c->d_inter, c->rec_cap * L * sizeof(uint32_t)));
    c->rows_cap = c->rec_cap;
    c->rows_L = L;
  }
  const size_t arz = (size_t)c->sim.num_sds * grid_nz(c) * grid_nr(c);
  const size_t a0z = (size_t)c->sim.num_sds * grid_nz(c);
  if (arz != c->arz_n) {
    dfree(c->d_Arz);
    c->arz_n = 0;
    CUDA_TRY(cudaMalloc(&c->d_Arz, arz * sizeof(unsigned long long)));
    c->arz_n = arz;
  }
  if (a0z != c->a0z_n) {
    dfree(c->d_A0z);
    c->a0z_n = 0;
    CUDA_TRY(cudaMalloc(&c->d_A0z, a0z * sizeof(unsigned long long)));
    c->a0z_n = a0z;
  }
  CUDA_TRY(cudaEventRecord(c->ev[2], c->stream));
  CUDA_TRY(cudaMemsetAsync(c->d_Arz, 0, arz * sizeof(unsigned long long), c->stream));
  CUDA_TRY(cudaMemsetAsync(c->d_A0z, 0, a0z * sizeof(unsigned long long), c->stream));
  CUDA_TRY(cudaMemsetAsync(c->d_counters + kCntReplay, 0, 2 * sizeof(unsigned long long),
                           c->stream));
  ReplayArgs A;
  A.records = c->d_records;
  A.rec_count = c->d_counters + kCntRecords;
  A.rec_cap = c->rec_cap;
  A.cursor = c->d_counters + kCntReplay;
  A.rows = c->d_rows;
  A.interactions = c->d_inter;
  A.A_rz = c->d_Arz;
  A.A0_z = c->d_A0z;
  A.budget = c->opts.replay_step_budget ? c->opts.replay_step_budget : kDefaultBudget;
  A.status = reinterpret_cast<int *>(c->d_counters + kCntStatus);
  CUDA_TRY(mcml::launch_replay(c->P, A, c->sim.source_probe_oblique != 0,
                               c->sim.detector_probe_oblique != 0, ref_grid(c), c->replay_grid,
                               c->stream));
  CUDA_TRY(cudaEventRecord(c->ev[3], c->stream));
  c->replayed = true;
  c->host_valid = false;
  return MCML_OK;
}

// Walk launch shape: threads per block and the register-capping minimum
// of resident blocks per SM; the grid fills every SM with as many blocks
// as fit.  Defaults: 128 threads, 8 blocks (64 registers per thread).
int choose_walk(mcml_ctx *c) {
  const int block = c->opts.block_size ? (int)c->opts.block_size : 128;
  int minb = c->opts.blocks_per_sm ? (int)c->opts.blocks_per_sm : (block == 128 ? 8 : 2048 / block / 2);
  const bool so = c->sim.source_probe_oblique != 0, dobl = c->sim.detector_probe_oblique != 0;
  const bool glass = has_glass_layer(c->P);
  const void *fn = walk_kernel_ptr(block, minb, so, dobl, glass);
  bool limit = false;  // no variant capped for minb: run the uncapped one, minb blocks/SM
  if (!fn) {
    limit = c->opts.blocks_per_sm != 0;
    minb = 1;
    fn = walk_kernel_ptr(block, 1, so, dobl, glass);
  }
  if (!fn) return set_error(MCML_E_INVALID, "block_size must be 64, 128 or 256");
  DeviceGuard g(c->device);
  int nb = 0;
  CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, block, 0));
  if (limit && (int)c->opts.blocks_per_sm < nb) nb = (int)c->opts.blocks_per_sm;
  if (nb < 1) nb = 1;
  c->walk_block = block;
  c->walk_min_blocks = minb;
  c->walk_grid = nb * c->sm_count;
  return MCML_OK;
}

void build_outputs(mcml_ctx *c, HostOutputs &o, std::vector<unsigned long long> &arz,
                   std::vector<unsigned long long> &a0z) {
  const int L = (int)c->sim.num_layers;
  const unsigned S = c->sim.num_sds;
  o.sim = &c->sim;
  o.der = &c->der;
  o.gpu_name = c->gpu_name;
  o.replayed = c->replayed;
  o.weight_sum.assign(S, 0.0);
  o.detected.assign(S, 0);
  o.rows.assign(S, {});
  for (unsigned s = 0; s < S; ++s) {
    const auto &idx = c->order[s];
    o.detected[s] = idx.size();
    double sum = 0.0;
    if (c->replayed) {
      o.rows[s].resize(idx.size() * (L + 2));
      for (size_t k = 0; k < idx.size(); ++k) {
        const float *src = &c->h_rows[(size_t)idx[k] * (L + 2)];
        std::copy(src, src + L + 2, &o.rows[s][k * (L + 2)]);
        sum += (double)src[0];
      }
    } else {
      for (uint32_t i : idx) sum += (double)c->h_rec[i].weight;
    }
    o.weight_sum[s] = sum;
  }
  o.nr = grid_nr(c);
  o.nz = grid_nz(c);
  o.dr = grid_dr(c);
  o.dz = grid_dz(c);
  o.A_rz = reinterpret_cast<const uint64_t *>(arz.data());
  o.A0_z = reinterpret_cast<const uint64_t *>(a0z.data());
}

}  // namespace

// ---------------------------------------------------------------------------
extern "C" {

const char *mcml_version(void) { return "mcml_b200 1.0 (MCML_GPU K3.02 file formats)"; }

const char *mcml_strerror(int status) {
  switch (status) {
    case MCML_OK: return "ok";
    case MCML_E_INVALID: return "invalid argument";
    case MCML_E_CUDA: return "CUDA error";
    case MCML_E_NOMEM: return "out of memory";
    case MCML_E_OVERFLOW: return "detection record buffer overflow";
    case MCML_E_IO: return "file I/O error";
    case MCML_E_PARSE: return "configuration parse error";
    case MCML_E_STATE: return "call sequence error";
    case MCML_E_BUDGET: return "kernel step budget exhausted";
    case MCML_E_NODEV: return "no CUDA device";
    default: return "unknown status";
  }
}

const char *mcml_last_error(void) { return g_last_error.c_str(); }

int mcml_device_count(int *count) {
  clear_error();
  if (!count) return set_error(MCML_E_INVALID, "null count");
  *count = 0;
  int n = 0;
  const cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return set_error(MCML_E_NODEV, std::string("cudaGetDeviceCount: ") + cudaGetErrorString(e));
  }
  *count = n;
  return MCML_OK;
}

int mcml_get_device_info(int device, mcml_device_info *info) {
  clear_error();
  if (!info) return set_error(MCML_E_INVALID, "null info");
  cudaDeviceProp p;
  CUDA_TRY(cudaGetDeviceProperties(&p, device));
  std::memset(info, 0, sizeof(*info));
  std::strncpy(info->name, p.name, sizeof(info->name) - 1);
  info->major = p.major;
  info->minor = p.minor;
  info->sm_count = p.multiProcessorCount;
  info->max_threads_per_sm = p.maxThreadsPerMultiProcessor;
  info->global_mem = p.totalGlobalMem;
  // io.cpp:487-526: 32 threads per block from CC 5.0 on, blocks/SM = max threads/SM / 32.
  const int ver = p.major * 10 + p.minor;
  const int tpb = ver < 30 ? 8 : (ver < 50 ? 16 : 32);
  info->reference_threads =
      (uint64_t)(p.maxThreadsPerMultiProcessor / tpb) * tpb * p.multiProcessorCount;
  return MCML_OK;
}

int mcml_create(const mcml_sim *sim, const mcml_opts *opts, mcml_ctx **out) {
  clear_error();
  if (!out) return set_error(MCML_E_INVALID, "null output pointer");
  *out = nullptr;
  int rc = validate_sim(sim);
  if (rc) return rc;
  mcml_opts o{};
  if (opts) o = *opts;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return set_error(MCML_E_NODEV, "no CUDA device");
  }
  if (o.device < 0 || o.device >= ndev) return set_error(MCML_E_INVALID, "GPU selection ERROR!");
  std::unique_ptr<mcml_ctx> c(new mcml_ctx());
  c->device = o.device;
  c->opts = o;
  DeviceGuard g(o.device);
  cudaDeviceProp p;
  CUDA_TRY(cudaGetDeviceProperties(&p, o.device));
  c->sm_count = p.multiProcessorCount;
  c->max_thr_sm = p.maxThreadsPerMultiProcessor;
  c->gpu_name = p.name;
  if (o.stream) {
    c->stream = (cudaStream_t)o.stream;
  } else {
    CUDA_TRY(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    c->own_stream = true;
  }
  for (auto &e : c->ev) CUDA_TRY(cudaEventCreate(&e));
  CUDA_TRY(cudaMalloc(&c->d_counters, kCntWords * sizeof(unsigned long long)));
  CUDA_TRY(cudaMalloc(&c->d_sums, 96 * sizeof(unsigned long long)));
  rc = set_sim(c.get(), sim);
  if (rc) return rc;
  uint64_t cap = o.record_capacity;
  if (!cap) {
    cap = c->N / 64;
    cap = std::max<uint64_t>(cap, 1ull << 16);
    cap = std::min<uint64_t>(cap, 1ull << 22);
  }
  rc = ensure_records(c.get(), cap);
  if (rc) return rc;
  rc = choose_walk(c.get());
  if (rc) return rc;
  c->replay_grid = 8 * c->sm_count;
  *out = c.release();
  return MCML_OK;
}

int mcml_set_sim(mcml_ctx *ctx, const mcml_sim *sim) {
  clear_error();
  if (!ctx) return set_error(MCML_E_INVALID, "null context");
  const int rc = validate_sim(sim);
  if (rc) return rc;
  int rc2 = set_sim(ctx, sim);
  if (rc2) return rc2;
  return choose_walk(ctx);
}


void mcml_destroy(mcml_ctx *ctx) { delete ctx; }

int mcml_launch_run(mcml_ctx *ctx) {
  clear_error();
  if (!ctx) return set_error(MCML_E_INVALID, "null context");
  return launch_run(ctx);
}

int mcml_get_result(mcml_ctx *ctx, mcml_result *result) {
  clear_error();
  if (!ctx) return set_error(MCML_E_INVALID, "null context");
  if (!ctx->ran) return set_error(MCML_E_STATE, "mcml_run has not been called");
  DeviceGuard g(ctx->device);
  return fill_result(ctx, result);
}

int mcml_run(mcml_ctx *ctx, mcml_result *result) {
  clear_error();
  if (!ctx) return set_error(MCML_E_INVALID, "null context");
  int rc = launch_run(ctx);
  if (rc) return rc;
  DeviceGuard g(ctx->device);
  rc = fill_result(ctx, result);
  if (rc == MCML_E_OVERFLOW) {
    // Deterministic: grow the record buffer to fit and walk again.
    unsigned long long n = 0;
    CUDA_TRY(cudaMemcpy(&n, ctx->d_counters + kCntRecords, sizeof(n), cudaMemcpyDeviceToHost));
    rc = ensure_records(ctx, n + n / 4 + 1024);
    if (rc) return rc;
    rc = launch_run(ctx);
    if (rc) return rc;
    rc = fill_result(ctx, result);
  }
  return rc;
}

int mcml_run_checkpointed(mcml_ctx *c, const mcml_checkpoint_opts *ck, mcml_result *result) {
  clear_error();
  if (!c || !ck || !ck->path || !ck->path[0]) return set_error(MCML_E_INVALID, "null argument");
  if (!c->d_slot_state || c->S > c->slot_cap)
    return set_error(MCML_E_STATE, "no simulation set: the last mcml_set_sim failed");
  DeviceGuard g(c->device);
  const std::string path = ck->path;
  const uint64_t digest = run_digest(c->sim, c->opts.seed, c->opts.slot_begin, c->S);
  CkptHeader h;
  bool exists = false;
  int rc = ckpt_read_header(path, h, exists);
  if (rc) return rc;
  if (exists) {
    if (h.run_digest != digest || h.seed != c->opts.seed || h.slot_begin != c->opts.slot_begin ||
        h.photons != c->N || h.slots != c->S)
      return set_error(MCML_E_CHECKPOINT, "checkpoint " + path +
                                              " belongs to another simulation, seed or slot layout");
  } else {
    ckpt_init(h);
    h.run_digest = digest;
    h.seed = c->opts.seed;
    h.slot_begin = c->opts.slot_begin;
    h.photons = c->N;
    h.slots = c->S;
    rc = ckpt_write_header(path, h);
    if (rc) return rc;
  }
  c->ran = c->replayed = c->host_valid = false;

  // Records so far back onto the device.
  uint64_t D = h.records;
  if (D > c->rec_cap) {
    rc = ensure_records(c, D + D / 4 + 1024);
    if (rc) return rc;
  }
  if (D) {
    std::vector<DetRecord> host(D);
    rc = ckpt_read_records(path, h, host.data());
    if (rc) return rc;
    CUDA_TRY(cudaMemcpy(c->d_records, host.data(), D * sizeof(DetRecord), cudaMemcpyHostToDevice));
  }
  CUDA_TRY(cudaMemsetAsync(c->d_sums, 0, 96 * sizeof(unsigned long long), c->stream));
  CUDA_TRY(cudaEventRecord(c->ev[0], c->stream));
  CUDA_TRY(launch_seed_slots(c->opts.seed, c->opts.slot_begin, c->S, c->d_slot_state,
                             c->sm_count, c->stream));
  CUDA_TRY(cudaEventRecord(c->ev[2], c->stream));

  const uint64_t lanes = (uint64_t)c->walk_grid * (uint64_t)c->walk_block;
  uint64_t chunk = ck->chunk_slots ? ck->chunk_slots : std::max<uint64_t>(32 * lanes, c->S / 64);
  chunk = std::max<uint64_t>(1, std::min<uint64_t>(chunk, c->S));
  uint64_t done = h.slots_done, steps = h.steps;
  uint32_t launched = 0;
  double walk_ms = 0.0;
  std::vector<DetRecord> fresh;
  while (done < c->S) {
    if (ck->max_chunks && launched >= ck->max_chunks) return MCML_INCOMPLETE;
    const uint64_t end = std::min<uint64_t>(c->S, done + chunk);
    unsigned long long cnt[kCntWords] = {};
    cnt[kCntSlot] = done;
    cnt[kCntRecords] = D;
    cnt[kCntSteps] = steps;
    CUDA_TRY(cudaMemcpyAsync(c->d_counters, cnt, sizeof(cnt), cudaMemcpyHostToDevice, c->stream));
    WalkArgs A;
    A.slot_state = c->d_slot_state;
    A.counters = c->d_counters;
    A.records = c->d_records;
    A.rec_cap = c->rec_cap;
    A.slot_end = end;
    CUDA_TRY(cudaEventRecord(c->ev[4], c->stream));
    CUDA_TRY(launch_walk(c->P, A, c->sim.source_probe_oblique != 0,
                         c->sim.detector_probe_oblique != 0, c->walk_block, c->walk_min_blocks,
                         c->walk_grid, c->stream));
    CUDA_TRY(cudaEventRecord(c->ev[1], c->stream));
    CUDA_TRY(cudaMemcpyAsync(cnt, c->d_counters, sizeof(cnt), cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (cnt[kCntRecords] > c->rec_cap) {
      // Records beyond the buffer were dropped: grow it, keep the first D,
      // walk this launch's slots again (their photons do not change).
      const uint64_t cap = cnt[kCntRecords] + cnt[kCntRecords] / 4 + 1024;
      DetRecord *bigger = nullptr;
      CUDA_TRY(cudaMalloc(&bigger, cap * sizeof(DetRecord)));
      if (D)
        CUDA_TRY(cudaMemcpy(bigger, c->d_records, D * sizeof(DetRecord), cudaMemcpyDeviceToDevice));
      dfree(c->d_records);
      c->d_records = bigger;
      c->rec_cap = cap;
      continue;
    }
    walk_ms += elapsed(c->ev[4], c->ev[1]);
    const uint64_t n = cnt[kCntRecords] - D;
    fresh.resize(n);
    if (n)
      CUDA_TRY(cudaMemcpy(fresh.data(), c->d_records + D, n * sizeof(DetRecord),
                          cudaMemcpyDeviceToHost));
    rc = ckpt_append(path, h, fresh.data(), n, end, cnt[kCntSteps]);
    if (rc) return rc;
    D = cnt[kCntRecords];
    steps = cnt[kCntSteps];
    done = end;
    ++launched;
  }
  // All slots walked: the state mcml_run leaves behind.
  {
    unsigned long long cnt[kCntWords] = {};
    cnt[kCntSlot] = c->S;
    cnt[kCntRecords] = D;
    cnt[kCntSteps] = steps;
    CUDA_TRY(cudaMemcpyAsync(c->d_counters, cnt, sizeof(cnt), cudaMemcpyHostToDevice, c->stream));
  }
  CUDA_TRY(launch_reduce_records(c->d_records, c->d_counters + kCntRecords, c->rec_cap,
                                 c->sim.num_sds, c->d_sums,
                                 reinterpret_cast<double *>(c->d_sums + 32),
                                 reinterpret_cast<double *>(c->d_sums + 64), c->sm_count,
                                 c->stream));
  c->ran = true;
  rc = fill_result(c, result);
  if (rc) return rc;
  if (result) {
    result->walk_ms = (float)walk_ms;
    result->seed_ms = elapsed(c->ev[0], c->ev[2]);
  }
  return MCML_OK;
}

int mcml_launch_replay(mcml_ctx *ctx) {
  clear_error();
  if (!ctx) return set_error(MCML_E_INVALID, "null context");
  return launch_replay(ctx);
}

int mcml_replay(mcml_ctx *ctx, mcml_result *result) {
  clear_error();
  if (!ctx) return set_error(MCML_E_INVALID, "null context");
  int rc = launch_replay(ctx);
  if (rc) return rc;
  rc = fetch_host(ctx);
  if (rc) return rc;
  if (result) {
    rc = fill_result(ctx, result);
    if (rc) return rc;
    const int L = (int)ctx->sim.num_layers;
    const double Nd = (double)ctx->N;
    for (unsigned s = 0; s < ctx->sim.num_sds; ++s) {
      double s1 = 0.0, s2 = 0.0;
      for (uint32_t i : ctx->order[s]) {
        const double w = ctx->h_rows[(size_t)i * (L + 2)];
        s1 += w;
        s2 += w * w;
      }
      result->detected[s] = ctx->order[s].size();
      result->weight_sum[s] = s1;
      result->weight_sumsq[s] = s2;
      result->reflectance[s] = s1 / ((double)0xFFFFFFFF * Nd);
      const double mean = s1 / Nd;
      double var = s2 / Nd - mean * mean;
      if (var < 0) var = 0;
      result->std_error[s] = Nd > 1 ? std::sqrt(var / (Nd - 1)) / (double)0xFFFFFFFF : 0.0;
    }
  }
  return MCML_OK;
}

int mcml_get_detections(mcml_ctx *ctx, int sds, uint64_t *photon_ids, float *weights,
                        uint64_t capacity, uint64_t *count) {
  clear_error();
  if (!ctx || !count) return set_error(MCML_E_INVALID, "null argument");
  if (sds < 1 || sds > (int)ctx->sim.num_sds) return set_error(MCML_E_INVALID, "sds out of range");
  int rc = fetch_host(ctx);
  if (rc) return rc;
  const auto &idx = ctx->order[sds - 1];
  *count = idx.size();
  const uint64_t n = std::min<uint64_t>(capacity, idx.size());
  for (uint64_t k = 0; k < n; ++k) {
    if (photon_ids) photon_ids[k] = ctx->h_rec[idx[k]].photon;
    if (weights) weights[k] = ctx->h_rec[idx[k]].weight;
  }
  return MCML_OK;
}

int mcml_get_rows(mcml_ctx *ctx, int sds, float *rows, uint32_t *interactions, uint64_t capacity,
                  uint64_t *count) {
  clear_error();
  if (!ctx || !count) return set_error(MCML_E_INVALID, "null argument");
  if (sds < 1 || sds > (int)ctx->sim.num_sds) return set_error(MCML_E_INVALID, "sds out of range");
  if (!ctx->replayed) return set_error(MCML_E_STATE, "mcml_replay has not been called");
  int rc = fetch_host(ctx);
  if (rc) return rc;
  const int L = (int)ctx->sim.num_layers;
  const auto &idx = ctx->order[sds - 1];
  *count = idx.size();
  const uint64_t n = std::min<uint64_t>(capacity, idx.size());
  for (uint64_t k = 0; k < n; ++k) {
    if (rows)
      std::memcpy(rows + k * (L + 2), &ctx->h_rows[(size_t)idx[k] * (L + 2)],
                  (L + 2) * sizeof(float));
    if (interactions)
      std::memcpy(interactions + k * L, &ctx->h_inter[(size_t)idx[k] * L], L * sizeof(uint32_t));
  }
  return MCML_OK;
}

int mcml_get_tallies(mcml_ctx *ctx, uint64_t *A_rz, uint64_t *A0_z) {
  clear_error();
  if (!ctx) return set_error(MCML_E_INVALID, "null context");
  if (!ctx->replayed) return set_error(MCML_E_STATE, "mcml_replay has not been called");
  DeviceGuard g(ctx->device);
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  if (A_rz)
    CUDA_TRY(cudaMemcpy(A_rz, ctx->d_Arz, ctx->arz_n * sizeof(uint64_t), cudaMemcpyDeviceToHost));
  if (A0_z)
    CUDA_TRY(cudaMemcpy(A0_z, ctx->d_A0z, ctx->a0z_n * sizeof(uint64_t), cudaMemcpyDeviceToHost));
  return MCML_OK;
}

int mcml_get_device_outputs(mcml_ctx *ctx, mcml_device_outputs *out) {
  clear_error();
  if (!ctx || !out) return set_error(MCML_E_INVALID, "null argument");
  DeviceGuard g(ctx->device);
  uint64_t D = 0;
  OrderedOutput o;
  int rc = order_on_device(ctx, &D, &o);
  if (rc) return rc;
  std::memset(out, 0, sizeof(*out));
  unsigned long long cnt[32];
  CUDA_TRY(cudaMemcpyAsync(cnt, ctx->d_sums, sizeof(cnt), cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  for (unsigned s = 0; s < ctx->sim.num_sds; ++s) out->detected[s] = cnt[s];
  out->records = o.records;
  out->n_records = D;
  out->row_len = ctx->sim.num_layers + 2;
  out->photons = ctx->N;
  if (ctx->replayed) {
    out->rows = o.rows;
    out->A_rz = reinterpret_cast<const uint64_t *>(ctx->d_Arz);
    out->A0_z = reinterpret_cast<const uint64_t *>(ctx->d_A0z);
    out->arz_count = ctx->arz_n;
    out->a0z_count = ctx->a0z_n;
  }
  out->stream = ctx->stream;
  return MCML_OK;
}

int mcml_average_pathlength(mcml_ctx *ctx, double *out) {
  clear_error();
  if (!ctx || !out) return set_error(MCML_E_INVALID, "null argument");
  if (!ctx->replayed) return set_error(MCML_E_STATE, "mcml_replay has not been called");
  int rc = fetch_host(ctx);
  if (rc) return rc;
  HostOutputs o;
  std::vector<unsigned long long> arz, a0z;
  build_outputs(ctx, o, arz, a0z);
  std::vector<double> avg;
  average_pathlength(o, avg);
  std::copy(avg.begin(), avg.end(), out);
  return MCML_OK;
}

int mcml_write_outputs(mcml_ctx *ctx, const char *dir, const char *output_txt, uint32_t flags,
                       double sim_s, double replay_s) {
  clear_error();
  if (!ctx || !output_txt) return set_error(MCML_E_INVALID, "null argument");
  const bool replay = (flags & MCML_OUT_REPLAY) != 0;
  if (replay && !ctx->replayed) return set_error(MCML_E_STATE, "mcml_replay has not been called");
  int rc = fetch_host(ctx);
  if (rc) return rc;
  HostOutputs o;
  std::vector<unsigned long long> arz, a0z;
  if (replay && (flags & MCML_OUT_ABSORBANCE)) {
    arz.resize(ctx->arz_n);
    a0z.resize(ctx->a0z_n);
    rc = mcml_get_tallies(ctx, reinterpret_cast<uint64_t *>(arz.data()),
                          reinterpret_cast<uint64_t *>(a0z.data()));
    if (rc) return rc;
  }
  build_outputs(ctx, o, arz, a0z);
  o.replayed = replay;
  return write_files(o, dir ? dir : "", output_txt, flags, sim_s, replay_s);
}

int mcml_uniform_stream(int device, uint64_t seed, uint64_t subsequence, uint64_t count,
                        float *out) {
  clear_error();
  if (!out && count) return set_error(MCML_E_INVALID, "null output");
  if (count == 0) return MCML_OK;
  DeviceGuard g(device);
  float *d = nullptr;
  CUDA_TRY(cudaMalloc(&d, count * sizeof(float)));
  cudaError_t e = launch_uniform_stream(seed, subsequence, count, d, nullptr);
  if (e == cudaSuccess) e = cudaMemcpy(out, d, count * sizeof(float), cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess)
    return set_error(MCML_E_CUDA, std::string("uniform stream: ") + cudaGetErrorString(e));
  return MCML_OK;
}

}  // extern "C"
