// batch.cu -- many tissue parameter sets in one persistent launch.
//
// The reference runs one simulation per launch sequence and its multi-set
// mode is broken (critical_arr is only allocated for the first
// simulation, io.cpp:193-197); a batch of parameter sets there means one
// process per set.  Here all sets share one persistent walk launch:
//
//   * set b has N_b photons on S_b = ceil(N_b / photons_per_slot) slots; its
//     slot s owns XORWOW subsequence s of seed_b = seed + b, exactly as a
//     single-set run with that seed and slot count, so a set's result in a
//     batch equals its result alone;
//   * global slot index = set_slot_begin[b] + s; lanes take global slots
//     from one cursor, find the set by binary search over the prefix array
//     and walk with that set's tables, read from global memory through L1
//     (a block's lanes walk many sets at once, so the tables cannot all sit
//     in shared memory);
//   * detections are summed per set and SDS (count, FP64 sum, sum of
//     squares) -- no records, no replay;
//   * the memsets, the seeding and the walk are captured once into a CUDA
//     graph and relaunched with one cudaGraphLaunch per run.
//
// The launch shape and photons per slot come from a small autotuner that
// times pilot runs of a scaled copy of the batch.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/mcml_b200.h"
#include "internal.h"
#include "kernels.h"
#include "params.h"
#include "photon.cuh"

namespace mcml {
namespace {

struct BatchSet {
  uint64_t num_photons;
  uint64_t num_slots;
  uint64_t slot_begin;  // global index of the set's first slot
  uint64_t seed;
  float start_weight;
  float det_reflectance;
  int32_t n_layers;
  int32_t n_sds;
};

struct BatchArgs {
  const SmemTables *tables;  // [B], in global memory
  const BatchSet *sets;      // [B]
  const uint64_t *slot_prefix;  // [B+1]: global slot index where each set begins
  const uint2 *slot_state;   // [total slots x 3]
  unsigned long long *cursor;
  unsigned long long *det_count;  // [B x 32]
  double *wsum;                   // [B x 32]
  double *wsq;                    // [B x 32]
  unsigned long long *steps;      // [B]
  uint64_t total_slots;
  int num_sets;
};

__device__ __forceinline__ int find_set(const uint64_t *prefix, int B, uint64_t g) {
  int lo = 0, hi = B;  // prefix[lo] <= g < prefix[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (prefix[mid] <= g) lo = mid; else hi = mid;
  }
  return lo;
}

// Per-set tables built on the device (the reference evaluates the probe
// trigonometry on the device): one block per set.
__global__ void batch_tables_kernel(const DevParams *params, SmemTables *tables) {
  load_tables(tables[blockIdx.x], params[blockIdx.x]);
}

// Seeds runs of consecutive global slots: curand_init at the start of a run
// and at every set boundary, skipahead_sequence(1) otherwise.
__global__ void batch_seed_kernel(const BatchSet *sets, const uint64_t *prefix, int B,
                                  uint64_t total, uint64_t run, uint2 *out) {
  const uint64_t g0 = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) * run;
  if (g0 >= total) return;
  const uint64_t g1 = g0 + run < total ? g0 + run : total;
  int b = find_set(prefix, B, g0);
  curandStateXORWOW st;
  curand_init(sets[b].seed, g0 - prefix[b], 0, &st);
  for (uint64_t g = g0;;) {
    out[g * 3 + 0] = make_uint2(st.d, st.v[0]);
    out[g * 3 + 1] = make_uint2(st.v[1], st.v[2]);
    out[g * 3 + 2] = make_uint2(st.v[3], st.v[4]);
    if (++g >= g1) break;
    if (g >= prefix[b + 1]) {
      while (g >= prefix[b + 1]) ++b;
      curand_init(sets[b].seed, g - prefix[b], 0, &st);
    } else {
      skipahead_sequence(1ull, &st);
    }
  }
}

// kGlass: some set has a tissue layer with mutr == FLT_MAX (see walk_step).
template <int kBlock, int kMinBlocks, bool kSrcOblique, bool kDetOblique, bool kGlass>
__global__ void __launch_bounds__(kBlock, kMinBlocks) batch_walk_kernel(const BatchArgs A) {
  curandStateXORWOW st;
  st.boxmuller_flag = 0;
  st.boxmuller_flag_double = 0;
  st.boxmuller_extra = 0.0f;
  st.boxmuller_extra_double = 0.0;
  Photon p;
  int b = 0;
  uint32_t k = 0, quota = 0, steps_acc = 0;
  int n_layers = 0, n_sds = 0;
  float start_w = 0.0f, det_refl = 0.0f;
  const SmemTables *tp = nullptr;

  auto next_slot = [&]() -> bool {
    const uint64_t g = atomicAdd(A.cursor, 1ull);
    if (g >= A.total_slots) return false;
    const int nb = find_set(A.slot_prefix, A.num_sets, g);
    if (nb != b || tp == nullptr) {
      b = nb;
      const BatchSet &bs = A.sets[b];
      n_layers = bs.n_layers;
      n_sds = bs.n_sds;
      start_w = bs.start_weight;
      det_refl = bs.det_reflectance;
      tp = &A.tables[b];
    }
    const BatchSet &bs = A.sets[b];
    const uint64_t s = g - A.slot_prefix[b];
    const uint64_t q = bs.num_photons / bs.num_slots;
    const uint64_t rem = bs.num_photons % bs.num_slots;
    const uint2 x = A.slot_state[g * 3 + 0], y = A.slot_state[g * 3 + 1],
                z = A.slot_state[g * 3 + 2];
    st.d = x.x;
    st.v[0] = x.y;
    st.v[1] = y.x;
    st.v[2] = y.y;
    st.v[3] = z.x;
    st.v[4] = z.y;
    k = 0;
    quota = (uint32_t)(q + (s < rem ? 1 : 0));
    return true;
  };

  if (!next_slot()) return;
  launch_photon<kSrcOblique>(p, &st, *tp, start_w);
  for (;;) {
    const int base = b * 32;
    const bool alive = walk_step<kDetOblique, kGlass>(p, st, *tp, n_layers, n_sds, det_refl,
                                              [&](int i, float w) {
                                                atomicAdd(&A.det_count[base + i], 1ull);
                                                atomicAdd(&A.wsum[base + i], (double)w);
                                                atomicAdd(&A.wsq[base + i],
                                                          (double)w * (double)w);
                                              });
    if (!alive) {
      steps_acc += (uint32_t)p.steps;
      const int prev_b = b;
      const bool slot_done = ++k >= quota;
      if (slot_done || steps_acc >= 0x40000000u) {
        atomicAdd(&A.steps[prev_b], (unsigned long long)steps_acc);
        steps_acc = 0;
      }
      if (slot_done && !next_slot()) break;
      launch_photon<kSrcOblique>(p, &st, *tp, start_w);
    }
  }
}

struct Variant {
  int block, min_blocks;
  const void *fn[8];  // [glass*4 + src_oblique*2 + det_oblique]
};

template <int B, int M>
Variant make_variant() {
  return Variant{B, M,
                 {(const void *)batch_walk_kernel<B, M, false, false, false>,
                  (const void *)batch_walk_kernel<B, M, false, true, false>,
                  (const void *)batch_walk_kernel<B, M, true, false, false>,
                  (const void *)batch_walk_kernel<B, M, true, true, false>,
                  (const void *)batch_walk_kernel<B, M, false, false, true>,
                  (const void *)batch_walk_kernel<B, M, false, true, true>,
                  (const void *)batch_walk_kernel<B, M, true, false, true>,
                  (const void *)batch_walk_kernel<B, M, true, true, true>}};
}

const std::vector<Variant> &variants() {
  static const std::vector<Variant> v = {make_variant<128, 8>(), make_variant<128, 1>(),
                                         make_variant<256, 4>(), make_variant<256, 1>()};
  return v;
}

#define BATCH_TRY(expr)                                                                  \
  do {                                                                                   \
    cudaError_t e_ = (expr);                                                             \
    if (e_ != cudaSuccess)                                                               \
      return set_error(MCML_E_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
  } while (0)

template <class T>
void dfree(T *&p) {
  if (p) cudaFree(p);
  p = nullptr;
}

}  // namespace
}  // namespace mcml

using namespace mcml;

struct mcml_batch {
  int device = 0;
  int sm_count = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int B = 0;
  int variant_kind = 0;  // glass*4 + src_oblique*2 + det_oblique
  std::vector<mcml_sim> sims;
  std::vector<DevParams> params;
  std::vector<BatchSet> sets;
  std::vector<uint64_t> prefix;
  uint64_t seed = 0;
  uint32_t photons_per_slot = 64;
  int variant = 0;  // index into variants()
  int grid = 0;
  bool use_graph = true;
  // device
  DevParams *d_params = nullptr;
  SmemTables *d_tables = nullptr;
  BatchSet *d_sets = nullptr;
  uint64_t *d_prefix = nullptr;
  uint2 *d_state = nullptr;
  uint64_t state_cap = 0;
  unsigned long long *d_cursor = nullptr;
  unsigned long long *d_count = nullptr;
  double *d_wsum = nullptr, *d_wsq = nullptr;
  unsigned long long *d_steps = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  bool launched = false;

  ~mcml_batch() {
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != device) cudaSetDevice(device);
    if (stream) cudaStreamSynchronize(stream);
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    dfree(d_params);
    dfree(d_tables);
    dfree(d_sets);
    dfree(d_prefix);
    dfree(d_state);
    dfree(d_cursor);
    dfree(d_count);
    dfree(d_wsum);
    dfree(d_wsq);
    dfree(d_steps);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (own_stream && stream) cudaStreamDestroy(stream);
    if (prev >= 0 && prev != device) cudaSetDevice(prev);
  }
};

namespace {

struct BatchDeviceGuard {
  int prev = -1;
  bool changed = false;
  explicit BatchDeviceGuard(int dev) {
    if (cudaGetDevice(&prev) == cudaSuccess && prev != dev) changed = cudaSetDevice(dev) == cudaSuccess;
  }
  ~BatchDeviceGuard() {
    if (changed) cudaSetDevice(prev);
  }
};

// Lays out the slots for the current photons_per_slot and (re)allocates the
// slot states; drops a captured graph that referenced the old layout.
int layout(mcml_batch *b) {
  b->prefix.assign(b->B + 1, 0);
  for (int i = 0; i < b->B; ++i) {
    const uint64_t N = b->sims[i].number_photons;
    uint64_t S = (N + b->photons_per_slot - 1) / b->photons_per_slot;
    if (S < 1) S = 1;
    if (N / S >= 0xFFFFFFFFull) return set_error(MCML_E_INVALID, "too many photons per slot");
    b->sets[i].num_slots = S;
    b->sets[i].slot_begin = b->prefix[i];
    b->prefix[i + 1] = b->prefix[i] + S;
    b->params[i].num_slots = S;
  }
  const uint64_t total = b->prefix[b->B];
  BatchDeviceGuard g(b->device);
  if (total > b->state_cap) {
    dfree(b->d_state);
    b->state_cap = 0;
    BATCH_TRY(cudaMalloc(&b->d_state, total * 3 * sizeof(uint2)));
    b->state_cap = total;
  }
  BATCH_TRY(cudaMemcpy(b->d_sets, b->sets.data(), b->B * sizeof(BatchSet), cudaMemcpyHostToDevice));
  BATCH_TRY(cudaMemcpy(b->d_prefix, b->prefix.data(), (b->B + 1) * sizeof(uint64_t),
                       cudaMemcpyHostToDevice));
  if (b->exec) {
    cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
  }
  if (b->graph) {
    cudaGraphDestroy(b->graph);
    b->graph = nullptr;
  }
  return MCML_OK;
}

int choose_grid(mcml_batch *b) {
  const Variant &v = variants()[b->variant];
  int nb = 0;
  BatchDeviceGuard g(b->device);
  BATCH_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, v.fn[b->variant_kind], v.block, 0));
  b->grid = std::max(nb, 1) * b->sm_count;
  return MCML_OK;
}

// Enqueues one batch run on the stream (captured into the graph when enabled).
int enqueue(mcml_batch *b) {
  const uint64_t total = b->prefix[b->B];
  BATCH_TRY(cudaMemsetAsync(b->d_cursor, 0, sizeof(unsigned long long), b->stream));
  BATCH_TRY(cudaMemsetAsync(b->d_count, 0, (size_t)b->B * 32 * sizeof(unsigned long long), b->stream));
  BATCH_TRY(cudaMemsetAsync(b->d_wsum, 0, (size_t)b->B * 32 * sizeof(double), b->stream));
  BATCH_TRY(cudaMemsetAsync(b->d_wsq, 0, (size_t)b->B * 32 * sizeof(double), b->stream));
  BATCH_TRY(cudaMemsetAsync(b->d_steps, 0, (size_t)b->B * sizeof(unsigned long long), b->stream));
  const uint64_t threads = (uint64_t)b->sm_count * 2048;
  const uint64_t run = (total + threads - 1) / threads;
  const uint64_t used = (total + run - 1) / run;
  batch_seed_kernel<<<(unsigned)((used + 255) / 256), 256, 0, b->stream>>>(
      b->d_sets, b->d_prefix, b->B, total, run, b->d_state);
  BATCH_TRY(cudaGetLastError());
  BatchArgs A;
  A.tables = b->d_tables;
  A.sets = b->d_sets;
  A.slot_prefix = b->d_prefix;
  A.slot_state = b->d_state;
  A.cursor = b->d_cursor;
  A.det_count = b->d_count;
  A.wsum = b->d_wsum;
  A.wsq = b->d_wsq;
  A.steps = b->d_steps;
  A.total_slots = total;
  A.num_sets = b->B;
  const Variant &v = variants()[b->variant];
  void *args[] = {(void *)&A};
  BATCH_TRY(cudaLaunchKernel(v.fn[b->variant_kind], dim3(b->grid), dim3(v.block), args, 0, b->stream));
  return MCML_OK;
}

int launch(mcml_batch *b) {
  BatchDeviceGuard g(b->device);
  BATCH_TRY(cudaEventRecord(b->ev0, b->stream));
  if (b->use_graph) {
    if (!b->exec) {
      BATCH_TRY(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
      const int rc = enqueue(b);
      cudaGraph_t graph = nullptr;
      const cudaError_t e = cudaStreamEndCapture(b->stream, &graph);
      if (rc) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
      }
      BATCH_TRY(e);
      b->graph = graph;
      BATCH_TRY(cudaGraphInstantiate(&b->exec, b->graph, 0));
    }
    BATCH_TRY(cudaGraphLaunch(b->exec, b->stream));
  } else {
    const int rc = enqueue(b);
    if (rc) return rc;
  }
  BATCH_TRY(cudaEventRecord(b->ev1, b->stream));
  b->launched = true;
  return MCML_OK;
}

int collect(mcml_batch *b, mcml_result *results) {
  BatchDeviceGuard g(b->device);
  BATCH_TRY(cudaStreamSynchronize(b->stream));
  if (!results) return MCML_OK;
  const size_t n = (size_t)b->B * 32;
  std::vector<unsigned long long> cnt(n), steps(b->B);
  std::vector<double> s1(n), s2(n);
  BATCH_TRY(cudaMemcpy(cnt.data(), b->d_count, n * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
  BATCH_TRY(cudaMemcpy(s1.data(), b->d_wsum, n * sizeof(double), cudaMemcpyDeviceToHost));
  BATCH_TRY(cudaMemcpy(s2.data(), b->d_wsq, n * sizeof(double), cudaMemcpyDeviceToHost));
  BATCH_TRY(cudaMemcpy(steps.data(), b->d_steps, b->B * sizeof(unsigned long long),
                       cudaMemcpyDeviceToHost));
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, b->ev0, b->ev1);
  for (int i = 0; i < b->B; ++i) {
    mcml_result &r = results[i];
    std::memset(&r, 0, sizeof(r));
    r.num_sds = b->sims[i].num_sds;
    r.photons = b->sims[i].number_photons;
    r.slots = b->sets[i].num_slots;
    r.steps = steps[i];
    r.walk_ms = ms;
    const double Nd = (double)r.photons;
    for (unsigned s = 0; s < r.num_sds; ++s) {
      const size_t k = (size_t)i * 32 + s + 1;
      r.detected[s] = cnt[k];
      r.weight_sum[s] = s1[k];
      r.weight_sumsq[s] = s2[k];
      r.reflectance[s] = s1[k] / ((double)0xFFFFFFFF * Nd);
      const double mean = s1[k] / Nd;
      double var = s2[k] / Nd - mean * mean;
      if (var < 0) var = 0;
      r.std_error[s] = Nd > 1 ? std::sqrt(var / (Nd - 1)) / (double)0xFFFFFFFF : 0.0;
    }
  }
  return MCML_OK;
}

}  // namespace

extern "C" {

int mcml_batch_create(const mcml_sim *sims, int num_sets, const mcml_batch_opts *opts,
                      mcml_batch **out) {
  clear_error();
  if (!out || !sims || num_sets < 1) return set_error(MCML_E_INVALID, "mcml_batch_create: bad arguments");
  *out = nullptr;
  mcml_batch_opts o{};
  if (opts) o = *opts;
  for (int i = 0; i < num_sets; ++i) {
    const int rc = validate_sim(&sims[i]);
    if (rc) return set_error(rc, "set " + std::to_string(i) + ": " + mcml_last_error());
    if (sims[i].source_probe_oblique != sims[0].source_probe_oblique ||
        sims[i].detector_probe_oblique != sims[0].detector_probe_oblique)
      return set_error(MCML_E_INVALID, "all sets of a batch need the same source/detector modes");
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return set_error(MCML_E_NODEV, "no CUDA device");
  }
  if (o.device < 0 || o.device >= ndev) return set_error(MCML_E_INVALID, "GPU selection ERROR!");
  std::unique_ptr<mcml_batch> b(new mcml_batch());
  b->device = o.device;
  BatchDeviceGuard g(o.device);
  BATCH_TRY(cudaDeviceGetAttribute(&b->sm_count, cudaDevAttrMultiProcessorCount, o.device));
  b->B = num_sets;
  b->seed = o.seed;
  b->photons_per_slot = o.photons_per_slot ? o.photons_per_slot : 64;
  b->use_graph = !o.no_graph;
  b->variant_kind = (sims[0].source_probe_oblique ? 2 : 0) + (sims[0].detector_probe_oblique ? 1 : 0);
  b->sims.assign(sims, sims + num_sets);
  b->params.resize(num_sets);
  b->sets.resize(num_sets);
  for (int i = 0; i < num_sets; ++i) {
    mcml_derived der;
    const int rc = derive(&sims[i], &der);
    if (rc) return rc;
    fill_dev_params(sims[i], der, sims[i].number_photons, 1, b->params[i]);
    if (has_glass_layer(b->params[i])) b->variant_kind |= 4;
    BatchSet &s = b->sets[i];
    s.num_photons = sims[i].number_photons;
    s.seed = o.seed + (uint64_t)i;
    s.start_weight = der.start_weight;
    s.det_reflectance = sims[i].detector_reflectance;
    s.n_layers = (int32_t)sims[i].num_layers;
    s.n_sds = (int32_t)sims[i].num_sds;
  }
  if (o.stream) {
    b->stream = (cudaStream_t)o.stream;
  } else {
    BATCH_TRY(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    b->own_stream = true;
  }
  BATCH_TRY(cudaEventCreate(&b->ev0));
  BATCH_TRY(cudaEventCreate(&b->ev1));
  BATCH_TRY(cudaMalloc(&b->d_params, num_sets * sizeof(DevParams)));
  BATCH_TRY(cudaMalloc(&b->d_tables, num_sets * sizeof(SmemTables)));
  BATCH_TRY(cudaMalloc(&b->d_sets, num_sets * sizeof(BatchSet)));
  BATCH_TRY(cudaMalloc(&b->d_prefix, (num_sets + 1) * sizeof(uint64_t)));
  BATCH_TRY(cudaMalloc(&b->d_cursor, sizeof(unsigned long long)));
  BATCH_TRY(cudaMalloc(&b->d_count, (size_t)num_sets * 32 * sizeof(unsigned long long)));
  BATCH_TRY(cudaMalloc(&b->d_wsum, (size_t)num_sets * 32 * sizeof(double)));
  BATCH_TRY(cudaMalloc(&b->d_wsq, (size_t)num_sets * 32 * sizeof(double)));
  BATCH_TRY(cudaMalloc(&b->d_steps, (size_t)num_sets * sizeof(unsigned long long)));
  BATCH_TRY(cudaMemcpy(b->d_params, b->params.data(), num_sets * sizeof(DevParams),
                       cudaMemcpyHostToDevice));
  batch_tables_kernel<<<num_sets, 64>>>(b->d_params, b->d_tables);
  BATCH_TRY(cudaGetLastError());
  BATCH_TRY(cudaDeviceSynchronize());
  b->variant = 0;
  for (size_t v = 0; v < variants().size(); ++v)
    if (o.block_size && variants()[v].block == (int)o.block_size &&
        (!o.blocks_per_sm || variants()[v].min_blocks == (int)o.blocks_per_sm))
      b->variant = (int)v;
  int rc = layout(b.get());
  if (rc) return rc;
  rc = choose_grid(b.get());
  if (rc) return rc;
  *out = b.release();
  return MCML_OK;
}

int mcml_batch_autotune(mcml_batch *b, double photon_fraction, mcml_batch_tuning *chosen) {
  clear_error();
  if (!b) return set_error(MCML_E_INVALID, "null batch");
  if (!(photon_fraction > 0 && photon_fraction <= 1)) photon_fraction = 1.0 / 16;
  // Pilot: the same sets with a fraction of their photons.
  std::vector<mcml_sim> pilot = b->sims;
  for (auto &s : pilot) {
    s.number_photons = (uint64_t)std::max(1.0, std::floor(s.number_photons * photon_fraction));
  }
  mcml_batch_opts o{};
  o.device = b->device;
  o.seed = b->seed;
  o.stream = b->stream;
  o.no_graph = 1;
  const uint32_t pps[] = {4, 8, 32};
  double best = 1e300;
  int best_v = b->variant;
  uint32_t best_pps = b->photons_per_slot;
  mcml_batch *p = nullptr;
  int rc = mcml_batch_create(pilot.data(), (int)pilot.size(), &o, &p);
  if (rc) return rc;
  std::unique_ptr<mcml_batch> guard(p);
  for (size_t v = 0; v < variants().size(); ++v) {
    for (uint32_t q : pps) {
      p->variant = (int)v;
      p->photons_per_slot = q;
      rc = layout(p);
      if (rc) return rc;
      rc = choose_grid(p);
      if (rc) return rc;
      rc = launch(p);  // warm-up (first launch of this shape)
      if (rc) return rc;
      rc = launch(p);
      if (rc) return rc;
      rc = collect(p, nullptr);
      if (rc) return rc;
      float ms = 0.0f;
      cudaEventElapsedTime(&ms, p->ev0, p->ev1);
      if (ms < best) {
        best = ms;
        best_v = (int)v;
        best_pps = q;
      }
    }
  }
  b->variant = best_v;
  b->photons_per_slot = best_pps;
  rc = layout(b);
  if (rc) return rc;
  rc = choose_grid(b);
  if (rc) return rc;
  if (chosen) {
    chosen->block_size = (uint32_t)variants()[best_v].block;
    chosen->blocks_per_sm = (uint32_t)variants()[best_v].min_blocks;
    chosen->photons_per_slot = best_pps;
    chosen->pilot_ms = (float)best;
  }
  return MCML_OK;
}

int mcml_batch_launch(mcml_batch *b) {
  clear_error();
  if (!b) return set_error(MCML_E_INVALID, "null batch");
  return launch(b);
}

int mcml_batch_get_results(mcml_batch *b, mcml_result *results) {
  clear_error();
  if (!b) return set_error(MCML_E_INVALID, "null batch");
  if (!b->launched) return set_error(MCML_E_STATE, "mcml_batch_launch has not been called");
  return collect(b, results);
}

int mcml_batch_run(mcml_batch *b, mcml_result *results) {
  clear_error();
  if (!b) return set_error(MCML_E_INVALID, "null batch");
  int rc = launch(b);
  if (rc) return rc;
  return collect(b, results);
}

void mcml_batch_destroy(mcml_batch *b) { delete b; }

}  // extern "C"
