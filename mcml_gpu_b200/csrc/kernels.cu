// kernels.cu -- the walk, replay and support kernels (sm_100a).
//
// Scheduling model (this library's, not the reference's):
//   * N photons are split over S "slots".  Slot s owns the XORWOW
//     subsequence s (curand_init(seed, s, 0)) and walks photons
//     s*q+min(s,r) ... in order, each starting where the previous one's
//     draws ended -- exactly what the reference's thread s does
//     (transport.cu:442-451, 733), but with a fixed count per slot
//     (q or q+1), so the result is deterministic.  With S equal to the
//     reference's thread count and N == S, slot s walks precisely the
//     photon the reference's thread s walks.
//   * The walk is one persistent launch.  Each lane takes slots from a
//     global cursor (one warp-aggregated atomic per group of lanes) and
//     relaunches its next photon the moment the current one dies, so no
//     lane idles until the slot queue is empty.  The host loop of
//     50000-step launches and the per-launch copies of the reference
//     (transport.cu:114-147) are gone.
//   * Detections are appended to one global record buffer; the replay
//     re-walks each record from its saved XORWOW state, again with
//     per-lane dynamic work fetching.
#include <cfloat>
#include <cstdint>
#include <cuda_runtime.h>

#include "kernels.h"
#include "photon.cuh"

namespace mcml {

namespace {

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }

// Warp-aggregated fetch-and-add of 1 per calling lane on *ctr.
__device__ __forceinline__ unsigned long long fetch_one(unsigned long long *ctr) {
  const unsigned mask = __activemask();
  const int leader = __ffs(mask) - 1;
  const unsigned rank = __popc(mask & ((1u << lane_id()) - 1u));
  unsigned long long base = 0;
  if ((int)lane_id() == leader) base = atomicAdd(ctr, (unsigned long long)__popc(mask));
  base = __shfl_sync(mask, base, leader);
  return base + rank;
}

__device__ __forceinline__ void load_state(curandStateXORWOW &st, const uint2 *slot_state,
                                           uint64_t slot) {
  const uint2 a = slot_state[slot * 3 + 0];
  const uint2 b = slot_state[slot * 3 + 1];
  const uint2 c = slot_state[slot * 3 + 2];
  st.d = a.x;
  st.v[0] = a.y;
  st.v[1] = b.x;
  st.v[2] = b.y;
  st.v[3] = c.x;
  st.v[4] = c.y;
}

__device__ __forceinline__ void clear_gauss(curandStateXORWOW &st) {
  st.boxmuller_flag = 0;
  st.boxmuller_flag_double = 0;
  st.boxmuller_extra = 0.0f;
  st.boxmuller_extra_double = 0.0;
}

// The XORWOW state at the launch of each lane's current photon, kept in
// shared memory (written once per photon, read only on a detection).
template <int kBlock>
struct SeedStore {
  uint32_t w[6][kBlock];
  // per-thread slot bookkeeping, touched only when a photon starts or ends
  // or is detected, so it lives here instead of in registers
  uint32_t slot[kBlock], k[kBlock], quota[kBlock], steps[kBlock];
  __device__ __forceinline__ void save(const curandStateXORWOW &st) {
    const int t = threadIdx.x;
    w[0][t] = st.d;
    w[1][t] = st.v[0];
    w[2][t] = st.v[1];
    w[3][t] = st.v[2];
    w[4][t] = st.v[3];
    w[5][t] = st.v[4];
  }
};

template <int kBlock>
__device__ __forceinline__ void append_record(const WalkArgs &A, uint64_t photon, int sds,
                                              float w, const SeedStore<kBlock> &sc) {
  const unsigned long long idx = atomicAdd(&A.counters[kCntRecords], 1ull);
  if (idx < A.rec_cap) {
    const int t = threadIdx.x;
    DetRecord r;
    r.photon = photon;
    r.sds = (uint32_t)sds;
    r.weight = w;
    r.d = sc.w[0][t];
    r.v[0] = sc.w[1][t];
    r.v[1] = sc.w[2][t];
    r.v[2] = sc.w[3][t];
    r.v[3] = sc.w[4][t];
    r.v[4] = sc.w[5][t];
    A.records[idx] = r;
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// Slot seeding: state of subsequence s at offset 0 (LaunchPhoton_Global's
// curand_init, transport.cu:733), 24 bytes per slot.  Each thread seeds a
// run of consecutive slots: curand_init for the first, then
// skipahead_sequence(1) -- one precomputed-matrix step of 2^67 draws --
// for each next one, which is far cheaper than a full curand_init.
__global__ void seed_slots_kernel(uint64_t seed, uint64_t slot_begin, uint64_t num_slots,
                                  uint64_t run, uint2 *out) {
  const uint64_t s0 = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) * run;
  if (s0 >= num_slots) return;
  const uint64_t s1 = s0 + run < num_slots ? s0 + run : num_slots;
  curandStateXORWOW st;
  curand_init(seed, slot_begin + s0, 0, &st);
  for (uint64_t s = s0;;) {
    out[s * 3 + 0] = make_uint2(st.d, st.v[0]);
    out[s * 3 + 1] = make_uint2(st.v[1], st.v[2]);
    out[s * 3 + 2] = make_uint2(st.v[3], st.v[4]);
    if (++s >= s1) break;
    skipahead_sequence(1ull, &st);
  }
}

// ---------------------------------------------------------------------------
// First pass (MCd, transport.cu:341-471).
// kGlass: some tissue layer has mutr == FLT_MAX (see walk_step).
template <int kBlock, int kMinBlocks, bool kSrcOblique, bool kDetOblique, bool kGlass>
__global__ void __launch_bounds__(kBlock, kMinBlocks)
    walk_kernel(const __grid_constant__ DevParams P, const WalkArgs A) {
  __shared__ SmemTables t;
  __shared__ SeedStore<kBlock> sc;
  __shared__ uint64_t s_q, s_rem;  // photons per slot; slots with one more
  if (threadIdx.x == 0) {
    s_q = P.num_photons / P.num_slots;
    s_rem = P.num_photons % P.num_slots;
  }
  load_tables(t, P);
  __syncthreads();
  const int tid = threadIdx.x;

  curandStateXORWOW st;
  clear_gauss(st);
  Photon p;
  sc.steps[tid] = 0;

  auto next_slot = [&]() -> bool {
    const uint64_t s = fetch_one(&A.counters[kCntSlot]);
    if (s >= A.slot_end) return false;
    sc.slot[tid] = (uint32_t)s;  // slots < 2^32
    load_state(st, A.slot_state, s);
    sc.k[tid] = 0;
    sc.quota[tid] = (uint32_t)(s_q + (s < s_rem ? 1 : 0));
    return true;
  };
  auto photon_index = [&]() -> uint64_t {
    const uint64_t s = sc.slot[tid];
    return s * s_q + (s < s_rem ? s : s_rem) + sc.k[tid];
  };

  if (!next_slot()) return;
  sc.save(st);
  launch_photon<kSrcOblique>(p, &st, t, P.start_weight);

  for (;;) {
    const bool alive = walk_step<kDetOblique, kGlass>(
        p, st, t, (int)P.n_layers, (int)P.n_sds, P.det_reflectance,
        [&](int i, float w) { append_record(A, photon_index(), i, w, sc); });
    if (!alive) {
      const uint32_t acc = sc.steps[tid] + (uint32_t)p.steps;  // with the photon that just ended
      const uint32_t kk = ++sc.k[tid];
      const bool slot_done = kk >= sc.quota[tid];
      if (slot_done || acc >= 0x40000000u) {
        atomicAdd(&A.counters[kCntSteps], (unsigned long long)acc);
        sc.steps[tid] = 0;
      } else {
        sc.steps[tid] = acc;
      }
      if (slot_done && !next_slot()) break;
      sc.save(st);
      launch_photon<kSrcOblique>(p, &st, t, P.start_weight);
    }
  }
}

// ---------------------------------------------------------------------------
// Replay (MCd_replay, transport.cu:473-622) of every detection record.
template <int kBlock, bool kSrcOblique, bool kDetOblique, bool kRefGrid>
__global__ void __launch_bounds__(kBlock) replay_kernel(const __grid_constant__ DevParams P,
                                                        const ReplayArgs A) {
  __shared__ SmemTables t;
  __shared__ float s_pl[kMaxLayers][kBlock];
  __shared__ uint32_t s_ni[kMaxLayers][kBlock];
  load_tables(t, P);
  __syncthreads();

  const unsigned long long total = *A.rec_count;
  const uint64_t D = total < A.rec_cap ? total : A.rec_cap;
  const int n_layers = (int)P.n_layers;
  const float det_refl = P.det_reflectance;
  const float start_w = P.start_weight;
  const int nr = kRefGrid ? 1000 : (int)P.grid_nr;
  const int nz = kRefGrid ? 500 : (int)P.grid_nz;
  const float dr = P.grid_dr;
  const float dz = P.grid_dz;
  const int tid = threadIdx.x;
  const int row_len = n_layers + 2;

  curandStateXORWOW st;
  clear_gauss(st);
  Photon p;

  for (;;) {
    const uint64_t item = fetch_one(A.cursor);
    if (item >= D) break;
    const DetRecord rec = A.records[item];
    st.d = rec.d;
    st.v[0] = rec.v[0];
    st.v[1] = rec.v[1];
    st.v[2] = rec.v[2];
    st.v[3] = rec.v[3];
    st.v[4] = rec.v[4];
    const int sds = (int)rec.sds;  // 1-based
    const unsigned sds0 = (unsigned)(sds - 1);
    launch_photon<kSrcOblique>(p, &st, t, start_w);
    for (int l = 0; l < n_layers; ++l) {
      s_pl[l][tid] = 0.0f;
      s_ni[l][tid] = 0u;
    }
    bool first_scatter = true;
    unsigned index_old = 0, w_run = 0;
    int steps = 0;
    float w_det = 0.0f;

    for (unsigned long long it = 0;; ++it) {
      if (it >= A.budget) {
        atomicOr(A.status, kStatusBudget);
        break;
      }
      float s;
      const int new_layer = hop(p, s, &st, t);
      steps++;
      s_pl[p.layer - 1][tid] += s;
      clamp_z(p, t, p.layer);

      if (new_layer != p.layer) {
        const int temp_layer = p.layer;
        s = 0.0f;
        if (!reflect(p, new_layer, &st, t)) {
          if (new_layer == 0) {
            bool hit;
            float wd = 0.0f;
            if (kDetOblique) {
              hit = fiber_hit(p, t, sds);
              wd = p.w;
            } else {
              const float uz_angle = acosf(fabsf(p.dz));
              const float distance = radius_xy(p);
              hit = ring_hit(p, t, sds, uz_angle, distance, wd);
            }
            if (hit) {
              w_det = wd;
              p.w = 0;
              break;
            }
            if (uni(&st) > det_refl) {
              p.w = 0;
              break;
            }
            p.dz *= -1;
            p.z *= -1;
            p.layer = temp_layer;
          }
          if (new_layer > n_layers) {
            p.w = 0;
            break;
          }
        }
      }

      if (s > 0.0f) {
        const float4 L = t.lay[p.layer];
        const unsigned w_temp = drop_weight(p, L.w);
        s_ni[p.layer - 1][tid] += 1u;
        // Absorbance tallies, transport.cu:580-600.
        int iz;
        if (kRefGrid)
          iz = min(__float2int_rz(__fdividef(p.z, 0.01f)), (int)(500 - 1));
        else
          iz = min(__float2int_rz(__fdividef(p.z, dz)), nz - 1);
        if (first_scatter) {
          atomicAdd(&A.A0_z[sds0 * nz + iz], (unsigned long long)w_temp);
          first_scatter = false;
        } else {
          int ir;
          if (kRefGrid)
            ir = min(__float2int_rz(__fdividef(radius_xy(p), 0.01f)), (int)1000 - 1);
          else
            ir = min(__float2int_rz(__fdividef(radius_xy(p), dr)), nr - 1);
          const unsigned index = sds0 * nr * nz + iz * nr + ir;
          if (index == index_old) {
            w_run += w_temp;
          } else {
            if (w_run != 0) atomicAdd(&A.A_rz[index_old], (unsigned long long)w_run);
            index_old = index;
            w_run = w_temp;
          }
        }
        spin(p, t.hg[p.layer], &st);
      }

      if (!survive<false>(p, &st)) break;
    }
    if (w_run != 0) atomicAdd(&A.A_rz[index_old], (unsigned long long)w_run);

    float *row = A.rows + item * row_len;
    row[0] = w_det;
    for (int l = 0; l < n_layers; ++l) row[1 + l] = s_pl[l][tid];
    row[n_layers + 1] = (float)steps;
    if (A.interactions) {
      uint32_t *ni = A.interactions + item * n_layers;
      for (int l = 0; l < n_layers; ++l) ni[l] = s_ni[l][tid];
    }
  }
}

// ---------------------------------------------------------------------------
// Per-SDS count, FP64 weight sum and sum of squares over the records.
__global__ void reduce_records_kernel(const DetRecord *rec, const unsigned long long *rec_count,
                                      unsigned long long rec_cap, unsigned n_sds,
                                      unsigned long long *det_count, double *wsum,
                                      double *wsq) {
  __shared__ unsigned long long c[kMaxSds + 1];
  __shared__ double s1[kMaxSds + 1];
  __shared__ double s2[kMaxSds + 1];
  for (int i = threadIdx.x; i <= kMaxSds; i += blockDim.x) {
    c[i] = 0;
    s1[i] = 0.0;
    s2[i] = 0.0;
  }
  __syncthreads();
  const unsigned long long total = *rec_count;
  const unsigned long long D = total < rec_cap ? total : rec_cap;
  for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < D;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    const unsigned s = rec[i].sds;
    const double w = (double)rec[i].weight;
    if (s >= 1 && s <= n_sds) {
      atomicAdd(&c[s], 1ull);
      atomicAdd(&s1[s], w);
      atomicAdd(&s2[s], w * w);
    }
  }
  __syncthreads();
  for (unsigned i = threadIdx.x + 1; i <= n_sds; i += blockDim.x) {
    if (c[i]) {
      atomicAdd(&det_count[i - 1], c[i]);
      atomicAdd(&wsum[i - 1], s1[i]);
      atomicAdd(&wsq[i - 1], s2[i]);
    }
  }
}

// Test support: the first `count` curand_uniform draws of a subsequence.
__global__ void uniform_stream_kernel(uint64_t seed, uint64_t subsequence, uint64_t count,
                                      float *out) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  curandStateXORWOW st;
  curand_init(seed, subsequence, 0, &st);
  for (uint64_t i = 0; i < count; ++i) out[i] = curand_uniform(&st);
}

// ---------------------------------------------------------------------------
// Host-side launchers.

cudaError_t launch_seed_slots(uint64_t seed, uint64_t slot_begin, uint64_t num_slots, uint2 *out,
                              int sm_count, cudaStream_t stream) {
  if (num_slots == 0) return cudaSuccess;
  const int block = 256;
  const uint64_t threads = (uint64_t)sm_count * 2048;  // one resident wave
  const uint64_t run = (num_slots + threads - 1) / threads;
  const uint64_t used = (num_slots + run - 1) / run;
  const int grid = (int)((used + block - 1) / block);
  seed_slots_kernel<<<grid, block, 0, stream>>>(seed, slot_begin, num_slots, run, out);
  return cudaGetLastError();
}

// Walk variants: (threads per block, minimum resident blocks per SM).  The
// second number caps the registers per thread (65536 / (threads * blocks)).
struct WalkVariant {
  int block, min_blocks;
  const void *fn[8];  // [glass*4 + src_oblique*2 + det_oblique]
};

template <int B, int M>
static WalkVariant make_variant() {
  return WalkVariant{B,
                     M,
                     {(const void *)walk_kernel<B, M, false, false, false>,
                      (const void *)walk_kernel<B, M, false, true, false>,
                      (const void *)walk_kernel<B, M, true, false, false>,
                      (const void *)walk_kernel<B, M, true, true, false>,
                      (const void *)walk_kernel<B, M, false, false, true>,
                      (const void *)walk_kernel<B, M, false, true, true>,
                      (const void *)walk_kernel<B, M, true, false, true>,
                      (const void *)walk_kernel<B, M, true, true, true>}};
}

static const WalkVariant *walk_variants(int *n) {
  static const WalkVariant v[] = {
      make_variant<64, 1>(),  make_variant<128, 1>(), make_variant<256, 1>(),
      make_variant<128, 8>(), make_variant<128, 10>(), make_variant<128, 12>(),
      make_variant<256, 4>(), make_variant<256, 5>(),  make_variant<256, 6>(),
  };
  *n = (int)(sizeof(v) / sizeof(v[0]));
  return v;
}

const void *walk_kernel_ptr(int block, int min_blocks, bool src_obl, bool det_obl, bool glass) {
  int n = 0;
  const WalkVariant *v = walk_variants(&n);
  for (int i = 0; i < n; ++i)
    if (v[i].block == block && v[i].min_blocks == min_blocks)
      return v[i].fn[(glass ? 4 : 0) + (src_obl ? 2 : 0) + (det_obl ? 1 : 0)];
  return nullptr;
}

bool has_glass_layer(const DevParams &P) {
  for (uint32_t l = 1; l <= P.n_layers; ++l)
    if (P.mutr[l] == FLT_MAX) return true;
  return false;
}

cudaError_t launch_walk(const DevParams &P, const WalkArgs &A, bool src_obl, bool det_obl,
                        int block, int min_blocks, int grid, cudaStream_t stream) {
  const void *fn = walk_kernel_ptr(block, min_blocks, src_obl, det_obl, has_glass_layer(P));
  if (!fn) return cudaErrorInvalidValue;
  void *args[] = {(void *)&P, (void *)&A};
  return cudaLaunchKernel(fn, dim3(grid), dim3(block), args, 0, stream);
}

template <bool kSrc, bool kDet>
static void replay_dispatch2(const DevParams &P, const ReplayArgs &A, bool ref_grid, int grid,
                             cudaStream_t stream) {
  if (ref_grid)
    replay_kernel<kReplayBlock, kSrc, kDet, true><<<grid, kReplayBlock, 0, stream>>>(P, A);
  else
    replay_kernel<kReplayBlock, kSrc, kDet, false><<<grid, kReplayBlock, 0, stream>>>(P, A);
}

cudaError_t launch_replay(const DevParams &P, const ReplayArgs &A, bool src_obl, bool det_obl,
                          bool ref_grid, int grid, cudaStream_t stream) {
  if (src_obl && det_obl)
    replay_dispatch2<true, true>(P, A, ref_grid, grid, stream);
  else if (src_obl)
    replay_dispatch2<true, false>(P, A, ref_grid, grid, stream);
  else if (det_obl)
    replay_dispatch2<false, true>(P, A, ref_grid, grid, stream);
  else
    replay_dispatch2<false, false>(P, A, ref_grid, grid, stream);
  return cudaGetLastError();
}

cudaError_t launch_reduce_records(const DetRecord *rec, const unsigned long long *rec_count,
                                  unsigned long long rec_cap, unsigned n_sds,
                                  unsigned long long *det_count, double *wsum, double *wsq,
                                  int sm_count, cudaStream_t stream) {
  reduce_records_kernel<<<sm_count, 256, 0, stream>>>(rec, rec_count, rec_cap, n_sds, det_count,
                                                      wsum, wsq);
  return cudaGetLastError();
}

cudaError_t launch_uniform_stream(uint64_t seed, uint64_t subsequence, uint64_t count, float *out,
                                  cudaStream_t stream) {
  uniform_stream_kernel<<<1, 32, 0, stream>>>(seed, subsequence, count, out);
  return cudaGetLastError();
}

}  // namespace mcml
