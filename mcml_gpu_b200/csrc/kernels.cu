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

struct SeedCopy {
  uint32_t d, v0, v1, v2, v3, v4;
  __device__ __forceinline__ void save(const curandStateXORWOW &st) {
    d = st.d;
    v0 = st.v[0];
    v1 = st.v[1];
    v2 = st.v[2];
    v3 = st.v[3];
    v4 = st.v[4];
  }
};

__device__ __forceinline__ void append_record(const WalkArgs &A, uint64_t photon, int sds,
                                              float w, const SeedCopy &sc) {
  const unsigned long long idx = atomicAdd(&A.counters[kCntRecords], 1ull);
  if (idx < A.rec_cap) {
    DetRecord r;
    r.photon = photon;
    r.sds = (uint32_t)sds;
    r.weight = w;
    r.d = sc.d;
    r.v[0] = sc.v0;
    r.v[1] = sc.v1;
    r.v[2] = sc.v2;
    r.v[3] = sc.v3;
    r.v[4] = sc.v4;
    A.records[idx] = r;
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// Slot seeding: state of subsequence s at offset 0 (LaunchPhoton_Global's
// curand_init, transport.cu:733), 24 bytes per slot.
__global__ void seed_slots_kernel(uint64_t seed, uint64_t slot_begin, uint64_t num_slots,
                                  uint2 *out) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t s = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; s < num_slots; s += stride) {
    curandStateXORWOW st;
    curand_init(seed, slot_begin + s, 0, &st);
    out[s * 3 + 0] = make_uint2(st.d, st.v[0]);
    out[s * 3 + 1] = make_uint2(st.v[1], st.v[2]);
    out[s * 3 + 2] = make_uint2(st.v[3], st.v[4]);
  }
}

// ---------------------------------------------------------------------------
// First pass (MCd, transport.cu:341-471).
template <int kBlock, bool kSrcOblique, bool kDetOblique>
__global__ void __launch_bounds__(kBlock) walk_kernel(const __grid_constant__ DevParams P,
                                                      const WalkArgs A) {
  __shared__ SmemTables t;
  load_tables(t, P);
  __syncthreads();

  const uint64_t S = P.num_slots;
  const uint64_t q = P.num_photons / S;
  const uint64_t rem = P.num_photons % S;
  const int n_layers = (int)P.n_layers;
  const int n_sds = (int)P.n_sds;
  const float det_refl = P.det_reflectance;
  const float start_w = P.start_weight;

  curandStateXORWOW st;
  clear_gauss(st);
  SeedCopy sc;
  Photon p;
  uint64_t photon = 0;
  uint64_t left = 0;
  uint32_t steps_acc = 0;

  auto next_slot = [&]() -> bool {
    const uint64_t slot = fetch_one(&A.counters[kCntSlot]);
    if (slot >= S) return false;
    load_state(st, A.slot_state, slot);
    photon = slot * q + (slot < rem ? slot : rem);
    left = q + (slot < rem ? 1 : 0) - 1;
    return true;
  };

  if (!next_slot()) return;
  sc.save(st);
  launch_photon<kSrcOblique>(p, &st, t, start_w);

  for (;;) {
    float s;
    const int new_layer = hop(p, s, &st, t);
    p.steps++;
    ++steps_acc;
    clamp_z(p, t, p.layer);

    if (new_layer != p.layer) {
      const int temp_layer = p.layer;
      s = 0.0f;
      if (!reflect(p, new_layer, &st, t)) {
        if (new_layer == 0) {
          bool detected = false;
          if (kDetOblique) {
            for (int i = 1; i <= n_sds; i++) {
              if (fiber_hit(p, t, i)) {
                append_record(A, photon, i, p.w, sc);
                detected = true;
              }
            }
          } else {
            const float uz_angle = acosf(fabsf(p.dz));
            const float distance = sqrtf(p.x * p.x + p.y * p.y);
            for (int i = 1; i <= n_sds; i++) {
              float wd;
              if (ring_hit(p, t, i, uz_angle, distance, wd)) {
                append_record(A, photon, i, wd, sc);
                detected = true;
              }
            }
          }
          if (detected) {
            p.w = 0;
          } else if (uni(&st) > det_refl) {
            p.w = 0;
          } else {
            p.dz *= -1;
            p.z *= -1;
            p.layer = temp_layer;
          }
        }
        if (new_layer > n_layers) p.w = 0;
      }
    }

    if (s > 0.0f) {
      const float4 L = t.lay[p.layer];
      drop_weight(p, L.w, L.z);
      spin(p, t.lay2[p.layer].x, &st);
    }

    if (!survive<true>(p, &st)) {
      if (left > 0) {
        --left;
        ++photon;
      } else {
        atomicAdd(&A.counters[kCntSteps], (unsigned long long)steps_acc);
        steps_acc = 0;
        if (!next_slot()) break;
      }
      if (steps_acc >= 0x40000000u) {
        atomicAdd(&A.counters[kCntSteps], (unsigned long long)steps_acc);
        steps_acc = 0;
      }
      sc.save(st);
      launch_photon<kSrcOblique>(p, &st, t, start_w);
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
              const float distance = sqrtf(p.x * p.x + p.y * p.y);
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
        const unsigned w_temp = drop_weight(p, L.w, L.z);
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
            ir = min(__float2int_rz(__fdividef(sqrtf(p.x * p.x + p.y * p.y), 0.01f)), (int)1000 - 1);
          else
            ir = min(__float2int_rz(__fdividef(sqrtf(p.x * p.x + p.y * p.y), dr)), nr - 1);
          const unsigned index = sds0 * nr * nz + iz * nr + ir;
          if (index == index_old) {
            w_run += w_temp;
          } else {
            if (w_run != 0) atomicAdd(&A.A_rz[index_old], (unsigned long long)w_run);
            index_old = index;
            w_run = w_temp;
          }
        }
        spin(p, t.lay2[p.layer].x, &st);
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
  uint64_t want = (num_slots + block - 1) / block;
  const uint64_t cap = (uint64_t)sm_count * 16;
  const int grid = (int)(want < cap ? want : cap);
  seed_slots_kernel<<<grid, block, 0, stream>>>(seed, slot_begin, num_slots, out);
  return cudaGetLastError();
}

template <int kBlock>
static cudaError_t walk_dispatch(const DevParams &P, const WalkArgs &A, bool src_obl,
                                 bool det_obl, int grid, cudaStream_t stream) {
  if (src_obl && det_obl)
    walk_kernel<kBlock, true, true><<<grid, kBlock, 0, stream>>>(P, A);
  else if (src_obl)
    walk_kernel<kBlock, true, false><<<grid, kBlock, 0, stream>>>(P, A);
  else if (det_obl)
    walk_kernel<kBlock, false, true><<<grid, kBlock, 0, stream>>>(P, A);
  else
    walk_kernel<kBlock, false, false><<<grid, kBlock, 0, stream>>>(P, A);
  return cudaGetLastError();
}

template <int kBlock>
static const void *walk_fn(bool src_obl, bool det_obl) {
  if (src_obl && det_obl) return (const void *)walk_kernel<kBlock, true, true>;
  if (src_obl) return (const void *)walk_kernel<kBlock, true, false>;
  if (det_obl) return (const void *)walk_kernel<kBlock, false, true>;
  return (const void *)walk_kernel<kBlock, false, false>;
}

const void *walk_kernel_ptr(int block, bool src_obl, bool det_obl) {
  switch (block) {
    case 64: return walk_fn<64>(src_obl, det_obl);
    case 128: return walk_fn<128>(src_obl, det_obl);
    case 256: return walk_fn<256>(src_obl, det_obl);
    default: return nullptr;
  }
}

cudaError_t launch_walk(const DevParams &P, const WalkArgs &A, bool src_obl, bool det_obl,
                        int block, int grid, cudaStream_t stream) {
  switch (block) {
    case 64: return walk_dispatch<64>(P, A, src_obl, det_obl, grid, stream);
    case 128: return walk_dispatch<128>(P, A, src_obl, det_obl, grid, stream);
    case 256: return walk_dispatch<256>(P, A, src_obl, det_obl, grid, stream);
    default: return cudaErrorInvalidValue;
  }
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
