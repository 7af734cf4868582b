// wmc.cu -- White Monte Carlo relabelling of replayed photons.
//
// A replayed photon's detected weight w, per-layer pathlengths PL_l and
// per-layer interaction counts n_l determine its weight under other
// optical coefficients without walking again.  In this walk the step length
// is drawn from mu_t = mu_a + mu_s and each interaction keeps the fraction
// mu_s/mu_t of the weight, so the path's contribution is proportional to
// prod_l mu_s_l^n_l exp(-mu_t_l PL_l); changing (mu_a, mu_s) to
// (mu_a', mu_s') multiplies it by
//
//     prod_l (mu_s'_l / mu_s_l)^n_l * exp(-sum_l (mu_t'_l - mu_t_l) PL_l).
//
// For mu_a alone this is exp(-sum dmu_a PL), the factor the reference uses
// for its average pathlength (transport.cu:285-292); the mu_s factor needs
// the interaction counts, which the reference does not record and this
// library's replay does.  Roulette and the integer weight quanta make the
// rescaled estimate unbiased in expectation, as White MC always is.
//
// Per (combo c, photon i) the kernel evaluates
//     R_c += exp2( sum_k a_ck F_ik ),   F_i = [PL_1..L, n_1..L, log2 w_i, 1]
// with a_c = [-(dmu_t)*log2(e) ..., log2(mu_s'/mu_s) ..., 1, 0]: a K=2L+2
// contraction, one exp2 (MUFU) and one add.  The exponents reach hundreds,
// so the contraction stays in FP32 on the CUDA cores (a bf16/tf32 tensor
// product would lose the exponent's low bits).  Photon features are staged
// through shared memory in chunks and each thread carries kPer combos over
// photon pairs on paired FP32 instructions; the photons are split over
// blockIdx.y and the partial sums added in FP64.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>

#include "../../include/mcml_b200.h"
#include "internal.h"

namespace mcml {
namespace {

constexpr int kThreads = 256;
constexpr int kPer = 2;      // combos per thread
constexpr int kChunk = 256;  // photons per shared-memory chunk (a multiple of 4)
constexpr int kMaxK = 2 * MCML_MAX_LAYERS + 2;

// Packs F_i (k-major within a photon, padded to kMaxK) for every photon.
__global__ void wmc_pack_kernel(const float *pl, const float *inter, const float *w,
                                uint64_t D, int L, float *F) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= D) return;
  float *f = F + i * kMaxK;
  for (int l = 0; l < L; ++l) {
    f[l] = pl[(uint64_t)l * D + i];
    f[L + l] = inter[(uint64_t)l * D + i];
  }
  const float wi = w[i];
  f[2 * L] = wi > 0.0f ? log2f(wi) : -INFINITY;
  f[2 * L + 1] = 1.0f;
  for (int k = 2 * L + 2; k < kMaxK; ++k) f[k] = 0.0f;
}

// 2^x on the MUFU unit (PTX ex2.approx, relative error about 2^-22;
// results below 2^-126 flush to zero, terms far below the photon weights
// that matter).
__device__ __forceinline__ float ex2(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// Each thread carries kPer combos and walks the photons in pairs: a pair's
// features sit interleaved in shared memory, {F_jk, F_j+1,k}, so that one
// 16-byte load feeds two k and every contraction step is one paired FMA
// (__ffma2_rn) over the two photons against the combo's coefficient held
// twice in a register pair.  A photon's exponent starts at its log2 weight
// (feature K-2, coefficient 1) and takes the 2L = K-2 pathlength and
// interaction terms, so the unit coefficient and the zero padding column
// cost nothing.  Two pairs are taken per iteration, which gives each
// thread 2*kPer independent FMA chains.  Per term that is L paired FMAs,
// one MUFU exp2, half a paired add and 1.5 shared loads; the FP32 lanes
// (2L + 1 operations per term) are the binding unit.
template <int K>
__global__ void __launch_bounds__(kThreads, 4) wmc_kernel(const float *F, uint64_t D,
                                                       const float *coef, uint64_t C,
                                                       double inv_scale, double *out) {
  static_assert(K % 2 == 0, "K = 2L+2 is even");
  __shared__ __align__(16) float2 sF[2][kChunk / 2][K];  // [buffer][photon pair][k]
  const uint64_t c0 = ((uint64_t)blockIdx.x * kThreads + threadIdx.x) * kPer;
  float2 a[kPer][K];
#pragma unroll
  for (int r = 0; r < kPer; ++r)
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const float v = (c0 + r < C) ? coef[(c0 + r) * kMaxK + k] : 0.0f;
      a[r][k] = make_float2(v, v);
    }
  double total[kPer];
#pragma unroll
  for (int r = 0; r < kPer; ++r) total[r] = 0.0;

  // this block's share of the photons (blockIdx.y of gridDim.y, whole chunks)
  const uint64_t chunks = (D + kChunk - 1) / kChunk;
  const uint64_t per = (chunks + gridDim.y - 1) / gridDim.y;
  const uint64_t d0 = blockIdx.y * per * kChunk;
  const uint64_t d1 = d0 + per * kChunk < D ? d0 + per * kChunk : D;
  // Chunk staging, double-buffered: the next chunk's features travel
  // (4-byte cp.async each) while this one is contracted.  Photons past the
  // end (padding to whole pairs of pairs) get weight 0: log2 w = -inf
  // (k = K-2) and 0 elsewhere, so their exp2 term is 0.
  auto stage = [&](uint64_t base, int buf) {
    const int n = (int)((d1 - base) < (uint64_t)kChunk ? (d1 - base) : (uint64_t)kChunk);
    const int np = (n + 3) / 4 * 2;
    for (int idx = threadIdx.x; idx < np * K; idx += kThreads) {
      const int jp = idx / K, k = idx % K;
      const int j = 2 * jp;
      float *dst = reinterpret_cast<float *>(&sF[buf][jp][k]);
      const float pad = k == K - 2 ? -INFINITY : 0.0f;
      if (j < n)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(
                         (unsigned)__cvta_generic_to_shared(dst)),
                     "l"(F + (base + j) * kMaxK + k)
                     : "memory");
      else
        dst[0] = pad;
      if (j + 1 < n)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(
                         (unsigned)__cvta_generic_to_shared(dst + 1)),
                     "l"(F + (base + j + 1) * kMaxK + k)
                     : "memory");
      else
        dst[1] = pad;
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  };
  int cur = 0;
  if (d0 < d1) stage(d0, 0);
  for (uint64_t base = d0; base < d1; base += kChunk) {
    const int n = (int)((d1 - base) < (uint64_t)kChunk ? (d1 - base) : (uint64_t)kChunk);
    const int np = (n + 3) / 4 * 2;  // photon pairs, an even number
    const bool more = base + kChunk < d1;
    if (more) stage(base + kChunk, cur ^ 1);
    if (more)
      asm volatile("cp.async.wait_group 1;\n" ::: "memory");
    else
      asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();
    float2 acc[kPer];
#pragma unroll
    for (int r = 0; r < kPer; ++r) acc[r] = make_float2(0.0f, 0.0f);
    for (int jp = 0; jp < np; jp += 2) {  // pairs jp and jp+1, added in order
      float2 e[2][kPer];
#pragma unroll
      for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int r = 0; r < kPer; ++r)
          e[h][r] = *reinterpret_cast<const float2 *>(&sF[cur][jp + h][K - 2]);  // log2 w
#pragma unroll
      for (int k = 0; k < K - 2; k += 2) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const float4 f = *reinterpret_cast<const float4 *>(&sF[cur][jp + h][k]);
#pragma unroll
          for (int r = 0; r < kPer; ++r)
            e[h][r] = __ffma2_rn(a[r][k], make_float2(f.x, f.y), e[h][r]);
#pragma unroll
          for (int r = 0; r < kPer; ++r)
            e[h][r] = __ffma2_rn(a[r][k + 1], make_float2(f.z, f.w), e[h][r]);
        }
      }
#pragma unroll
      for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int r = 0; r < kPer; ++r)
          acc[r] = __fadd2_rn(acc[r], make_float2(ex2(e[h][r].x), ex2(e[h][r].y)));
    }
#pragma unroll
    for (int r = 0; r < kPer; ++r) total[r] += (double)acc[r].x + (double)acc[r].y;
    __syncthreads();  // all warps are done with this buffer before it is refilled
    cur ^= 1;
  }
#pragma unroll
  for (int r = 0; r < kPer; ++r)
    if (c0 + r < C && d0 < d1) atomicAdd(&out[c0 + r], total[r] * inv_scale);
}

// Per-combo coefficient rows a_c (padded to kMaxK).
__global__ void wmc_coef_kernel(const float *combos, uint64_t C, int L, const float *base,
                                float *coef) {
  const uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= C) return;
  const float *x = combos + c * 2 * L;  // mua'_1..L, mus'_1..L
  float *a = coef + c * kMaxK;
  const float log2e = 1.4426950408889634f;
  for (int l = 0; l < L; ++l) {
    const float dmut = (x[l] - base[l]) + (x[L + l] - base[L + l]);
    a[l] = -dmut * log2e;
    a[L + l] = log2f(x[L + l] / base[L + l]);
  }
  a[2 * L] = 1.0f;
  a[2 * L + 1] = 0.0f;
  for (int k = 2 * L + 2; k < kMaxK; ++k) a[k] = 0.0f;
}

template <int K>
cudaError_t launch_wmc(const float *F, uint64_t D, const float *coef, uint64_t C,
                       double inv_scale, double *out, cudaStream_t s) {
  // combos across blockIdx.x, photons split across blockIdx.y so that a
  // few hundred combos still fill every SM; partial sums meet in FP64 atomics
  const uint64_t per_block = (uint64_t)kThreads * kPer;
  const unsigned gx = (unsigned)((C + per_block - 1) / per_block);
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // one wave: as many blocks as are resident at once (every block gets the
  // same number of photon chunks, so a second wave would only add a tail)
  int resident = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, wmc_kernel<K>, kThreads, 0) !=
          cudaSuccess ||
      resident < 1)
    resident = 4;
  const uint64_t chunks = (D + kChunk - 1) / kChunk;
  const uint64_t want = ((uint64_t)resident * sms + gx - 1) / gx;
  const unsigned gy = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(std::min<uint64_t>(chunks, want), 65535));
  cudaError_t e = cudaMemsetAsync(out, 0, C * sizeof(double), s);
  if (e != cudaSuccess) return e;
  wmc_kernel<K><<<dim3(gx, gy), kThreads, 0, s>>>(F, D, coef, C, inv_scale, out);
  return cudaGetLastError();
}

}  // namespace
}  // namespace mcml

using namespace mcml;

extern "C" int mcml_wmc_rescale(const mcml_wmc_set *set, const float *base_mua,
                                const float *base_mus, const float *combos, uint64_t num_combos,
                                double scale, double *out, void *workspace,
                                uint64_t workspace_bytes, void *stream) {
  clear_error();
  if (!set || !base_mua || !base_mus || !combos || !out)
    return set_error(MCML_E_INVALID, "mcml_wmc_rescale: null argument");
  const int L = (int)set->num_layers;
  if (L < 1 || L > MCML_MAX_LAYERS) return set_error(MCML_E_INVALID, "num_layers must be in [1,10]");
  const uint64_t D = set->count;
  const uint64_t need = mcml_wmc_workspace_bytes(D, num_combos);
  if (!workspace || workspace_bytes < need)
    return set_error(MCML_E_INVALID, "mcml_wmc_rescale: workspace of " + std::to_string(need) +
                                         " bytes needed");
  if (num_combos == 0) return MCML_OK;
  if (!(scale > 0)) return set_error(MCML_E_INVALID, "scale must be > 0");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // workspace: base[2L] | coef[C x kMaxK] | F[D x kMaxK]
  float *base = static_cast<float *>(workspace);
  float *coef = base + 2 * MCML_MAX_LAYERS + 4;
  float *F = coef + num_combos * kMaxK;
  float hbase[2 * MCML_MAX_LAYERS];
  for (int l = 0; l < L; ++l) {
    hbase[l] = base_mua[l];
    hbase[L + l] = base_mus[l];
  }
  cudaError_t e = cudaMemcpyAsync(base, hbase, 2 * L * sizeof(float), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) {
    wmc_coef_kernel<<<(unsigned)((num_combos + 255) / 256), 256, 0, s>>>(combos, num_combos, L,
                                                                         base, coef);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess && D > 0) {
    wmc_pack_kernel<<<(unsigned)((D + 255) / 256), 256, 0, s>>>(set->pathlength, set->interactions,
                                                                set->weight, D, L, F);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    const double inv = 1.0 / scale;
    if (D == 0) {
      e = cudaMemsetAsync(out, 0, num_combos * sizeof(double), s);
    } else {
      switch (2 * L + 2) {
        case 4: e = launch_wmc<4>(F, D, coef, num_combos, inv, out, s); break;
        case 6: e = launch_wmc<6>(F, D, coef, num_combos, inv, out, s); break;
        case 8: e = launch_wmc<8>(F, D, coef, num_combos, inv, out, s); break;
        case 10: e = launch_wmc<10>(F, D, coef, num_combos, inv, out, s); break;
        case 12: e = launch_wmc<12>(F, D, coef, num_combos, inv, out, s); break;
        case 14: e = launch_wmc<14>(F, D, coef, num_combos, inv, out, s); break;
        case 16: e = launch_wmc<16>(F, D, coef, num_combos, inv, out, s); break;
        case 18: e = launch_wmc<18>(F, D, coef, num_combos, inv, out, s); break;
        case 20: e = launch_wmc<20>(F, D, coef, num_combos, inv, out, s); break;
        default: e = launch_wmc<22>(F, D, coef, num_combos, inv, out, s); break;
      }
    }
  }
  if (e != cudaSuccess)
    return set_error(MCML_E_CUDA, std::string("mcml_wmc_rescale: ") + cudaGetErrorString(e));
  return MCML_OK;
}

extern "C" uint64_t mcml_wmc_workspace_bytes(uint64_t num_photons, uint64_t num_combos) {
  return (uint64_t)(2 * MCML_MAX_LAYERS + 4) * sizeof(float) +
         (num_combos + num_photons) * (uint64_t)(2 * MCML_MAX_LAYERS + 2) * sizeof(float);
}
