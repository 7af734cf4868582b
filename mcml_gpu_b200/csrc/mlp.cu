// mlp.cu -- BF16 MLP ensemble: training and inference kernels.
//
// The surrogate maps a tissue's layer parameters to per-SDS
// log-reflectance.  Network: in -> hidden x depth (GELU) -> out, an
// ensemble of E members trained side by side (gridDim.z = member).
// Weights are kept in FP32 (master copy, Adam state) and mirrored to BF16
// for the tensor-core GEMMs, which accumulate in FP32.
//
// Forward: tc_layer_kernel, one 128-row tile per CTA on the tcgen05
// tensor cores (operands in shared memory, FP32 accumulator in tensor
// memory, bias + GELU epilogue from tcgen05.ld).
//
// Backward: the hidden layers' dH = (dZ W^T) * gelu'(Z) on tc_layer_kernel
// (weights as a K-major B operand) and the weight gradients dW = X^T dZ
// (X as an MN-major A operand, 256-row batch slices added atomically); the
// output layer's 3-wide dH on the CUDA cores (narrow_back_kernel); dW of
// batches that are not whole 256-row slices on the GEMM below.
//
// Backward GEMM: C[M x N] = op(A)[M x K] * op(B)[K x N], BF16 operands staged in
// shared memory, mma.sync m16n8k16 fragments loaded with ldmatrix, FP32
// accumulators, and a fused epilogue:
//   kGeluBack : dZ = bf16(acc * gelu'(Zprev))   (back through an activation)
//   kStoreF32 : G = acc (FP32; weight gradients)
// op(A) = A or A^T, op(B) = B or B^T by template flags.
#include <cuda.h>  // CUtensorMap (the encoder is reached through the runtime)
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <random>
#include <string>
#include <vector>

#include "../../include/mcml_b200.h"
#include "internal.h"

namespace mcml {
namespace {

typedef __nv_bfloat16 bf16;

constexpr int BM = 64, BN = 64, BK = 32;  // CTA tile
constexpr int kGemmThreads = 128;         // 4 warps, 2 x 2, warp tile 32 x 32
constexpr int PAD = 8;                    // smem row padding (bf16 elements)

enum Epi { kGeluBack = 2, kStoreF32 = 3 };

// GELU in its tanh form, 0.5 z (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3))),
// with the hardware tanh (tanh.approx.f32, relative error ~2^-11, below
// the bf16 rounding of the activations): a handful of instructions instead
// of an erf evaluation, in the epilogue that bounds the forward kernel.
__device__ __forceinline__ float tanh_hw(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float gelu(float z) {
  const float t = tanh_hw(0.7978845608f * fmaf(0.044715f * z, z * z, z));
  return fmaf(0.5f * z, t, 0.5f * z);
}
// gelu() on two values with paired FP32 instructions (sm_100 FMUL2/FFMA2):
// each component rounded exactly as gelu() rounds it, half the issue slots.
__device__ __forceinline__ float2 gelu2(float2 z) {
  const float2 a = __fmul2_rn(make_float2(0.044715f, 0.044715f), z);
  const float2 zz = __fmul2_rn(z, z);
  const float2 u = __fmul2_rn(make_float2(0.7978845608f, 0.7978845608f), __ffma2_rn(a, zz, z));
  const float2 t = make_float2(tanh_hw(u.x), tanh_hw(u.y));
  const float2 h = __fmul2_rn(make_float2(0.5f, 0.5f), z);
  return __ffma2_rn(h, t, h);
}
__device__ __forceinline__ float gelu_grad(float z) {
  const float z2 = z * z;
  const float t = tanh_hw(0.7978845608f * fmaf(0.044715f * z, z2, z));
  return 0.5f * (1.0f + t) + 0.5f * z * (1.0f - t * t) * 0.7978845608f * fmaf(0.134145f, z2, 1.0f);
}

__device__ __forceinline__ unsigned smem_u32(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

struct GemmArgs {
  int M, N, K;
  const bf16 *A;
  long long lda, strideA;  // per-member strides (elements)
  const bf16 *B;
  long long ldb, strideB;
  const float *bias;       // unused by the backward epilogues
  long long strideBias;
  float *outF;             // FP32 output (weight gradients G)
  long long ldo, strideO;
  bf16 *outH;              // BF16 output (dZ for kGeluBack)
  long long ldh, strideH;
  const float *aux;        // Zprev for kGeluBack
  long long ldx, strideX;
  int splits, kper;        // kStoreF32: K split over gridDim.z (partial sums added atomically)
};

template <bool TA, bool TB, int EPI>
__global__ void __launch_bounds__(kGemmThreads) gemm_kernel(const GemmArgs g) {
  __shared__ __align__(16) bf16 As[BM][BK + PAD];
  __shared__ __align__(16) bf16 Bs[BK][BN + PAD];
  const int splits = g.splits > 1 ? g.splits : 1;
  const int z = blockIdx.z / splits;  // ensemble member
  const int k_begin = splits > 1 ? (int)(blockIdx.z % splits) * g.kper : 0;
  const int k_end = splits > 1 ? min(g.K, k_begin + g.kper) : g.K;
  const bf16 *A = g.A + z * g.strideA;
  const bf16 *B = g.B + z * g.strideB;
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
  float acc[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int r = 0; r < 4; ++r) acc[i][j][r] = 0.0f;

  for (int k0 = k_begin; k0 < k_end; k0 += BK) {
    // A tile: As[m][k] = op(A)(m0+m, k0+k); consecutive threads read
    // consecutive global addresses in either orientation.
    for (int e = tid; e < BM * BK; e += kGemmThreads) {
      int m, k;
      if (TA) { m = e % BM; k = e / BM; } else { k = e % BK; m = e / BK; }
      const int gm = m0 + m, gk = k0 + k;
      bf16 v = __float2bfloat16(0.0f);
      if (gm < g.M && gk < k_end) v = TA ? A[(long long)gk * g.lda + gm] : A[(long long)gm * g.lda + gk];
      As[m][k] = v;
    }
    for (int e = tid; e < BK * BN; e += kGemmThreads) {
      int k, n;
      if (TB) { k = e % BK; n = e / BK; } else { n = e % BN; k = e / BN; }
      const int gk = k0 + k, gn = n0 + n;
      bf16 v = __float2bfloat16(0.0f);
      if (gk < k_end && gn < g.N) v = TB ? B[(long long)gn * g.ldb + gk] : B[(long long)gk * g.ldb + gn];
      Bs[k][n] = v;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < BK; kk += 16) {
      unsigned a[2][4], b[4][2];
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int row = wm + i * 16 + (lane & 15);
        const int col = kk + (lane >> 4) * 8;
        asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                     : "=r"(a[i][0]), "=r"(a[i][1]), "=r"(a[i][2]), "=r"(a[i][3])
                     : "r"(smem_u32(&As[row][col])));
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int krow = kk + (lane & 15);
        const int col = wn + j * 8;
        asm volatile("ldmatrix.sync.aligned.m8n8.x2.trans.shared.b16 {%0,%1}, [%2];\n"
                     : "=r"(b[j][0]), "=r"(b[j][1])
                     : "r"(smem_u32(&Bs[krow][col])));
      }
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
          asm volatile(
              "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
              "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
              : "+f"(acc[i][j][0]), "+f"(acc[i][j][1]), "+f"(acc[i][j][2]), "+f"(acc[i][j][3])
              : "r"(a[i][0]), "r"(a[i][1]), "r"(a[i][2]), "r"(a[i][3]), "r"(b[j][0]),
                "r"(b[j][1]));
    }
    __syncthreads();
  }

  // Epilogue: thread holds rows (lane>>2) and (lane>>2)+8, columns 2*(lane&3)+{0,1}.
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const int m = m0 + wm + i * 16 + (lane >> 2) + (r >= 2 ? 8 : 0);
        const int n = n0 + wn + j * 8 + 2 * (lane & 3) + (r & 1);
        if (m >= g.M || n >= g.N) continue;
        const float v = acc[i][j][r];
        if (EPI == kStoreF32) {
          float *o = &g.outF[z * g.strideO + (long long)m * g.ldo + n];
          if (splits > 1)
            atomicAdd(o, v);
          else
            *o = v;
        } else {  // kGeluBack
          const float zp = g.aux[z * g.strideX + (long long)m * g.ldx + n];
          g.outH[z * g.strideH + (long long)m * g.ldh + n] = __float2bfloat16(v * gelu_grad(zp));
        }
      }
}

template <bool TA, bool TB, int EPI>
cudaError_t gemm(const GemmArgs &g, int members, cudaStream_t s) {
  dim3 grid((g.N + BN - 1) / BN, (g.M + BM - 1) / BM, members * (g.splits > 1 ? g.splits : 1));
  gemm_kernel<TA, TB, EPI><<<grid, kGemmThreads, 0, s>>>(g);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Forward layer on the 5th-generation tensor cores (tcgen05):
//   C[M x N] = A[M x K] * W[K x N] (+ bias, epilogue), one 128-row tile per CTA.
// A (activations, row-major) is staged in shared memory K-major, W
// (row-major, fan_in x fan_out) MN-major, both in the no-swizzle
// core-matrix layout (8 rows x 16 bytes per core matrix):
//   A: element (r, k) at (k/8)*kLboA + (r/8)*128 + (r%8)*16 + (k%8)*2
//   W: element (k, n) at (k/8)*LboB  + (n/8)*128 + (k%8)*16 + (n%8)*2
// so the descriptors carry SBO = 128 bytes (next 8 rows / 8 columns) and
// LBO = the distance between K groups of 8.  One thread issues the K/16
// MMAs (M = 128, N <= 256, BF16 in, FP32 accumulator in tensor memory),
// commits them to an mbarrier, and all eight warps read the accumulator
// back with tcgen05.ld (warp w: TMEM lanes 32*(w%4).., column half w/4)
// for the bias + GELU epilogue.  Every wait is bounded; a timeout sets
// *status and the tile is skipped.
constexpr int TCM = 128;            // rows per tile (UMMA M)
constexpr int kLboA = (TCM / 8) * 128;
constexpr long long kTcSpin = 1ll << 22;
// Polls of the end-of-kernel drain waits: those wait only for copies and
// MMAs this CTA already issued, which finish in bounded time, so their
// limit is far above the per-stage one and independent of it.
constexpr long long kTcDrainSpin = 1ll << 26;

// K columns per A chunk: the largest of 64, 32, 16 that divides K (K is a
// multiple of 16), so that the chunks cover every column.
__host__ __device__ __forceinline__ int tc_chunk_k(int K) {
  return K % 64 == 0 ? 64 : K % 32 == 0 ? 32 : 16;
}

enum TcEpi {
  kTcBiasGelu = 0,  // H = bf16(gelu(acc + b)), Z = acc + b (optional)
  kTcBias = 1,      // Y = acc + b (FP32, the output layer)
  kTcGeluBack = 2,  // H = bf16(acc * gelu'(aux)) (back through an activation)
  kTcAddF32 = 3     // Z += acc (FP32 atomics: partial sums of a split K)
};

struct TcArgs {
  int M, N, K, n_valid;     // N: MMA width (multiple of 16); n_valid <= N real columns
  const bf16 *A;            // M x K, row-major, lda
  long long lda, strideA;
  const bf16 *W;            // K x n_valid row-major (B MN-major), or N x K row-major (B K-major)
  long long strideW;
  const float *aux;         // kTcGeluBack: the pre-activations Z of the layer below
  long long ldaux, strideAux;
  const float *bias;
  long long strideBias;
  float *Z;                 // kTcBiasGelu: pre-activations (may be null); kTcBias: output
  long long ldz, strideZ;
  bf16 *H;                  // kTcBiasGelu: activations
  long long ldh, strideH;
  unsigned *status;
  long long spin;           // polls per pipeline wait before it gives up (timeout)
  int slots;                // A ring slots (chunks of up to 64 K columns), 2..16
  int splits;               // K split over gridDim.z (member = z / splits, slice = z % splits)
  long long sliceA, sliceW; // element offsets of one K slice in A and W
  int use_tma;              // A chunks by TMA, 128-byte swizzled (K-major A, K % 64 == 0)
  int use_tma_h;            // H written by TMA from per-warp staging (64-byte swizzle)
};

__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version (Blackwell)
  return d;                // base offset 0, no swizzle
}

// K-major operand as TMA writes it with 128-byte swizzling: rows of 128 B
// (64 BF16), 8-row groups 1024 B apart (SBO), the two 16-byte K halves of
// an MMA adjacent (LBO field 1); K steps within the 128-byte atom advance
// the start address by 32 B.  The tile base must be 1024-byte aligned.
__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)1 << 16;             // LBO: 16 B
  d |= (uint64_t)(1024 >> 4) << 32;   // SBO: 1024 B
  d |= (uint64_t)1 << 46;             // descriptor version (Blackwell)
  d |= (uint64_t)2 << 61;             // 128-byte swizzle
  return d;
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t phase,
                                          long long limit = kTcSpin) {
  for (long long i = 0; i < limit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred P;\n mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n"
        " selp.u32 %0, 1, 0, P;\n}\n"
        : "=r"(done)
        : "r"(bar), "r"(phase)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void tmem_wait() {
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
}

// 32 consecutive accumulator columns of this warp's 32 tensor-memory lanes.
__device__ __forceinline__ void tmem_ld32(uint32_t (&v)[32], uint32_t taddr) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
      "%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
        "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
        "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]),
        "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]),
        "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
      : "r"(taddr));
}

// Bias (+ GELU) of 32 accumulator columns [c0, c0+32) of one row; all
// columns are real (N even multiple of 32 means no padding here).
template <int EPI>
__device__ __forceinline__ void epilogue32(const TcArgs &g, const uint32_t (&v)[32], int z, int row,
                                           int c0, const float *bias, unsigned char *stage,
                                           int lane) {
  if (EPI == kTcBiasGelu) {
    float *zrow = g.Z ? g.Z + z * g.strideZ + (long long)row * g.ldz + c0 : nullptr;
    uint4 *hrow = reinterpret_cast<uint4 *>(g.H + z * g.strideH + (long long)row * g.ldh + c0);
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      float2 f[4];
#pragma unroll
      for (int i = 0; i < 4; ++i)
        f[i] = __fadd2_rn(make_float2(__uint_as_float(v[b * 8 + 2 * i]),
                                      __uint_as_float(v[b * 8 + 2 * i + 1])),
                          *reinterpret_cast<const float2 *>(bias + c0 + b * 8 + 2 * i));
      if (zrow) {
        reinterpret_cast<float4 *>(zrow)[2 * b] = make_float4(f[0].x, f[0].y, f[1].x, f[1].y);
        reinterpret_cast<float4 *>(zrow)[2 * b + 1] = make_float4(f[2].x, f[2].y, f[3].x, f[3].y);
      }
      __align__(16) __nv_bfloat162 h[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const float2 g2 = gelu2(f[i]);
        h[i] = __floats2bfloat162_rn(g2.x, g2.y);
      }
      if (stage)  // this lane's row of the warp's 32 x 32 tile, 64-byte swizzled
        *reinterpret_cast<uint4 *>(stage + lane * 64 + ((b ^ ((lane >> 1) & 3)) * 16)) =
            *reinterpret_cast<const uint4 *>(h);
      else
        hrow[b] = *reinterpret_cast<const uint4 *>(h);
    }
  } else if (EPI == kTcGeluBack) {
    const float4 *zrow =
        reinterpret_cast<const float4 *>(g.aux + z * g.strideAux + (long long)row * g.ldaux + c0);
    uint4 *hrow = reinterpret_cast<uint4 *>(g.H + z * g.strideH + (long long)row * g.ldh + c0);
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const float4 z0 = zrow[2 * b], z1 = zrow[2 * b + 1];
      const float zp[8] = {z0.x, z0.y, z0.z, z0.w, z1.x, z1.y, z1.z, z1.w};
      __align__(16) __nv_bfloat162 h[4];
#pragma unroll
      for (int i = 0; i < 4; ++i)
        h[i] = __floats2bfloat162_rn(__uint_as_float(v[b * 8 + 2 * i]) * gelu_grad(zp[2 * i]),
                                     __uint_as_float(v[b * 8 + 2 * i + 1]) * gelu_grad(zp[2 * i + 1]));
      if (stage)
        *reinterpret_cast<uint4 *>(stage + lane * 64 + ((b ^ ((lane >> 1) & 3)) * 16)) =
            *reinterpret_cast<const uint4 *>(h);
      else
        hrow[b] = *reinterpret_cast<const uint4 *>(h);
    }
  } else if (EPI == kTcAddF32) {
    float *y = g.Z + z * g.strideZ + (long long)row * g.ldz;
    if (c0 + 32 <= g.n_valid && (reinterpret_cast<uintptr_t>(y + c0) & 15) == 0) {
      // whole columns, 16-byte aligned: vector reductions (sm_90+), a
      // quarter of the atomic operations
#pragma unroll
      for (int i = 0; i < 32; i += 4)
        atomicAdd(reinterpret_cast<float4 *>(y + c0 + i),
                  make_float4(__uint_as_float(v[i]), __uint_as_float(v[i + 1]),
                              __uint_as_float(v[i + 2]), __uint_as_float(v[i + 3])));
    } else {
#pragma unroll
      for (int i = 0; i < 32; ++i)
        if (c0 + i < g.n_valid) atomicAdd(&y[c0 + i], __uint_as_float(v[i]));
    }
  } else {
    float *y = g.Z + z * g.strideZ + (long long)row * g.ldz;
#pragma unroll
    for (int i = 0; i < 32; ++i)
      if (c0 + i < g.n_valid) y[c0 + i] = __uint_as_float(v[i]) + bias[c0 + i];
  }
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                   bar)
               : "memory");
}

// Roles (12 warps): warps 0-2 stream A in K chunks of up to 64 into a ring
// of shared-memory slots (cp.async, completion arriving on a_full[slot]);
// warp 3, lane 0,
// issues the MMAs of a tile chunk by chunk into one of two tensor-memory
// accumulators, releasing each chunk (a_empty) and then the accumulator
// (acc_full) with tcgen05.commit; warps 4-11 drain an accumulator (bias,
// GELU, stores) while the next tile's MMAs run, and hand it back
// (acc_empty).  Every wait is bounded: a timeout sets *status and ends the
// waiting role; the others then run out of their own waits.  Whatever ends
// the roles, the CTA drains its asynchronous work before it frees tensor
// memory and exits: the TMA producer waits until every A load it issued has
// landed (a load's a_full phase completes when its bytes arrive), the MMA
// issuer commits all MMAs it issued to the drain barrier and waits for it,
// cp.async copies are waited for and the epilogue's TMA stores are read out.
constexpr int kTcWarps = 12;
constexpr int kProducers = 96;  // warps 0-2

template <int EPI, bool kBK, bool kAMN>
__global__ void __launch_bounds__(kTcWarps * 32, 1)
    tc_layer_kernel(const TcArgs g, const __grid_constant__ CUtensorMap tmA,
                    const __grid_constant__ CUtensorMap tmH) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  // 1024-byte aligned base (the swizzled A tiles need it)
  unsigned char *smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int splits = g.splits > 1 ? g.splits : 1;
  const int z = blockIdx.z / splits;      // ensemble member
  const int slice = blockIdx.z % splits;  // K slice
  const int K = g.K, N = g.N;
  const int tiles = (g.M + TCM - 1) / TCM;
  const int KC = tc_chunk_k(K);   // K per chunk
  const int nch = K / KC;          // chunks per tile
  const int nslots = g.slots;      // A ring: chunk i of the CTA's sequence uses slot i % nslots
  const uint32_t slot_bytes = (uint32_t)(KC / 8) * kLboA;
  const uint32_t lboB = (uint32_t)(N / 8) * 128;
  const bool tma = g.use_tma != 0;
  unsigned char *sB = smem;
  unsigned char *sA = smem + (((size_t)K * N * 2 + 1023) & ~(size_t)1023);
  // per epilogue warp two 2 KB staging tiles for the TMA stores of H
  unsigned char *sStage = sA + (size_t)nslots * slot_bytes;
  const size_t stage_bytes = g.use_tma_h ? (size_t)8 * 2 * 2048 : 0;
  float *sBias = reinterpret_cast<float *>(sStage + stage_bytes);
  uint64_t *bars = reinterpret_cast<uint64_t *>(sBias + 256);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(bars + 37);
  const uint32_t sA_u = smem_u32(sA), sB_u = smem_u32(sB), bars_u = smem_u32(bars);
  auto a_full = [&](int s) { return bars_u + 8u * s; };
  auto a_empty = [&](int s) { return bars_u + 8u * (16 + s); };
  auto acc_full = [&](int b) { return bars_u + 8u * (32 + b); };
  auto acc_empty = [&](int b) { return bars_u + 8u * (34 + b); };
  const uint32_t drain_bar = bars_u + 8u * 36;  // completion of every MMA issued
  const uint32_t need = 2u * (uint32_t)N;
  const uint32_t ncols = need <= 32 ? 32 : need <= 64 ? 64 : need <= 128 ? 128 : need <= 256 ? 256 : 512;

  if (tid == 0) {
    for (int c = 0; c < nslots; ++c) {
      mbar_init(a_full(c), tma ? 1 : kProducers);
      mbar_init(a_empty(c), 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(acc_full(b), 1);
      mbar_init(acc_empty(b), 256);
    }
    mbar_init(drain_bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     smem_u32(tslot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  // The layer's weights and bias, once per CTA, by all warps.
  const bf16 *W = g.W + z * g.strideW + slice * g.sliceW;
  if (kBK) {
    // B K-major from W (N x K, row-major): element (n, k) at
    // (k/8)*lboB + (n/8)*128 + (n%8)*16 + (k%8)*2, n % 8 fastest per 8 lanes
    const int kc8 = K / 8;
    for (int c = tid; c < N * kc8; c += kTcWarps * 32) {
      const int n_lo = c & 7, rest = c >> 3;
      const int kc = rest % kc8, n = (rest / kc8) * 8 + n_lo;
      const uint32_t dst = sB_u + kc * lboB + (n >> 3) * 128 + n_lo * 16;
      const bf16 *src = W + (long long)n * K + kc * 8;
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src) : "memory");
    }
  } else if (g.n_valid == N) {
    const int nc8 = N / 8;
    for (int c = tid; c < K * nc8; c += kTcWarps * 32) {
      const int k_lo = c & 7, rest = c >> 3;
      const int nc = rest % nc8, k = (rest / nc8) * 8 + k_lo;
      const uint32_t dst = sB_u + (k >> 3) * lboB + nc * 128 + k_lo * 16;
      const bf16 *src = W + (long long)k * N + nc * 8;
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src) : "memory");
    }
  } else {
    bf16 *sb = reinterpret_cast<bf16 *>(sB);
    for (int e = tid; e < K * N; e += kTcWarps * 32) {
      const int k = e / N, n = e % N;
      const bf16 v = n < g.n_valid ? W[(long long)k * g.n_valid + n] : __float2bfloat16(0.0f);
      sb[((k >> 3) * lboB + (n >> 3) * 128 + (k & 7) * 16 + (n & 7) * 2) / 2] = v;
    }
  }
  const float *bias = g.bias ? g.bias + z * g.strideBias : nullptr;
  for (int n = tid; n < N; n += kTcWarps * 32)
    sBias[n] = (g.bias && n < g.n_valid) ? bias[n] : 0.0f;
  asm volatile("cp.async.wait_all;\n" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = *tslot;
  const bf16 *A = g.A + z * g.strideA + slice * g.sliceA;

  if (warp < 3 && tma) {
    // ---- producer (one thread): each A chunk is one TMA box of 64 K x 128
    // rows, 128-byte swizzled, counted on a_full by its byte total; rows
    // past M read as zeros.  Coordinates: (K offset, row, member).
    if (tid == 0) {
      int gi = 0;  // after the loop: the number of loads issued
      bool alive = true;
      for (int tile = blockIdx.x; tile < tiles && alive; tile += gridDim.x) {
        for (int c = 0; c < nch; ++c, ++gi) {
          const int slot = gi % nslots, use = gi / nslots;
          if (use > 0 && !mbar_wait(a_empty(slot), (uint32_t)((use - 1) & 1), g.spin)) {
            atomicOr(g.status, 1u);
            alive = false;
            break;
          }
          const uint32_t dst = sA_u + (uint32_t)slot * slot_bytes;
          asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(a_full(slot)),
                       "r"(slot_bytes)
                       : "memory");
          asm volatile(
              "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
              " [%0], [%1, {%3, %4, %5}], [%2];\n" ::"r"(dst),
              "l"(reinterpret_cast<uint64_t>(&tmA)), "r"(a_full(slot)), "r"(c * KC),
              "r"(tile * TCM), "r"(z)
              : "memory");
        }
      }
      // Drain: the last load issued into each slot has landed once that
      // use's a_full phase is complete (already so if the MMAs consumed it).
      for (int slot = 0; slot < nslots && slot < gi; ++slot) {
        const int last_use = (gi - 1 - slot) / nslots;
        if (!mbar_wait(a_full(slot), (uint32_t)(last_use & 1), kTcDrainSpin))
          atomicOr(g.status, 2u);
      }
    }
    __syncwarp();
  } else if (warp < 3) {
    // ---- producers: A chunks into the ring.  Each thread's copies of a
    // chunk arrive on a_full[slot] by themselves when they land
    // (cp.async.mbarrier.arrive.noinc; the barrier expects all 96 producer
    // threads), so the producers never wait for their own copies and run as
    // far ahead as the ring allows: a slot is refilled once the MMAs of the
    // chunk that used it last have completed (a_empty).
    const int per_chunk = TCM * KC / 8;  // 16-byte copies per chunk
    int gi = 0;                          // chunk sequence number
    for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
      const int m0 = tile * TCM;
      bool alive = true;
      for (int c = 0; c < nch; ++c, ++gi) {
        const int slot = gi % nslots, use = gi / nslots;
        if (use > 0 && !mbar_wait(a_empty(slot), (uint32_t)((use - 1) & 1), g.spin)) {
          atomicOr(g.status, 1u);
          alive = false;
          break;
        }
        const uint32_t base = sA_u + (uint32_t)slot * slot_bytes;
        if (kAMN) {
          // A MN-major from a K x M row-major array (A(m, k) at A[k*lda + m]):
          // element (m, k) at (k/8)*kLboA + (m/8)*128 + (k%8)*16 + (m%8)*2
          for (int e = tid; e < per_chunk; e += kProducers) {
            const int k_lo = e & 7, rest = e >> 3;
            const int mc = rest % (TCM / 8), kg = rest / (TCM / 8);
            const uint32_t dst = base + kg * kLboA + mc * 128 + k_lo * 16;
            const int gm = m0 + mc * 8;
            const int gk = c * KC + kg * 8 + k_lo;
            const bf16 *src = A + (long long)gk * g.lda + (gm < g.M ? gm : 0);
            const uint32_t bytes = gm < g.M ? 16u : 0u;
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src),
                         "r"(bytes)
                         : "memory");
          }
        } else {
          for (int e = tid; e < per_chunk; e += kProducers) {
            const int r_lo = e & 7, rest = e >> 3;
            const int kl = rest % (KC / 8), r = (rest / (KC / 8)) * 8 + r_lo;
            const uint32_t dst = base + kl * kLboA + (r >> 3) * 128 + r_lo * 16;
            const int gr = m0 + r;
            const bf16 *src = A + (long long)(gr < g.M ? gr : 0) * g.lda + (c * (KC / 8) + kl) * 8;
            const uint32_t bytes = gr < g.M ? 16u : 0u;
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src),
                         "r"(bytes)
                         : "memory");
          }
        }
        asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];\n" ::"r"(a_full(slot))
                     : "memory");
      }
      if (!alive) break;
    }
  } else if (warp == 3) {
    // ---- MMA issuer
    if (lane == 0) {
      const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) |
                             ((kAMN ? 1u : 0u) << 15) |  // A: MN-major or K-major
                             ((kBK ? 0u : 1u) << 16) |   // B: K-major or MN-major
                             ((uint32_t)(N >> 3) << 17) | ((uint32_t)(TCM >> 4) << 24);
      int t = 0;
      for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x, ++t) {
        const int b = t & 1, u = t >> 1;
        if (u > 0 && !mbar_wait(acc_empty(b), (uint32_t)((u - 1) & 1), g.spin)) {
          atomicOr(g.status, 1u);
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        const uint32_t d = tmem + (uint32_t)(b * N);
        bool ok = true;
        for (int c = 0; c < nch && ok; ++c) {
          const int gi = t * nch + c, slot = gi % nslots, use = gi / nslots;
          if (!mbar_wait(a_full(slot), (uint32_t)(use & 1), g.spin)) {
            atomicOr(g.status, 1u);
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
          const uint32_t base = sA_u + (uint32_t)slot * slot_bytes;
          for (int j = 0; j < KC / 16; ++j) {
            const int ks = c * (KC / 16) + j;  // K step of 16 within the tile
            const uint64_t ad = tma ? umma_desc_sw128(base + 32 * j)
                                    : umma_desc(base + 2 * j * kLboA, kLboA, 128);
            const uint64_t bd = umma_desc(sB_u + 2 * ks * lboB, lboB, 128);
            const uint32_t acc = ks > 0 ? 1u : 0u;
            asm volatile(
                "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d),
                "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
                : "memory");
          }
          umma_commit(a_empty(slot));
        }
        if (!ok) break;
        umma_commit(acc_full(b));
      }
      // Drain: the commit tracks every MMA this thread issued before it.
      umma_commit(drain_bar);
      if (!mbar_wait(drain_bar, 0u, kTcDrainSpin)) atomicOr(g.status, 2u);
    }
    __syncwarp();
  } else {
    // ---- epilogue: warp w drains TMEM lanes 32*(w%4).. , column half (w-4)/4
    const int q = warp & 3, half = (warp - 4) >> 2;
    const int c_begin = half * (N / 2);
    // staging tile of this warp's next TMA store: alternates over every
    // store of the kernel, so that the wait for all but the latest store
    // group to finish reading always covers the tile about to be rewritten
    // (also when a tile has a single 32-column chunk per warp)
    int sbuf = 0;
    int t = 0;
    for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x, ++t) {
      const int b = t & 1, u = t >> 1;
      // whole warps or none: tcgen05.ld is warp-collective
      if (!__all_sync(0xffffffffu, mbar_wait(acc_full(b), (uint32_t)(u & 1), g.spin))) {
        atomicOr(g.status, 1u);
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      const int row = tile * TCM + q * 32 + lane;
      const uint32_t tbase = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * N);
      if ((N / 2) % 32 == 0) {
        const int chunks = (N / 2) / 32;
        unsigned char *my_stage = g.use_tma_h ? sStage + (warp - 4) * 4096 : nullptr;
        const int row0 = tile * TCM + q * 32;
        // one 32-column chunk: bias/GELU in registers, then either direct
        // stores or this warp's staging tile handed to a TMA store
        auto emit = [&](const uint32_t (&v)[32], int c0) {
          unsigned char *st = my_stage ? my_stage + sbuf * 2048 : nullptr;
          sbuf ^= 1;
          if (st) {
            if (lane == 0) asm volatile("cp.async.bulk.wait_group.read 1;\n" ::: "memory");
            __syncwarp();
          }
          if (row < g.M) epilogue32<EPI>(g, v, z, row, c0, sBias, st, lane);
          if (st) {
            asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
            __syncwarp();
            if (lane == 0) {
              asm volatile(
                  "cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%2, %3, %4}], [%1];\n" ::"l"(
                      reinterpret_cast<uint64_t>(&tmH)),
                  "r"(smem_u32(st)), "r"(c0), "r"(row0), "r"(z)
                  : "memory");
              asm volatile("cp.async.bulk.commit_group;\n" ::: "memory");
            }
          }
        };
        uint32_t va[32], vb[32];
        tmem_ld32(va, tbase + c_begin);
        tmem_wait();
        for (int c = 0; c < chunks; c += 2) {
          if (c + 1 < chunks) tmem_ld32(vb, tbase + c_begin + (c + 1) * 32);
          emit(va, c_begin + c * 32);
          tmem_wait();
          if (c + 1 < chunks) {
            if (c + 2 < chunks) tmem_ld32(va, tbase + c_begin + (c + 2) * 32);
            emit(vb, c_begin + (c + 1) * 32);
            tmem_wait();
          }
        }
      } else {
        for (int c0 = c_begin; c0 < c_begin + N / 2; c0 += 8) {
          uint32_t v[8];
          asm volatile(
              "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n"
              : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]),
                "=r"(v[6]), "=r"(v[7])
              : "r"(tbase + (uint32_t)c0));
          tmem_wait();
          if (row >= g.M) continue;
          float f[8];
#pragma unroll
          for (int i = 0; i < 8; ++i) f[i] = __uint_as_float(v[i]) + sBias[c0 + i];
          if (EPI == kTcAddF32) {
            float *y = g.Z + z * g.strideZ + (long long)row * g.ldz;
#pragma unroll
            for (int i = 0; i < 8; ++i)
              if (c0 + i < g.n_valid) atomicAdd(&y[c0 + i], __uint_as_float(v[i]));
          } else if (EPI == kTcGeluBack) {
            const float *zp = g.aux + z * g.strideAux + (long long)row * g.ldaux + c0;
            __align__(16) bf16 h[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) h[i] = __float2bfloat16(__uint_as_float(v[i]) * gelu_grad(zp[i]));
            *reinterpret_cast<uint4 *>(g.H + z * g.strideH + (long long)row * g.ldh + c0) =
                *reinterpret_cast<const uint4 *>(h);
          } else if (EPI == kTcBiasGelu) {
            if (g.Z) {
              float4 *zp = reinterpret_cast<float4 *>(g.Z + z * g.strideZ + (long long)row * g.ldz + c0);
              zp[0] = make_float4(f[0], f[1], f[2], f[3]);
              zp[1] = make_float4(f[4], f[5], f[6], f[7]);
            }
            __align__(16) bf16 h[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) h[i] = __float2bfloat16(gelu(f[i]));
            *reinterpret_cast<uint4 *>(g.H + z * g.strideH + (long long)row * g.ldh + c0) =
                *reinterpret_cast<const uint4 *>(h);
          } else {
            float *y = g.Z + z * g.strideZ + (long long)row * g.ldz;
#pragma unroll
            for (int i = 0; i < 8; ++i)
              if (c0 + i < g.n_valid) y[c0 + i] = f[i];
          }
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
      mbar_arrive(acc_empty(b));
    }
  }
  asm volatile("cp.async.wait_all;\n" ::: "memory");
  if (g.use_tma_h && warp >= 4 && lane == 0)
    asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory");  // H stores done
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(ncols)
                 : "memory");
  }
}

// ---------------------------------------------------------------------------
// Whole-network forward for inference on the tensor cores: every layer of
// every member in one launch.  CTA (c, member z) takes batches of
// batch_rows rows (whole 128-row tiles) and runs each batch through all the
// layers before the next batch.  The hidden layers run on the tensor cores,
// one *pass* per (batch, layer); the output layer (at most kFusedMaxOut
// columns) is folded into the last hidden layer's epilogue, which rounds
// that layer's activations to BF16 as a store would and multiplies them by
// the output weights on the CUDA cores, so no pass loads them back.  The
// batch's activations pass between layers through the CTA's own
// batch_rows scratch rows, written in place: a layer's epilogue stores
// tile t only after that tile's MMAs -- and so its loads of tile t -- have
// completed, and the next layer loads tile t only after those stores have
// (h_done).  One buffer per CTA keeps the whole scratch (148 x 1024 rows x
// 512 bytes at width 256) inside L2; two buffers did not fit and measured
// 3.36 against 3.00 ms for 1e6 queries x 4 members (the folded output
// layer then took it to 2.62 ms).  Every A operand
// (layer 0: the normalised inputs, padded to 64 columns; later layers: the
// scratch) streams in by TMA in 64-column chunks, 128-byte swizzled.
//
// Roles (20 warps), all running through the same sequence of passes with
// no block-wide barrier between passes:
//  * warp 0, lane 0 -- A producer: chunk loads into a ring of shared-memory
//    slots (a_full / a_empty).  Before loading tile t of layer l > 0 it
//    waits h_done[t], which the epilogue completes once layer l-1's stores
//    of tile t have finished.
//  * warp 3, lane 0 -- MMA issuer: per pass it waits for the layer's
//    weights (w_full), issues the tiles' tcgen05.mma into two 256-column
//    tensor-memory accumulators (acc_full / acc_empty), and once the pass's
//    MMAs have completed (mma_done) brings the next pass's weights in with
//    bulk copies of their packed image -- while the epilogue still works on
//    the pass's last tile.
//  * warps 4-19 -- epilogue, four warps per TMEM lane quarter, each taking
//    every fourth 32-column chunk: bias + GELU into a 64-byte-swizzled
//    staging tile written out by TMA stores; in the last pass bias + GELU
//    + BF16 rounding times the output weights, the four warps' partial
//    sums of a row added in a fixed order through shared memory (sRed,
//    red_bar) into the FP32 rows of Y.  The epilogue threads copy each pass's
//    bias into one of three shared-memory buffers (bias_ready): the
//    double-buffered accumulators keep the slowest epilogue thread within
//    two tiles, so within two passes, of the fastest.
// The mbarriers are set up once; every phase is derived from counters that
// run across passes.  Every wait is bounded: a timeout sets *status and
// s_err, and every role stops at its next check; the CTA then drains its
// copies and MMAs before it frees tensor memory.
constexpr int kMaxFusedLayers = 12;
constexpr int kFusedMaxTiles = 16;  // batch_rows / 128
constexpr int kFusedEpiWarps = 16;  // warps 4..19
constexpr int kFusedMaxOut = 3;     // output columns folded into the last hidden epilogue
constexpr int kFusedWarps = 4 + kFusedEpiWarps;
constexpr int kFusedParts = kFusedEpiWarps / 4;  // epilogue warps per TMEM lane quarter

struct FusedArgs {
  int n;                // rows
  int layers;           // weight matrices (depth + 1)
  int batch_rows;       // rows per batch, a multiple of 128, at most 128 * kFusedMaxTiles
  int K[kMaxFusedLayers];         // contraction widths, multiples of 64
  int N[kMaxFusedLayers];         // MMA widths, multiples of 16, at most 256
  int n_valid[kMaxFusedLayers];   // real output columns
  long long img_off[kMaxFusedLayers];  // byte offset of a layer's B image in a member's image
  long long b_off[kMaxFusedLayers];    // bias offsets in a member's FP32 parameters
  const unsigned char *img;       // packed B images, member z at z * img_stride
  long long img_stride;
  const float *Wf;                // FP32 parameters (the biases); member z at z * strideW
  long long strideW;
  float *Y;                       // members x n x n_valid[last]
  const bf16 *W16;                // BF16 parameters (the output layer's weights); member z at z * strideW
  long long w_off_out, b_off_out; // the output layer's weights and bias
  int out_dim;                    // at most kFusedMaxOut
  int slots;                      // A ring slots
  unsigned *status;
  long long spin;
};

// Global -> shared bulk copy (no tensor map) completing on an mbarrier.
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes,
                                         uint32_t bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
          dst),
      "l"(src), "r"(bytes), "r"(bar)
      : "memory");
}

// Bias + GELU of 32 accumulator columns [c0, c0+32) of one row, rounded to
// BF16 like a stored activation, then folded into the output layer:
// acc[o] += h_c * Wout[c][o] in column order.
__device__ __forceinline__ void fused_gelu_fold32(const uint32_t (&v)[32], int c0,
                                                  const float *bias, const float4 *wo,
                                                  float (&acc)[kFusedMaxOut]) {
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    const float2 b = *reinterpret_cast<const float2 *>(bias + c0 + 2 * i);
    const float2 g2 = gelu2(
        __fadd2_rn(make_float2(__uint_as_float(v[2 * i]), __uint_as_float(v[2 * i + 1])), b));
    const __nv_bfloat162 h = __floats2bfloat162_rn(g2.x, g2.y);
    const float hx = __low2float(h), hy = __high2float(h);
    const float4 w0 = wo[c0 + 2 * i], w1 = wo[c0 + 2 * i + 1];
    acc[0] = fmaf(hx, w0.x, acc[0]);
    acc[1] = fmaf(hx, w0.y, acc[1]);
    acc[2] = fmaf(hx, w0.z, acc[2]);
    acc[0] = fmaf(hy, w1.x, acc[0]);
    acc[1] = fmaf(hy, w1.y, acc[1]);
    acc[2] = fmaf(hy, w1.z, acc[2]);
  }
}

__global__ void __launch_bounds__(kFusedWarps * 32, 1)
    tc_fused_forward_kernel(const FusedArgs f, const __grid_constant__ CUtensorMap tmX,
                            const __grid_constant__ CUtensorMap tmA,
                            const __grid_constant__ CUtensorMap tmH) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char *smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int z = blockIdx.z;
  const int nslots = f.slots;
  constexpr uint32_t kSlot = 64 / 8 * kLboA;  // one 64-column x 128-row chunk
  int maxB = 0;
  for (int l = 0; l < f.layers; ++l) maxB = max(maxB, f.K[l] * f.N[l] * 2);
  unsigned char *sB = smem;
  unsigned char *sA = smem + (((size_t)maxB + 1023) & ~(size_t)1023);
  unsigned char *sStage = sA + (size_t)nslots * kSlot;
  float *sBias = reinterpret_cast<float *>(sStage + (size_t)kFusedEpiWarps * 2048);  // [3][256]
  float4 *sWo = reinterpret_cast<float4 *>(sBias + 3 * 256);  // [256]: output weights, FP32
  float *sRed = reinterpret_cast<float *>(sWo + 256);  // [2][kFusedParts-1][128][3] partial outputs
  uint64_t *bars = reinterpret_cast<uint64_t *>(sRed + 2 * (kFusedParts - 1) * 128 * 3);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(bars + 60);
  const uint32_t sA_u = smem_u32(sA), sB_u = smem_u32(sB), bars_u = smem_u32(bars);
  auto a_full = [&](int s) { return bars_u + 8u * s; };
  auto a_empty = [&](int s) { return bars_u + 8u * (16 + s); };
  auto acc_full = [&](int b) { return bars_u + 8u * (32 + b); };
  auto acc_empty = [&](int b) { return bars_u + 8u * (34 + b); };
  const uint32_t w_full = bars_u + 8u * 36;
  const uint32_t mma_done = bars_u + 8u * 37;
  auto h_done = [&](int t) { return bars_u + 8u * (38 + t); };
  auto bias_ready = [&](int i) { return bars_u + 8u * (54 + i); };  // 3 of the 4 used
  auto red_bar = [&](int i) { return bars_u + 8u * (58 + i); };
  volatile int &s_err = *reinterpret_cast<volatile int *>(tslot + 1);

  if (tid == 0) {
    s_err = 0;
    for (int c = 0; c < nslots; ++c) {
      mbar_init(a_full(c), 1);
      mbar_init(a_empty(c), 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(acc_full(b), 1);
      mbar_init(acc_empty(b), kFusedEpiWarps * 32);
    }
    mbar_init(w_full, 1);
    mbar_init(mma_done, 1);
    for (int t = 0; t < kFusedMaxTiles; ++t) mbar_init(h_done(t), kFusedEpiWarps);
    for (int i = 0; i < 3; ++i) mbar_init(bias_ready(i), kFusedEpiWarps * 32);
    for (int i = 0; i < 2; ++i) mbar_init(red_bar(i), kFusedEpiWarps * 32);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  {
    // the output layer's weights (BF16 values, held as FP32)
    const int H = f.K[f.layers - 1];
    const bf16 *wo = f.W16 + (long long)z * f.strideW + f.w_off_out;
    for (int k = tid; k < H; k += kFusedWarps * 32) {
      float w[4] = {0.0f, 0.0f, 0.0f, 0.0f};
      for (int o = 0; o < f.out_dim; ++o) w[o] = __bfloat162float(wo[(long long)k * f.out_dim + o]);
      sWo[k] = make_float4(w[0], w[1], w[2], w[3]);
    }
  }
  if (warp == 0) {  // two 256-column accumulators: all of tensor memory
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     smem_u32(tslot)),
                 "r"(512)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = *tslot;

  const int L = f.layers;
  const int BR = f.batch_rows;
  const int batches = (f.n + BR - 1) / BR;
  const int nb = (int)blockIdx.x < batches
                     ? (batches - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x
                     : 0;
  // the layers that run on the tensor cores; the output layer is folded
  // into the last one's epilogue
  const int LP = L - 1;
  const int passes = nb * LP;
  const int cta = z * gridDim.x + blockIdx.x;
  // the rows and tiles of pass wp's batch
  auto pass_rows = [&](int wp, int &r0, int &tiles) {
    const int bt = (int)blockIdx.x + (wp / LP) * (int)gridDim.x;
    r0 = bt * BR;
    const int rows = min(BR, f.n - r0);
    tiles = (rows + TCM - 1) / TCM;
  };

  if (warp == 0) {
    // ---- A producer
    if (lane == 0) {
      int gi = 0;  // chunk sequence number over all passes
      bool alive = true;
      for (int wp = 0; wp < passes && alive; ++wp) {
        const int j = wp / LP, l = wp % LP;
        int r0, tiles;
        pass_rows(wp, r0, tiles);
        const int nch = f.K[l] / 64;
        const int a_row0 = cta * BR;  // layer l-1's output, this CTA's scratch rows
        for (int t = 0; t < tiles && alive; ++t) {
          if (l > 0) {
            // layer l-1's stores of this tile are complete (completion
            // number j*(LP-1) + l-1 of h_done[t]: one per stored layer and batch)
            if (s_err || !mbar_wait(h_done(t), (uint32_t)((j * (LP - 1) + l - 1) & 1), f.spin)) {
              atomicOr(f.status, 1u);
              s_err = 1;
              alive = false;
              break;
            }
            asm volatile("fence.proxy.async.global;\n" ::: "memory");
          }
          for (int c = 0; c < nch; ++c, ++gi) {
            const int slot = gi % nslots, use = gi / nslots;
            if (use > 0 &&
                (s_err || !mbar_wait(a_empty(slot), (uint32_t)((use - 1) & 1), f.spin))) {
              atomicOr(f.status, 1u);
              s_err = 1;
              alive = false;
              break;
            }
            const uint32_t dst = sA_u + (uint32_t)slot * kSlot;
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(
                             a_full(slot)),
                         "r"(kSlot)
                         : "memory");
            const uint64_t map = l == 0 ? reinterpret_cast<uint64_t>(&tmX)
                                        : reinterpret_cast<uint64_t>(&tmA);
            const int row = l == 0 ? r0 + t * TCM : a_row0 + t * TCM;
            asm volatile(
                "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
                " [%0], [%1, {%3, %4, %5}], [%2];\n" ::"r"(dst),
                "l"(map), "r"(a_full(slot)), "r"(c * 64), "r"(row), "r"(0)
                : "memory");
          }
        }
      }
      // drain: every load issued has landed (its slot's a_full phase)
      for (int slot = 0; slot < nslots && slot < gi; ++slot) {
        const int last_use = (gi - 1 - slot) / nslots;
        if (!mbar_wait(a_full(slot), (uint32_t)(last_use & 1), kTcDrainSpin)) {
          atomicOr(f.status, 2u);
          s_err = 1;
        }
      }
    }
    __syncwarp();
  } else if (warp == 3) {
    // ---- MMA issuer (and the weight loads)
    if (lane == 0) {
      const unsigned char *img = f.img + (long long)z * f.img_stride;
      auto load_weights = [&](int wp) {
        const int l = wp % LP;
        const uint32_t bytes = (uint32_t)(f.K[l] * f.N[l] * 2);
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(w_full),
                     "r"(bytes)
                     : "memory");
        for (uint32_t off = 0; off < bytes; off += 32768u)
          bulk_g2s(sB_u + off, img + f.img_off[l] + off, min(32768u, bytes - off), w_full);
      };
      int gi = 0, tseq = 0;
      int w_pending = -1;  // pass whose weights were requested and not yet waited for
      if (passes > 0) {
        load_weights(0);
        w_pending = 0;
      }
      bool alive = true;
      for (int wp = 0; wp < passes && alive; ++wp) {
        const int l = wp % LP;
        int r0, tiles;
        pass_rows(wp, r0, tiles);
        (void)r0;
        if (s_err || !mbar_wait(w_full, (uint32_t)(wp & 1), f.spin)) {
          atomicOr(f.status, 1u);
          s_err = 1;
          break;
        }
        w_pending = -1;
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        const int N = f.N[l], nch = f.K[l] / 64;
        // B K-major (bit 16 clear): the packed image's 128-byte-swizzled rows
        const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) |
                               ((uint32_t)(N >> 3) << 17) | ((uint32_t)(TCM >> 4) << 24);
        for (int t = 0; t < tiles && alive; ++t, ++tseq) {
          const int b = tseq & 1, u = tseq >> 1;
          if (u > 0 && (s_err || !mbar_wait(acc_empty(b), (uint32_t)((u - 1) & 1), f.spin))) {
            atomicOr(f.status, 1u);
            s_err = 1;
            alive = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
          const uint32_t d = tmem + (uint32_t)(b * 256);
          for (int c = 0; c < nch; ++c, ++gi) {
            const int slot = gi % nslots, use = gi / nslots;
            if (s_err || !mbar_wait(a_full(slot), (uint32_t)(use & 1), f.spin)) {
              atomicOr(f.status, 1u);
              s_err = 1;
              alive = false;
              break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            const uint32_t base = sA_u + (uint32_t)slot * kSlot;
#pragma unroll
            for (int jj = 0; jj < 4; ++jj) {
              const int ks = c * 4 + jj;
              const uint64_t ad = umma_desc_sw128(base + 32 * jj);
              const uint64_t bd =
                  umma_desc_sw128(sB_u + (uint32_t)c * (uint32_t)(N * 128) + 32 * jj);
              const uint32_t acc = ks > 0 ? 1u : 0u;
              asm volatile(
                  "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                  " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d),
                  "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
                  : "memory");
            }
            umma_commit(a_empty(slot));
          }
          if (alive) umma_commit(acc_full(b));
        }
        // every MMA of this pass (issued so far) has read the weights
        umma_commit(mma_done);
        if (!mbar_wait(mma_done, (uint32_t)(wp & 1), kTcDrainSpin)) {
          atomicOr(f.status, 2u);
          s_err = 1;
          alive = false;
        }
        if (alive && wp + 1 < passes) {
          load_weights(wp + 1);
          w_pending = wp + 1;
        }
      }
      if (w_pending >= 0 && !mbar_wait(w_full, (uint32_t)(w_pending & 1), kTcDrainSpin)) {
        atomicOr(f.status, 2u);
        s_err = 1;
      }
    }
    __syncwarp();
  } else if (warp >= 4) {
    // ---- epilogue: warp w drains TMEM lanes 32*(w%4).. (the lanes it may
    // access) and the 32-column chunks part, part + kFusedParts, ... of them
    const int q = warp & 3, part = (warp - 4) >> 2;
    unsigned char *my_stage = sStage + (warp - 4) * 2048;  // one staging tile per warp
    int pend = -1;    // lane 0: tile whose stores are issued but not yet signalled
    auto signal_stored = [&]() {
      if (lane == 0 && pend >= 0) {
        asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory");
        asm volatile("fence.proxy.async.global;\n" ::: "memory");
        mbar_arrive(h_done(pend));
        pend = -1;
      }
    };
    int tseq = 0;
    int otile = 0;  // tiles of the last pass so far (sRed / red_bar buffer and phase)
    bool alive = true;
    for (int wp = 0; wp < passes && alive; ++wp) {
      const int l = wp % LP;
      const bool last = l == LP - 1;
      int r0, tiles;
      pass_rows(wp, r0, tiles);
      const int N = f.N[l], nv = f.n_valid[l];
      const int rows = min(BR, f.n - r0);
      const int h_row0 = cta * BR;
      // this pass's bias into buffer wp % 3, completed on bias_ready
      float *bias = sBias + (wp % 3) * 256;
      {
        const int e = tid - 128;  // 0..511
        if (e < 256) bias[e] = e < nv ? f.Wf[(long long)z * f.strideW + f.b_off[l] + e] : 0.0f;
        mbar_arrive(bias_ready(wp % 3));
        if (s_err || !mbar_wait(bias_ready(wp % 3), (uint32_t)((wp / 3) & 1), f.spin)) {
          atomicOr(f.status, 1u);
          s_err = 1;
          alive = false;
          break;
        }
      }
      for (int t = 0; t < tiles; ++t, ++tseq) {
        const int b = tseq & 1, u = tseq >> 1;
        signal_stored();
        if (!__all_sync(0xffffffffu, s_err == 0 &&
                                         mbar_wait(acc_full(b), (uint32_t)(u & 1), f.spin))) {
          atomicOr(f.status, 1u);
          s_err = 1;
          alive = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        const uint32_t tbase = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * 256);
        const int lrow = t * TCM + q * 32 + lane;  // row within the batch
        if (!last) {
          // bias + GELU -> BF16 staging -> TMA store into the scratch rows
          TcArgs g{};
          const int chunks = (N / 2) / 32;
          auto emit = [&](const uint32_t (&v)[32], int c0) {
            unsigned char *st = my_stage;
            // the previous store has finished reading the staging tile
            if (lane == 0) asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory");
            __syncwarp();
            epilogue32<kTcBiasGelu>(g, v, 0, 0, c0, bias, st, lane);
            asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
            __syncwarp();
            if (lane == 0) {
              asm volatile(
                  "cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%2, %3, %4}], [%1];\n" ::"l"(
                      reinterpret_cast<uint64_t>(&tmH)),
                  "r"(smem_u32(st)), "r"(c0), "r"(h_row0 + t * TCM + q * 32), "r"(0)
                  : "memory");
              asm volatile("cp.async.bulk.commit_group;\n" ::: "memory");
            }
          };
          (void)chunks;
          uint32_t va[32];
          for (int c = part; c < N / 32; c += kFusedParts) {
            tmem_ld32(va, tbase + c * 32);
            tmem_wait();
            emit(va, c * 32);
          }
          pend = t;
        } else {
          // last tensor-core layer: bias + GELU + BF16 rounding folded into
          // the output layer; the four warps of a lane quarter add their
          // partial sums in part order through sRed, and part 0 writes Y
          float acc[kFusedMaxOut] = {0.0f, 0.0f, 0.0f};
          uint32_t va[32];
          for (int c = part; c < N / 32; c += kFusedParts) {
            tmem_ld32(va, tbase + c * 32);
            tmem_wait();
            fused_gelu_fold32(va, c * 32, bias, sWo, acc);
          }
          const int ob = otile & 1;
          const int row = q * 32 + lane;
          if (part > 0) {
            float *r = sRed + (((ob * (kFusedParts - 1)) + part - 1) * 128 + row) * 3;
            r[0] = acc[0];
            r[1] = acc[1];
            r[2] = acc[2];
          }
          mbar_arrive(red_bar(ob));
          if (part == 0) {
            if (s_err || !mbar_wait(red_bar(ob), (uint32_t)((otile >> 1) & 1), f.spin)) {
              atomicOr(f.status, 1u);
              s_err = 1;
            } else if (lrow < rows) {
              float *y = f.Y + ((long long)z * f.n + r0 + lrow) * f.out_dim;
              const float *bo = f.Wf + (long long)z * f.strideW + f.b_off_out;
#pragma unroll
              for (int o = 0; o < kFusedMaxOut; ++o) {
                float sum = acc[o];
#pragma unroll
                for (int pp = 0; pp < kFusedParts - 1; ++pp)
                  sum += sRed[(((ob * (kFusedParts - 1)) + pp) * 128 + row) * 3 + o];
                if (o < f.out_dim) y[o] = sum + bo[o];
              }
            }
          }
          ++otile;
        }
        asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
        mbar_arrive(acc_empty(b));
      }
      signal_stored();  // the pass's last tile
    }
    if (lane == 0) asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory");
    __syncwarp();
  }
  // ---- teardown: every role has drained what it issued
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(512)
                 : "memory");
  }
}

// Packed B images of the fused forward: member z, layer l at
// z * img_stride + img_off[l], element (k, n) of the K x N operand (zero
// past the layer's fan_in rows and fan_out columns) stored K-major in
// 64-column chunks of N rows x 128 bytes with the 128-byte swizzle (the
// 16-byte unit k%64/8 of row n at unit (k%64/8) ^ (n%8)) -- the layout TMA
// gives the A operand, so one bulk copy puts the image in shared memory
// ready for the MMA.  (Measured against the MN-major no-swizzle layout of
// the layer kernel: 2.605 against 2.624 ms for 1e6 queries x 4 members.)
struct FusedPack {
  int layers;
  int K[kMaxFusedLayers], N[kMaxFusedLayers], fan_in[kMaxFusedLayers], n_valid[kMaxFusedLayers];
  long long elem_begin[kMaxFusedLayers + 1];  // element prefix over the layers (per member)
  long long img_off[kMaxFusedLayers];
  long long w_off[kMaxFusedLayers];
};

__global__ void fused_pack_kernel(const bf16 *W16, long long strideW, const FusedPack pk,
                                  unsigned char *img, long long img_stride) {
  const int z = blockIdx.z;
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= pk.elem_begin[pk.layers]) return;
  int l = 0;
  while (e >= pk.elem_begin[l + 1]) ++l;
  const long long i = e - pk.elem_begin[l];
  const int N = pk.N[l];
  const int k = (int)(i / N), n = (int)(i % N);
  const bf16 v = (k < pk.fan_in[l] && n < pk.n_valid[l])
                     ? W16[(long long)z * strideW + pk.w_off[l] + (long long)k * pk.n_valid[l] + n]
                     : __float2bfloat16(0.0f);
  const int kk = k & 63;
  const long long byte = pk.img_off[l] + (long long)(k >> 6) * N * 128 + (long long)n * 128 +
                         (((kk >> 3) ^ (n & 7)) << 4) + (kk & 7) * 2;
  *reinterpret_cast<bf16 *>(img + (long long)z * img_stride + byte) = v;
}

constexpr size_t kTcSmemMax = 227 * 1024;  // opt-in shared memory per block
constexpr size_t kTcSmemFixed = 256 * 4 + 37 * 8 + 16;  // bias, barriers, TMEM slot

size_t tc_slot_bytes(int K) { return (size_t)tc_chunk_k(K) / 8 * kLboA; }

// A ring slots: as many as fit beside the weights (at most 16).
size_t tc_align1k(size_t n) { return (n + 1023) & ~(size_t)1023; }

constexpr size_t kTcStageBytes = 8 * 2 * 2048;  // H staging for TMA stores

// A ring slots: as many as fit beside the weights and the staging (at most 16).
int tc_slots(int K, int N, bool stage) {
  const size_t room = kTcSmemMax - tc_align1k((size_t)K * N * 2) - kTcSmemFixed - 1024 -
                      (stage ? kTcStageBytes : 0);
  return (int)std::min<size_t>(16, room / tc_slot_bytes(K));
}

size_t tc_smem_bytes(int K, int N, int slots, bool stage) {
  // weights, A ring, bias + barriers, 1 KB of alignment slack; at least
  // 120 KB so that one CTA runs per SM and its tensor-memory allocation
  // never waits for another's
  const size_t need = tc_align1k((size_t)K * N * 2) + (size_t)slots * tc_slot_bytes(K) +
                      kTcSmemFixed + 1024 + (stage ? kTcStageBytes : 0);
  return std::max<size_t>(need, 120 * 1024);
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                  const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                  const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// cuTensorMapEncodeTiled through the runtime's driver entry point (no
// link-time dependency on the driver library); null if unavailable.
EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *ptr = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(ptr);
    else
      cudaGetLastError();
  });
  return fn;
}

// Tensor map of A as (K, rows, member) for 64 x 128 boxes with 128-byte
// swizzling.  False when A cannot be described (the caller then streams A
// with cp.async).
bool encode_a_map(const TcArgs &g, int members, CUtensorMap *map) {
  EncodeTiledFn fn = encode_tiled();
  if (!fn || g.K % 64 != 0) return false;
  const cuuint64_t dims[3] = {(cuuint64_t)g.K, (cuuint64_t)g.M, (cuuint64_t)members};
  const cuuint64_t strides[2] = {(cuuint64_t)g.lda * 2, (cuuint64_t)g.strideA * 2};
  const cuuint32_t box[3] = {64, TCM, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  if (strides[0] % 16 || (members > 1 && strides[1] % 16) || ((uintptr_t)g.A & 15)) return false;
  return fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<bf16 *>(g.A), dims, strides, box,
            estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Tensor map of H as (column, row, member) for 32 x 32 store boxes with
// 64-byte swizzling, matching the epilogue warps' staging tiles.
bool encode_h_map(const TcArgs &g, int members, CUtensorMap *map) {
  EncodeTiledFn fn = encode_tiled();
  if (!fn || !g.H) return false;
  const cuuint64_t dims[3] = {(cuuint64_t)g.N, (cuuint64_t)g.M, (cuuint64_t)members};
  const cuuint64_t strides[2] = {(cuuint64_t)g.ldh * 2, (cuuint64_t)g.strideH * 2};
  const cuuint32_t box[3] = {32, 32, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  if (strides[0] % 16 || (members > 1 && strides[1] % 16) || ((uintptr_t)g.H & 15)) return false;
  return fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, g.H, dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B,
            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int EPI, bool kBK = false, bool kAMN = false>
cudaError_t tc_layer(const TcArgs &g, int members, cudaStream_t s) {
  if (g.N % 16 || g.N < 16 || g.N > 256 || g.K % 16 || g.K < 16 || g.K > 256 || g.n_valid > g.N)
    return cudaErrorInvalidValue;
  TcArgs a = g;
  if (a.spin <= 0) a.spin = kTcSpin;
  CUtensorMap hmap;
  std::memset(&hmap, 0, sizeof(hmap));
  const bool stage = (EPI == kTcBiasGelu || EPI == kTcGeluBack) && (g.N / 2) % 32 == 0 &&
                     g.n_valid == g.N && encode_h_map(g, members, &hmap);
  a.use_tma_h = stage ? 1 : 0;
  a.slots = tc_slots(g.K, g.N, stage);
  if (a.slots < 2) return cudaErrorInvalidValue;
  const size_t smem = tc_smem_bytes(g.K, g.N, a.slots, stage);
  // per device (the attribute belongs to the context); setting it twice
  // from two threads is harmless, the flags only save the calls
  static std::atomic<bool> configured[64];
  static std::atomic<int> sm_count[64];
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  if (!configured[dev].load()) {
    e = cudaFuncSetAttribute(tc_layer_kernel<EPI, kBK, kAMN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kTcSmemMax);
    if (e != cudaSuccess) return e;
    configured[dev].store(true);
  }
  int sms = sm_count[dev].load();
  if (!sms) {
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    sm_count[dev].store(sms);
  }
  // persistent: one CTA per SM shared out among the members, each CTA
  // walking its member's 128-row tiles with the weights resident
  const int tiles = (g.M + TCM - 1) / TCM;
  const int zs = std::max(1, members) * std::max(1, g.splits);
  const int per_z = std::max(1, sms / zs);
  dim3 grid(std::min(tiles, per_z), 1, zs);
  CUtensorMap map;
  std::memset(&map, 0, sizeof(map));
  a.use_tma = (!kAMN && encode_a_map(a, members, &map)) ? 1 : 0;
  tc_layer_kernel<EPI, kBK, kAMN><<<grid, kTcWarps * 32, smem, s>>>(a, map, hmap);
  return cudaGetLastError();
}

// X rows of a minibatch -> BF16, normalised, zero-padded to in_pad columns.
// Training state read by the kernels of a step, so that one recorded step
// (a CUDA graph) serves every minibatch of an epoch: the rows of the
// epoch's shuffles consumed so far, the Adam steps taken, the learning rate.
struct TrainStep {
  unsigned long long offset;
  long long t;
  float lr;
};

// Marks a minibatch done: the next one starts `rows` further into the shuffles.
__global__ void advance_step_kernel(TrainStep *st, unsigned long long rows) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    st->offset += rows;
    st->t += 1;
  }
}

__global__ void gather_x_kernel(const float *X, const uint32_t *idx, int n, int in_dim, int in_pad,
                                const float *mean, const float *inv_std, long long idx_stride,
                                bf16 *out, long long out_stride, const TrainStep *st) {
  const int z = blockIdx.z;
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long long)n * in_pad) return;
  const int r = (int)(e / in_pad), c = (int)(e % in_pad);
  float v = 0.0f;
  if (c < in_dim) {
    if (idx && st) idx += st->offset;
    const uint32_t row = idx ? idx[z * idx_stride + r] : (uint32_t)r;
    v = (X[(long long)row * in_dim + c] - mean[c]) * inv_std[c];
  }
  out[z * out_stride + e] = __float2bfloat16(v);
}

// Loss (mean squared error of normalised targets) and dY = 2 (Y - T) / (n * out).
__global__ void loss_grad_kernel(const float *Yp, long long strideY, const float *T,
                                 const uint32_t *idx, long long idx_stride, int n, int out_dim,
                                 const float *tmean, const float *tinv, bf16 *dY,
                                 long long strideD, float *loss, const TrainStep *st) {
  const int z = blockIdx.z;
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  float l = 0.0f;
  if (st) idx += st->offset;
  if (e < (long long)n * out_dim) {
    const int r = (int)(e / out_dim), c = (int)(e % out_dim);
    const uint32_t row = idx[z * idx_stride + r];
    const float t = (T[(long long)row * out_dim + c] - tmean[c]) * tinv[c];
    const float d = Yp[z * strideY + e] - t;
    l = d * d;
    dY[z * strideD + e] = __float2bfloat16(2.0f * d / (float)((long long)n * out_dim));
  }
  for (int o = 16; o > 0; o >>= 1) l += __shfl_down_sync(0xffffffffu, l, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(&loss[z], l / (float)((long long)n * out_dim));
}

// db[j] += sum over rows [y*rows_per, (y+1)*rows_per) of dZ[:, j] (BF16 in,
// FP32 out): one row slice per blockIdx.y, the slices added atomically.
__global__ void bias_grad_kernel(const bf16 *dZ, long long strideD, int n, int cols, int rows_per,
                                 float *db, long long strideB) {
  const int z = blockIdx.z;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cols) return;
  const long long r0 = (long long)blockIdx.y * rows_per;
  const long long r1 = r0 + rows_per < n ? r0 + rows_per : n;
  const bf16 *src = dZ + z * strideD + c;
  float s = 0.0f;
  for (long long r = r0; r < r1; ++r) s += __bfloat162float(src[r * cols]);
  atomicAdd(&db[z * strideB + c], s);
}

// dH = (dZ W^T) * gelu'(Z) of a layer whose fan-out fo is not a multiple
// of 16 (the output layer): fo FP32 multiply-adds of the BF16 operands per
// element, in order, then the GELU derivative and one rounding to BF16 --
// the tensor-core kernel's arithmetic for a K this narrow.
__global__ void narrow_back_kernel(const bf16 *dZ, int ld_dz, long long stride_dz, const bf16 *W,
                                   long long strideW, int fo, const float *Z, int ldz,
                                   long long strideZ, bf16 *dH, int ldh, long long strideH, int n,
                                   int fi) {
  // thread j: hidden unit j (fi <= blockDim.x), its fo weights held in
  // registers when fo <= 4; blocks stride over the rows, four at a time
  const int zm = blockIdx.z;
  const int j = threadIdx.x;
  if (j >= fi) return;
  const bf16 *w = W + zm * strideW + (long long)j * fo;
  const bf16 *dzm = dZ + zm * stride_dz;
  const float *Zm = Z + zm * strideZ;
  bf16 *dHm = dH + zm * strideH;
  if (fo <= 4) {
    float wr[4];
#pragma unroll
    for (int o = 0; o < 4; ++o) wr[o] = o < fo ? __bfloat162float(w[o]) : 0.0f;
    for (int r0 = blockIdx.x * 4; r0 < n; r0 += gridDim.x * 4) {
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int r = r0 + i;
        if (r >= n) break;
        const bf16 *dz = dzm + (long long)r * ld_dz;
        float acc = 0.0f;
#pragma unroll
        for (int o = 0; o < 4; ++o)
          if (o < fo) acc = fmaf(__bfloat162float(dz[o]), wr[o], acc);
        const float zz = Zm[(long long)r * ldz + j];
        dHm[(long long)r * ldh + j] = __float2bfloat16(acc * gelu_grad(zz));
      }
    }
    return;
  }
  for (int r = blockIdx.x; r < n; r += gridDim.x) {
    const bf16 *dz = dzm + (long long)r * ld_dz;
    float acc = 0.0f;
    for (int o = 0; o < fo; ++o) acc = fmaf(__bfloat162float(dz[o]), __bfloat162float(w[o]), acc);
    const float zz = Zm[(long long)r * ldz + j];
    dHm[(long long)r * ldh + j] = __float2bfloat16(acc * gelu_grad(zz));
  }
}

// Adam on the FP32 master weights; refreshes the BF16 mirror.
// Adam step number st->t + 1 with learning rate st->lr.
__global__ void adam_kernel(float *w, const float *grad, float *m, float *v, bf16 *w16,
                            long long n, const TrainStep *st, float b1, float b2, float eps) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float t = (float)(st->t + 1);
  const float c1 = 1.0f - powf(b1, t), c2 = 1.0f - powf(b2, t);
  const float lr = st->lr;
  const float gr = grad[i];
  const float mi = b1 * m[i] + (1.0f - b1) * gr;
  const float vi = b2 * v[i] + (1.0f - b2) * gr * gr;
  m[i] = mi;
  v[i] = vi;
  const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  w[i] = wi;
  if (w16) w16[i] = __float2bfloat16(wi);
}

__global__ void to_bf16_kernel(const float *x, bf16 *y, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = __float2bfloat16(x[i]);
}

// Ensemble mean and standard deviation of de-normalised outputs.
__global__ void ensemble_kernel(const float *Y, long long strideY, int E, long long n_out,
                                const float *tmean, const float *tstd, int out_dim, float *mean,
                                float *spread) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n_out) return;
  const int c = (int)(e % out_dim);
  float s = 0.0f, s2 = 0.0f;
  for (int z = 0; z < E; ++z) {
    const float y = Y[z * strideY + e] * tstd[c] + tmean[c];
    s += y;
    s2 += y * y;
  }
  const float mu = s / E;
  mean[e] = mu;
  if (spread) spread[e] = sqrtf(fmaxf(s2 / E - mu * mu, 0.0f));
}

#define MLP_TRY(expr)                                                                    \
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

struct mcml_mlp {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int in_dim = 0, in_pad = 0, hidden = 0, depth = 0, out_dim = 0, E = 0;
  int layers = 0;                  // depth + 1 weight matrices
  std::vector<int> fan_in, fan_out;
  std::vector<long long> w_off, b_off;  // offsets into the per-member parameter block
  long long per_member = 0;        // parameters per member
  long long stride = 0;            // per_member rounded up to 8 (16-byte aligned BF16 blocks)
  unsigned *d_status = nullptr;    // tensor-core kernel timeouts
  // Polls per pipeline wait of the tensor-core kernel before it gives up:
  // kTcSpin, or MCML_MLP_WAIT_POLLS read once when the network is created
  // (a test sets it tiny to make the waits run out on purpose).
  long long spin = kTcSpin;
  float *d_w = nullptr;            // E x stride FP32 master (weights then biases per layer)
  float *d_m = nullptr, *d_v = nullptr, *d_g = nullptr;
  bf16 *d_w16 = nullptr;           // BF16 mirror (same layout)
  float *d_xmean = nullptr, *d_xinv = nullptr, *d_tmean = nullptr, *d_tinv = nullptr,
        *d_tstd = nullptr;
  std::vector<float> h_tmean, h_tstd;
  long long adam_t = 0;
  // activations for a batch of up to cap rows
  int cap = 0;
  // whole-network inference (tc_fused_forward_kernel): inputs and outputs of
  // up to fcap rows, and the CTAs' activation scratch
  bf16 *d_fx = nullptr;            // fcap x in_pad rounded up to 64
  float *d_fy = nullptr;           // E x fcap x out
  bf16 *d_act = nullptr;           // batch rows x hidden per CTA
  unsigned char *d_wimg = nullptr; // packed B images of the weights (E x image)
  long long fcap = 0;
  bf16 *d_x = nullptr;             // E x cap x in_pad
  float *d_z = nullptr;            // E x depth x cap x hidden (pre-activations)
  bf16 *d_h = nullptr;             // E x depth x cap x hidden (activations)
  float *d_y = nullptr;            // E x cap x out
  bf16 *d_dy = nullptr;            // E x cap x max(hidden, out)
  bf16 *d_dh = nullptr;            // E x cap x hidden
  uint32_t *d_idx = nullptr;       // E x cap
  float *d_loss = nullptr;         // E
  uint32_t *d_perm = nullptr;      // E x n: one epoch's shuffles
  TrainStep *d_step = nullptr;     // device-side minibatch offset, Adam step, learning rate
  TrainStep h_step{};              // staging for its upload
  // One recorded training step (a CUDA graph), replayed for every full
  // minibatch of an epoch; recorded again when its inputs (X, T, n, batch,
  // activation buffers) change.
  cudaGraphExec_t step_exec = nullptr;
  const float *step_X = nullptr, *step_T = nullptr;
  uint64_t step_n = 0;
  uint32_t step_batch = 0;
  long long step_cap = 0;
  size_t perm_cap = 0;

  ~mcml_mlp() {
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != device) cudaSetDevice(device);
    if (stream) cudaStreamSynchronize(stream);
    dfree(d_w); dfree(d_m); dfree(d_v); dfree(d_g); dfree(d_w16);
    dfree(d_xmean); dfree(d_xinv); dfree(d_tmean); dfree(d_tinv); dfree(d_tstd);
    dfree(d_x); dfree(d_z); dfree(d_h); dfree(d_y); dfree(d_dy); dfree(d_dh); dfree(d_idx);
    dfree(d_loss);
    dfree(d_perm);
    dfree(d_step);
    dfree(d_fx);
    dfree(d_fy);
    dfree(d_act);
    dfree(d_wimg);
    if (step_exec) cudaGraphExecDestroy(step_exec);
    dfree(d_status);
    if (own_stream && stream) cudaStreamDestroy(stream);
    if (prev >= 0 && prev != device) cudaSetDevice(prev);
  }
};

namespace {

struct MlpGuard {
  int prev = -1;
  bool changed = false;
  explicit MlpGuard(int dev) {
    if (cudaGetDevice(&prev) == cudaSuccess && prev != dev) changed = cudaSetDevice(dev) == cudaSuccess;
  }
  ~MlpGuard() {
    if (changed) cudaSetDevice(prev);
  }
};

int ensure_cap(mcml_mlp *p, int rows) {
  if (rows <= p->cap) return MCML_OK;
  dfree(p->d_x); dfree(p->d_z); dfree(p->d_h); dfree(p->d_y); dfree(p->d_dy); dfree(p->d_dh);
  dfree(p->d_idx);
  p->cap = 0;
  const long long E = p->E, H = p->hidden, D = p->depth;
  MLP_TRY(cudaMalloc(&p->d_x, E * rows * p->in_pad * sizeof(bf16)));
  MLP_TRY(cudaMalloc(&p->d_z, E * D * rows * H * sizeof(float)));
  MLP_TRY(cudaMalloc(&p->d_h, E * D * rows * H * sizeof(bf16)));
  MLP_TRY(cudaMalloc(&p->d_y, E * rows * p->out_dim * sizeof(float)));
  MLP_TRY(cudaMalloc(&p->d_dy, E * rows * std::max<long long>(H, p->out_dim) * sizeof(bf16)));
  MLP_TRY(cudaMalloc(&p->d_dh, E * rows * H * sizeof(bf16)));
  MLP_TRY(cudaMalloc(&p->d_idx, E * rows * sizeof(uint32_t)));
  p->cap = rows;
  return MCML_OK;
}

// Forward of all members on rows [0, n) already gathered into d_x, on the
// tensor cores (tc_layer_kernel): hidden layers keep Z (FP32) for the
// backward pass and H (BF16) for the next layer; the output layer writes Y.
// shared_x: every member reads the same normalised input rows (inference),
// gathered once instead of once per member.
int forward(mcml_mlp *p, int n, bool keep_z, bool shared_x = false) {
  const long long H = p->hidden, cap = p->cap, P = p->stride, D = p->depth;
  for (int l = 0; l < p->layers; ++l) {
    TcArgs g;
    std::memset(&g, 0, sizeof(g));
    g.M = n;
    g.K = l == 0 ? p->in_pad : (int)H;
    g.n_valid = p->fan_out[l];
    g.N = (p->fan_out[l] + 15) / 16 * 16;
    if (l == 0) {
      g.A = p->d_x;
      g.lda = p->in_pad;
      g.strideA = shared_x ? 0 : cap * p->in_pad;
    } else {
      g.A = p->d_h + (long long)(l - 1) * cap * H;
      g.lda = H;
      g.strideA = D * cap * H;
    }
    g.W = p->d_w16 + p->w_off[l];
    g.strideW = P;
    g.bias = p->d_w + p->b_off[l];
    g.strideBias = P;
    g.status = p->d_status;
    g.spin = p->spin;
    if (l < p->depth) {
      g.Z = keep_z ? p->d_z + (long long)l * cap * H : nullptr;
      g.ldz = H;
      g.strideZ = D * cap * H;
      g.H = p->d_h + (long long)l * cap * H;
      g.ldh = H;
      g.strideH = D * cap * H;
      MLP_TRY(tc_layer<kTcBiasGelu>(g, p->E, p->stream));
    } else {
      g.Z = p->d_y;
      g.ldz = p->out_dim;
      g.strideZ = cap * p->out_dim;
      MLP_TRY(tc_layer<kTcBias>(g, p->E, p->stream));
    }
  }
  return MCML_OK;
}

// Tensor-core kernel timeouts seen so far (then cleared): MCML_E_BUDGET.
int check_status(mcml_mlp *p) {
  unsigned st = 0;
  MLP_TRY(cudaMemcpyAsync(&st, p->d_status, sizeof(st), cudaMemcpyDeviceToHost, p->stream));
  MLP_TRY(cudaStreamSynchronize(p->stream));
  if (st) {
    MLP_TRY(cudaMemset(p->d_status, 0, sizeof(unsigned)));
    // bit 0: a pipeline wait gave up (the layer's tiles are incomplete);
    // bit 1: even the end-of-kernel drain of issued copies and MMAs did
    if (st & 2u)
      return set_error(MCML_E_BUDGET, "tensor-core kernel: a pipeline wait and the drain of "
                                      "its issued copies and MMAs timed out");
    return set_error(MCML_E_BUDGET, "tensor-core kernel: a pipeline wait timed out "
                                    "(issued copies and MMAs drained)");
  }
  return MCML_OK;
}

// Whole-network inference (tc_fused_forward_kernel) applies when every
// hidden layer can stream its activations by TMA and store them in 32-column
// TMA tiles: hidden width a multiple of 64, at most kMaxFusedLayers layers,
// an output of at most kFusedMaxOut columns, hidden biases at 8-byte-aligned
// offsets.  Its results differ from the layer kernel's only by the order in
// which the output layer's FP32 sums are added (a few units in the last
// place).
bool fused_eligible(const mcml_mlp *p) {
  if (!(p->hidden % 64 == 0 && p->hidden <= 256 && p->layers <= kMaxFusedLayers &&
        p->layers >= 2 && p->out_dim <= kFusedMaxOut && p->in_pad <= 256))
    return false;
  for (int l = 0; l + 1 < p->layers; ++l)
    if (p->b_off[l] % 2) return false;
  return true;
}

constexpr int kFusedBatchRows = 1024;         // rows a CTA takes through all layers at once
constexpr long long kFusedRows = 1ll << 22;   // rows per launch

// Tensor map over a BF16 row-major array (cols x rows, one plane) with the
// given box and swizzle.
bool encode_rows_map(void *base, long long cols, long long rows, cuuint32_t bx, cuuint32_t by,
                     CUtensorMapSwizzle sw, CUtensorMap *map) {
  EncodeTiledFn fn = encode_tiled();
  if (!fn) return false;
  const cuuint64_t dims[3] = {(cuuint64_t)cols, (cuuint64_t)rows, 1};
  const cuuint64_t strides[2] = {(cuuint64_t)cols * 2, (cuuint64_t)rows * cols * 2};
  const cuuint32_t box[3] = {bx, by, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  return fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, base, dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, sw, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

int fused_predict(mcml_mlp *p, const float *X, uint64_t n, float *mean, float *spread) {
  int dev = 0, sms = 0;
  MLP_TRY(cudaGetDevice(&dev));
  MLP_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int per_member = std::max(1, sms / p->E);
  const long long ctas = (long long)per_member * p->E;
  const long long scratch_rows = ctas * kFusedBatchRows;
  const long long rows_cap = std::min<long long>(kFusedRows, (long long)n);
  const int in64 = (p->in_pad + 63) / 64 * 64;  // layer 0's contraction width
  if (!p->d_act) {
    MLP_TRY(cudaMalloc(&p->d_act, scratch_rows * p->hidden * sizeof(bf16)));
  }
  if (rows_cap > p->fcap) {
    dfree(p->d_fx);
    dfree(p->d_fy);
    p->fcap = 0;
    MLP_TRY(cudaMalloc(&p->d_fx, rows_cap * in64 * sizeof(bf16)));
    MLP_TRY(cudaMalloc(&p->d_fy, p->E * rows_cap * p->out_dim * sizeof(float)));
    p->fcap = rows_cap;
  }
  // B images of the current weights
  FusedPack pk;
  std::memset(&pk, 0, sizeof(pk));
  FusedArgs f;
  std::memset(&f, 0, sizeof(f));
  pk.layers = p->layers;
  long long img_bytes = 0, elems = 0;
  int maxB = 0;
  for (int l = 0; l < p->layers; ++l) {
    const int K = l == 0 ? in64 : p->fan_in[l];
    const int N = (p->fan_out[l] + 15) / 16 * 16;
    pk.K[l] = f.K[l] = K;
    pk.N[l] = f.N[l] = N;
    pk.fan_in[l] = p->fan_in[l];
    pk.n_valid[l] = f.n_valid[l] = p->fan_out[l];
    pk.w_off[l] = p->w_off[l];
    pk.elem_begin[l] = elems;
    pk.img_off[l] = f.img_off[l] = img_bytes;
    f.b_off[l] = p->b_off[l];
    elems += (long long)K * N;
    img_bytes += (long long)K * N * 2;
    maxB = std::max(maxB, K * N * 2);
  }
  pk.elem_begin[p->layers] = elems;
  if (!p->d_wimg) MLP_TRY(cudaMalloc(&p->d_wimg, p->E * img_bytes));
  fused_pack_kernel<<<dim3((unsigned)((elems + 255) / 256), 1, p->E), 256, 0, p->stream>>>(
      p->d_w16, p->stride, pk, p->d_wimg, img_bytes);
  MLP_TRY(cudaGetLastError());
  CUtensorMap xmap, amap, hmap;
  std::memset(&xmap, 0, sizeof(xmap));
  std::memset(&amap, 0, sizeof(amap));
  std::memset(&hmap, 0, sizeof(hmap));
  if (!encode_rows_map(p->d_fx, in64, p->fcap, 64, TCM, CU_TENSOR_MAP_SWIZZLE_128B, &xmap) ||
      !encode_rows_map(p->d_act, p->hidden, scratch_rows, 64, TCM, CU_TENSOR_MAP_SWIZZLE_128B,
                       &amap) ||
      !encode_rows_map(p->d_act, p->hidden, scratch_rows, 32, 32, CU_TENSOR_MAP_SWIZZLE_64B, &hmap))
    return set_error(MCML_E_CUDA, "mlp: tensor maps of the fused forward");
  f.layers = p->layers;
  f.batch_rows = kFusedBatchRows;
  f.img = p->d_wimg;
  f.W16 = p->d_w16;
  f.w_off_out = p->w_off[p->layers - 1];
  f.b_off_out = p->b_off[p->layers - 1];
  f.out_dim = p->out_dim;
  f.img_stride = img_bytes;
  f.Wf = p->d_w;
  f.strideW = p->stride;
  f.status = p->d_status;
  f.spin = p->spin;
  // weights, one staging tile per epilogue warp, three bias buffers, 58
  // barriers, TMEM slot, 1 KB of alignment slack
  const size_t fixed =
      tc_align1k((size_t)maxB) + kFusedEpiWarps * 2048 + 3 * 256 * 4 + 256 * 16 +
      2 * (kFusedParts - 1) * 128 * 3 * 4 + 60 * 8 + 16 + 1024;
  const size_t slot = tc_slot_bytes(64);
  f.slots = (int)std::min<size_t>(16, (kTcSmemMax - fixed) / slot);
  if (f.slots < 2) return set_error(MCML_E_INVALID, "mlp: layers too wide for the fused forward");
  const size_t smem = fixed + (size_t)f.slots * slot;
  static std::atomic<bool> configured[64];
  if (dev >= 0 && dev < 64 && !configured[dev].load()) {
    MLP_TRY(cudaFuncSetAttribute(tc_fused_forward_kernel,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmemMax));
    configured[dev].store(true);
  }
  for (uint64_t r0 = 0; r0 < n; r0 += (uint64_t)rows_cap) {
    const int rows = (int)std::min<uint64_t>((uint64_t)rows_cap, n - r0);
    gather_x_kernel<<<dim3((unsigned)(((long long)rows * in64 + 255) / 256), 1, 1), 256, 0,
                      p->stream>>>(X + r0 * p->in_dim, nullptr, rows, p->in_dim, in64,
                                   p->d_xmean, p->d_xinv, 0, p->d_fx, 0, nullptr);
    MLP_TRY(cudaGetLastError());
    f.n = rows;
    f.Y = p->d_fy;
    tc_fused_forward_kernel<<<dim3(per_member, 1, p->E), kFusedWarps * 32, smem, p->stream>>>(
        f, xmap, amap, hmap);
    MLP_TRY(cudaGetLastError());
    ensemble_kernel<<<(unsigned)(((long long)rows * p->out_dim + 255) / 256), 256, 0, p->stream>>>(
        p->d_fy, (long long)rows * p->out_dim, p->E, (long long)rows * p->out_dim, p->d_tmean,
        p->d_tstd, p->out_dim, mean + r0 * p->out_dim, spread ? spread + r0 * p->out_dim : nullptr);
    MLP_TRY(cudaGetLastError());
  }
  return MCML_OK;
}

// Backward from dY (in d_dy, BF16) to all weight/bias gradients in d_g.
int backward(mcml_mlp *p, int n) {
  const long long H = p->hidden, cap = p->cap, P = p->stride, D = p->depth;
  // dW = X^T dZ runs over the batch: split it so that a few layers of
  // 256 x 256 still fill the GPU, partial sums added atomically into d_g
  const int splits = std::max(1, std::min(16, n / 256));
  const int kper = ((n + splits - 1) / splits + BK - 1) / BK * BK;
  MLP_TRY(cudaMemsetAsync(p->d_g, 0, p->E * P * sizeof(float), p->stream));
  // with whole slices of 256 rows the weight gradients run on the tensor
  // cores: one slice per CTA group, A = X_l^T read MN-major from X_l
  const bool tc_dw = n % 256 == 0;
  bf16 *dcur = p->d_dy;   // gradient w.r.t. the current layer's output (pre-activation)
  bf16 *dnext = p->d_dh;
  long long dcur_ld = p->out_dim;
  for (int l = p->layers - 1; l >= 0; --l) {
    const int fo = p->fan_out[l], fi = p->fan_in[l];
    // dW_l = X_l^T dZ_l  (M = fi, N = fo, K = n)
    if (tc_dw) {
      TcArgs w;
      std::memset(&w, 0, sizeof(w));
      w.M = fi;
      w.N = (fo + 15) / 16 * 16;
      w.n_valid = fo;
      w.K = 256;
      w.A = l == 0 ? p->d_x : p->d_h + (long long)(l - 1) * cap * H;
      w.lda = l == 0 ? p->in_pad : H;
      w.strideA = l == 0 ? cap * p->in_pad : D * cap * H;
      w.sliceA = 256 * w.lda;
      w.W = dcur;
      w.strideW = cap * std::max<long long>(H, p->out_dim);
      w.sliceW = 256 * dcur_ld;
      w.Z = p->d_g + p->w_off[l];
      w.ldz = fo;
      w.strideZ = P;
      w.splits = n / 256;
      w.status = p->d_status;
      w.spin = p->spin;
      MLP_TRY((tc_layer<kTcAddF32, false, true>(w, p->E, p->stream)));
    } else {
    GemmArgs g;
    std::memset(&g, 0, sizeof(g));
    g.M = fi;
    g.N = fo;
    g.K = n;
    if (l == 0) {
      g.A = p->d_x;
      g.lda = p->in_pad;
      g.strideA = cap * p->in_pad;
    } else {
      g.A = p->d_h + (long long)(l - 1) * cap * H;
      g.lda = H;
      g.strideA = D * cap * H;
    }
    g.B = dcur;
    g.ldb = dcur_ld;
    g.strideB = cap * std::max<long long>(H, p->out_dim);
    g.outF = p->d_g + p->w_off[l];
    g.ldo = fo;
    g.strideO = P;
    // the batch dimension split over blocks (d_g zeroed above)
    g.splits = splits;
    g.kper = kper;
    MLP_TRY((gemm<true, false, kStoreF32>(g, p->E, p->stream)));
    }
    // db_l = column sums of dZ_l: blocks of 128 columns x 64 rows (more
    // rows per block only past 65535 row blocks), partial sums added
    // atomically into d_g (zeroed above)
    {
      const int rows_per = std::max(64, (n + 65534) / 65535);
      bias_grad_kernel<<<dim3((fo + 127) / 128, (n + rows_per - 1) / rows_per, p->E), 128, 0,
                         p->stream>>>(dcur, cap * std::max<long long>(H, p->out_dim), n, fo, rows_per,
                                      p->d_g + p->b_off[l], P);
    }
    MLP_TRY(cudaGetLastError());
    if (l == 0) break;
    // dZ_{l-1} = (dZ_l W_l^T) * gelu'(Z_{l-1})   (M = n, N = fi, K = fo):
    // on the tensor cores (W_l as a K-major B operand) when fo is a hidden
    // width; the output layer's narrow fo (3 multiply-adds per element) on
    // the CUDA cores
    if (fo % 16 == 0) {
      TcArgs t;
      std::memset(&t, 0, sizeof(t));
      t.M = n;
      t.N = fi;
      t.n_valid = fi;
      t.K = fo;
      t.A = dcur;
      t.lda = dcur_ld;
      t.strideA = cap * std::max<long long>(H, p->out_dim);
      t.W = p->d_w16 + p->w_off[l];
      t.strideW = P;
      t.aux = p->d_z + (long long)(l - 1) * cap * H;
      t.ldaux = H;
      t.strideAux = D * cap * H;
      t.H = dnext;
      t.ldh = H;
      t.strideH = cap * std::max<long long>(H, p->out_dim);
      t.status = p->d_status;
      t.spin = p->spin;
      MLP_TRY((tc_layer<kTcGeluBack, true>(t, p->E, p->stream)));
      std::swap(dcur, dnext);
      dcur_ld = H;
      continue;
    }
    // one thread per hidden unit (fi <= 256), blocks striding over the rows
    narrow_back_kernel<<<dim3((unsigned)std::min((n + 3) / 4, 1024), 1, p->E), 256, 0,
                         p->stream>>>(
        dcur, dcur_ld, cap * std::max<long long>(H, p->out_dim), p->d_w16 + p->w_off[l], P, fo,
        p->d_z + (long long)(l - 1) * cap * H, (int)H, D * cap * H, dnext, (int)H,
        cap * std::max<long long>(H, p->out_dim), n, fi);
    MLP_TRY(cudaGetLastError());
    std::swap(dcur, dnext);
    dcur_ld = H;
  }
  return MCML_OK;
}

}  // namespace

extern "C" {

int mcml_mlp_create(const mcml_mlp_config *cfg, mcml_mlp **out) {
  clear_error();
  if (!cfg || !out) return set_error(MCML_E_INVALID, "mcml_mlp_create: null argument");
  *out = nullptr;
  // The tensor-core forward takes K <= 256 and N <= 256 in multiples of 16.
  if (cfg->in_dim < 1 || cfg->hidden < 16 || cfg->depth < 1 || cfg->out_dim < 1 ||
      cfg->ensemble < 1 || cfg->in_dim > 256 || cfg->hidden > 256 || cfg->hidden % 16 != 0 ||
      cfg->out_dim > cfg->hidden)
    return set_error(MCML_E_INVALID,
                     "mcml_mlp_create: bad dimensions (in_dim <= 256; hidden a multiple of 16, "
                     "at most 256; out_dim <= hidden)");
  std::unique_ptr<mcml_mlp> p(new mcml_mlp());
  p->device = cfg->device;
  if (const char *e = std::getenv("MCML_MLP_WAIT_POLLS")) {
    const long long v = std::atoll(e);
    if (v > 0) p->spin = v;
  }
  MlpGuard gd(cfg->device);
  p->in_dim = cfg->in_dim;
  p->in_pad = (cfg->in_dim + 15) / 16 * 16;
  p->hidden = cfg->hidden;
  p->depth = cfg->depth;
  p->out_dim = cfg->out_dim;
  p->E = cfg->ensemble;
  p->layers = cfg->depth + 1;
  long long off = 0;
  for (int l = 0; l < p->layers; ++l) {
    const int fi = l == 0 ? p->in_pad : p->hidden;
    const int fo = l == p->depth ? p->out_dim : p->hidden;
    p->fan_in.push_back(fi);
    p->fan_out.push_back(fo);
    p->w_off.push_back(off);
    off += (long long)fi * fo;
    p->b_off.push_back(off);
    off += fo;
  }
  p->per_member = off;
  p->stride = (off + 7) / 8 * 8;
  const long long total = p->stride * p->E;
  if (cfg->stream) {
    p->stream = (cudaStream_t)cfg->stream;
  } else {
    MLP_TRY(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking));
    p->own_stream = true;
  }
  MLP_TRY(cudaMalloc(&p->d_step, sizeof(TrainStep)));
  MLP_TRY(cudaMalloc(&p->d_w, total * sizeof(float)));
  MLP_TRY(cudaMalloc(&p->d_m, total * sizeof(float)));
  MLP_TRY(cudaMalloc(&p->d_v, total * sizeof(float)));
  MLP_TRY(cudaMalloc(&p->d_g, total * sizeof(float)));
  MLP_TRY(cudaMalloc(&p->d_w16, total * sizeof(bf16)));
  MLP_TRY(cudaMalloc(&p->d_xmean, p->in_pad * sizeof(float)));
  MLP_TRY(cudaMalloc(&p->d_xinv, p->in_pad * sizeof(float)));
  MLP_TRY(cudaMalloc(&p->d_tmean, p->out_dim * sizeof(float)));
  MLP_TRY(cudaMalloc(&p->d_tinv, p->out_dim * sizeof(float)));
  MLP_TRY(cudaMalloc(&p->d_tstd, p->out_dim * sizeof(float)));
  MLP_TRY(cudaMalloc(&p->d_loss, p->E * sizeof(float)));
  MLP_TRY(cudaMalloc(&p->d_status, sizeof(unsigned)));
  MLP_TRY(cudaMemset(p->d_status, 0, sizeof(unsigned)));
  // He-uniform weights (per member seed), zero biases; the padded input
  // rows of the first matrix are zero.
  std::vector<float> w(total, 0.0f);
  for (int e = 0; e < p->E; ++e) {
    std::mt19937_64 rng(cfg->seed * 1000003ull + (uint64_t)e);
    for (int l = 0; l < p->layers; ++l) {
      const int fi = p->fan_in[l], fo = p->fan_out[l];
      const int real_in = l == 0 ? p->in_dim : fi;
      const float lim = std::sqrt(6.0f / (float)real_in) * (l == p->depth ? 0.5f : 1.0f);
      std::uniform_real_distribution<float> U(-lim, lim);
      float *W = w.data() + (long long)e * p->stride + p->w_off[l];
      for (int i = 0; i < fi; ++i)
        for (int j = 0; j < fo; ++j) W[(long long)i * fo + j] = i < real_in ? U(rng) : 0.0f;
    }
  }
  MLP_TRY(cudaMemcpy(p->d_w, w.data(), total * sizeof(float), cudaMemcpyHostToDevice));
  MLP_TRY(cudaMemset(p->d_m, 0, total * sizeof(float)));
  MLP_TRY(cudaMemset(p->d_v, 0, total * sizeof(float)));
  to_bf16_kernel<<<(unsigned)((total + 255) / 256), 256, 0, p->stream>>>(p->d_w, p->d_w16, total);
  MLP_TRY(cudaGetLastError());
  std::vector<float> zeros(p->in_pad, 0.0f), ones(p->in_pad, 1.0f);
  MLP_TRY(cudaMemcpy(p->d_xmean, zeros.data(), p->in_pad * sizeof(float), cudaMemcpyHostToDevice));
  MLP_TRY(cudaMemcpy(p->d_xinv, ones.data(), p->in_pad * sizeof(float), cudaMemcpyHostToDevice));
  p->h_tmean.assign(p->out_dim, 0.0f);
  p->h_tstd.assign(p->out_dim, 1.0f);
  MLP_TRY(cudaMemcpy(p->d_tmean, p->h_tmean.data(), p->out_dim * sizeof(float), cudaMemcpyHostToDevice));
  MLP_TRY(cudaMemcpy(p->d_tinv, p->h_tstd.data(), p->out_dim * sizeof(float), cudaMemcpyHostToDevice));
  MLP_TRY(cudaMemcpy(p->d_tstd, p->h_tstd.data(), p->out_dim * sizeof(float), cudaMemcpyHostToDevice));
  MLP_TRY(cudaStreamSynchronize(p->stream));
  *out = p.release();
  return MCML_OK;
}

int mcml_mlp_set_normalization(mcml_mlp *p, const float *x_mean, const float *x_std,
                               const float *t_mean, const float *t_std) {
  clear_error();
  if (!p || !x_mean || !x_std || !t_mean || !t_std) return set_error(MCML_E_INVALID, "null argument");
  MlpGuard gd(p->device);
  std::vector<float> xm(p->in_pad, 0.0f), xi(p->in_pad, 0.0f), tm(p->out_dim), ti(p->out_dim),
      ts(p->out_dim);
  for (int i = 0; i < p->in_dim; ++i) {
    xm[i] = x_mean[i];
    xi[i] = x_std[i] > 0 ? 1.0f / x_std[i] : 0.0f;  // a constant feature contributes nothing
  }
  for (int j = 0; j < p->out_dim; ++j) {
    tm[j] = t_mean[j];
    ts[j] = t_std[j] > 0 ? t_std[j] : 1.0f;
    ti[j] = 1.0f / ts[j];
  }
  p->h_tmean = tm;
  p->h_tstd = ts;
  MLP_TRY(cudaMemcpy(p->d_xmean, xm.data(), p->in_pad * sizeof(float), cudaMemcpyHostToDevice));
  MLP_TRY(cudaMemcpy(p->d_xinv, xi.data(), p->in_pad * sizeof(float), cudaMemcpyHostToDevice));
  MLP_TRY(cudaMemcpy(p->d_tmean, tm.data(), p->out_dim * sizeof(float), cudaMemcpyHostToDevice));
  MLP_TRY(cudaMemcpy(p->d_tinv, ti.data(), p->out_dim * sizeof(float), cudaMemcpyHostToDevice));
  MLP_TRY(cudaMemcpy(p->d_tstd, ts.data(), p->out_dim * sizeof(float), cudaMemcpyHostToDevice));
  return MCML_OK;
}

int64_t mcml_mlp_num_params(const mcml_mlp *p) { return p ? p->per_member : -1; }

int mcml_mlp_get_params(mcml_mlp *p, float *host, int member) {
  clear_error();
  if (!p || !host || member < 0 || member >= p->E) return set_error(MCML_E_INVALID, "bad argument");
  MlpGuard gd(p->device);
  MLP_TRY(cudaStreamSynchronize(p->stream));
  MLP_TRY(cudaMemcpy(host, p->d_w + (long long)member * p->stride, p->per_member * sizeof(float),
                     cudaMemcpyDeviceToHost));
  return MCML_OK;
}

int mcml_mlp_set_params(mcml_mlp *p, const float *host, int member) {
  clear_error();
  if (!p || !host || member < 0 || member >= p->E) return set_error(MCML_E_INVALID, "bad argument");
  MlpGuard gd(p->device);
  float *dst = p->d_w + (long long)member * p->stride;
  MLP_TRY(cudaMemcpy(dst, host, p->per_member * sizeof(float), cudaMemcpyHostToDevice));
  to_bf16_kernel<<<(unsigned)((p->per_member + 255) / 256), 256, 0, p->stream>>>(
      dst, p->d_w16 + (long long)member * p->stride, p->per_member);
  MLP_TRY(cudaGetLastError());
  MLP_TRY(cudaStreamSynchronize(p->stream));
  return MCML_OK;
}

// One forward + backward on rows [0, n) of (X, T) for every member (no
// update): loss per member and the FP32 gradients (host, E x num_params).
int mcml_mlp_gradients(mcml_mlp *p, const float *X, const float *T, int n, float *loss_out,
                       float *grads_out) {
  clear_error();
  if (!p || !X || !T || n < 1) return set_error(MCML_E_INVALID, "bad argument");
  MlpGuard gd(p->device);
  int rc = ensure_cap(p, n);
  if (rc) return rc;
  std::vector<uint32_t> idx((size_t)p->E * p->cap, 0);
  for (int e = 0; e < p->E; ++e)
    for (int i = 0; i < n; ++i) idx[(size_t)e * p->cap + i] = (uint32_t)i;
  MLP_TRY(cudaMemcpyAsync(p->d_idx, idx.data(), idx.size() * sizeof(uint32_t), cudaMemcpyHostToDevice,
                          p->stream));
  const long long cap = p->cap;
  gather_x_kernel<<<dim3((unsigned)((n * p->in_pad + 255) / 256), 1, p->E), 256, 0, p->stream>>>(
      X, p->d_idx, n, p->in_dim, p->in_pad, p->d_xmean, p->d_xinv, cap, p->d_x, cap * p->in_pad,
      nullptr);
  MLP_TRY(cudaGetLastError());
  rc = forward(p, n, true);
  if (rc) return rc;
  MLP_TRY(cudaMemsetAsync(p->d_loss, 0, p->E * sizeof(float), p->stream));
  loss_grad_kernel<<<dim3((unsigned)((n * p->out_dim + 255) / 256), 1, p->E), 256, 0, p->stream>>>(
      p->d_y, cap * p->out_dim, T, p->d_idx, cap, n, p->out_dim, p->d_tmean, p->d_tinv, p->d_dy,
      cap * std::max(p->hidden, p->out_dim), p->d_loss, nullptr);
  MLP_TRY(cudaGetLastError());
  rc = backward(p, n);
  if (rc) return rc;
  rc = check_status(p);
  if (rc) return rc;
  if (loss_out) MLP_TRY(cudaMemcpy(loss_out, p->d_loss, p->E * sizeof(float), cudaMemcpyDeviceToHost));
  if (grads_out)
    MLP_TRY(cudaMemcpy2D(grads_out, p->per_member * sizeof(float), p->d_g,
                         p->stride * sizeof(float), p->per_member * sizeof(float), p->E,
                         cudaMemcpyDeviceToHost));
  return MCML_OK;
}

// One epoch of minibatch Adam over n rows of (X [n x in], T [n x out]),
// DEVICE arrays.  Each member sees its own shuffle.  loss_out: mean loss
// per member over the epoch (host, E floats).
int mcml_mlp_train_epoch(mcml_mlp *p, const float *X, const float *T, uint64_t n, uint32_t batch,
                         float lr, uint64_t shuffle_seed, float *loss_out) {
  clear_error();
  if (!p || !X || !T || n < 1 || batch < 1) return set_error(MCML_E_INVALID, "bad argument");
  if (n >= (1ull << 32)) return set_error(MCML_E_INVALID, "at most 2^32 - 1 rows");
  MlpGuard gd(p->device);
  int rc = ensure_cap(p, (int)std::min<uint64_t>(batch, n));
  if (rc) return rc;
  // The epoch's shuffles (one per member) go to the device in one copy;
  // minibatches index into them, so the steps below never wait for the host.
  std::vector<uint32_t> perm((size_t)p->E * n);
  for (int e = 0; e < p->E; ++e) {
    uint32_t *pe = &perm[(size_t)e * n];
    for (uint64_t i = 0; i < n; ++i) pe[i] = (uint32_t)i;
    std::mt19937_64 rng(shuffle_seed * 7919ull + (uint64_t)e);
    std::shuffle(pe, pe + n, rng);
  }
  if (perm.size() > p->perm_cap) {
    dfree(p->d_perm);
    p->perm_cap = 0;
    if (p->step_exec) {  // the recorded step reads the old shuffle buffer
      cudaGraphExecDestroy(p->step_exec);
      p->step_exec = nullptr;
    }
    MLP_TRY(cudaMalloc(&p->d_perm, perm.size() * sizeof(uint32_t)));
    p->perm_cap = perm.size();
  }
  MLP_TRY(cudaMemcpyAsync(p->d_perm, perm.data(), perm.size() * sizeof(uint32_t),
                          cudaMemcpyHostToDevice, p->stream));
  // d_loss sums the minibatch means over the epoch
  MLP_TRY(cudaMemsetAsync(p->d_loss, 0, p->E * sizeof(float), p->stream));
  p->h_step.offset = 0;
  p->h_step.t = p->adam_t;
  p->h_step.lr = lr;
  MLP_TRY(cudaMemcpyAsync(p->d_step, &p->h_step, sizeof(TrainStep), cudaMemcpyHostToDevice,
                          p->stream));
  // Full minibatches only (the rows left over wait for the next shuffle), or
  // one step over all rows when there are fewer than a batch.
  const int rows = (int)std::min<uint64_t>(batch, n);
  const uint64_t steps = n >= batch ? n / batch : 1;
  const long long cap = p->cap, total = p->stride * p->E;
  // one step: gather, forward, loss, backward, Adam, advance
  auto record_step = [&]() -> int {
    gather_x_kernel<<<dim3((unsigned)((rows * p->in_pad + 255) / 256), 1, p->E), 256, 0, p->stream>>>(
        X, p->d_perm, rows, p->in_dim, p->in_pad, p->d_xmean, p->d_xinv, (long long)n, p->d_x,
        cap * p->in_pad, p->d_step);
    MLP_TRY(cudaGetLastError());
    int r = forward(p, rows, true);
    if (r) return r;
    loss_grad_kernel<<<dim3((unsigned)((rows * p->out_dim + 255) / 256), 1, p->E), 256, 0, p->stream>>>(
        p->d_y, cap * p->out_dim, T, p->d_perm, (long long)n, rows, p->out_dim, p->d_tmean,
        p->d_tinv, p->d_dy, cap * std::max(p->hidden, p->out_dim), p->d_loss, p->d_step);
    MLP_TRY(cudaGetLastError());
    r = backward(p, rows);
    if (r) return r;
    adam_kernel<<<(unsigned)((total + 255) / 256), 256, 0, p->stream>>>(
        p->d_w, p->d_g, p->d_m, p->d_v, p->d_w16, total, p->d_step, 0.9f, 0.999f, 1e-8f);
    MLP_TRY(cudaGetLastError());
    advance_step_kernel<<<1, 32, 0, p->stream>>>(p->d_step, (unsigned long long)rows);
    MLP_TRY(cudaGetLastError());
    return MCML_OK;
  };
  // The ~20 launches of a step are recorded once into a CUDA graph and the
  // graph is replayed per minibatch: the launches are short and their
  // host-side set-up dominated a step.  A stream that cannot be captured
  // keeps the plain launches.
  const bool same = p->step_exec && p->step_X == X && p->step_T == T && p->step_n == n &&
                    p->step_batch == batch && p->step_cap == cap && steps > 1;
  if (!same && p->step_exec) {
    cudaGraphExecDestroy(p->step_exec);
    p->step_exec = nullptr;
  }
  if (!p->step_exec && steps > 1) {
    cudaGraph_t graph = nullptr;
    if (cudaStreamBeginCapture(p->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
      const int r = record_step();
      const cudaError_t e = cudaStreamEndCapture(p->stream, &graph);
      if (r == MCML_OK && e == cudaSuccess && graph &&
          cudaGraphInstantiate(&p->step_exec, graph, 0) == cudaSuccess) {
        p->step_X = X;
        p->step_T = T;
        p->step_n = n;
        p->step_batch = batch;
        p->step_cap = cap;
      } else {
        p->step_exec = nullptr;
      }
      if (graph) cudaGraphDestroy(graph);
    }
    cudaGetLastError();  // a failed capture leaves the plain launches below
    clear_error();
  }
  for (uint64_t k = 0; k < steps; ++k) {
    if (p->step_exec) {
      MLP_TRY(cudaGraphLaunch(p->step_exec, p->stream));
    } else {
      rc = record_step();
      if (rc) return rc;
    }
  }
  p->adam_t += (long long)steps;
  std::vector<float> loss(p->E);
  MLP_TRY(cudaMemcpyAsync(loss.data(), p->d_loss, p->E * sizeof(float), cudaMemcpyDeviceToHost,
                          p->stream));
  rc = check_status(p);
  if (rc) return rc;
  if (loss_out)
    for (int e = 0; e < p->E; ++e) loss_out[e] = loss[e] / (float)steps;
  return MCML_OK;
}

// Inference: X [n x in] DEVICE -> mean [n x out] and ensemble spread
// [n x out] (DEVICE, de-normalised).  Networks whose hidden width is a
// multiple of 64 and whose output has at most 3 columns run all layers in
// one launch per up to 2^22 rows (fused_predict; MCML_MLP_FUSED=0 in the
// environment turns it off); the others layer by layer in chunks of
// `chunk` rows (0: 131072).  Both paths round at the same points; they
// differ only in the order of the output layer's FP32 additions.
int mcml_mlp_predict(mcml_mlp *p, const float *X, uint64_t n, float *mean, float *spread,
                     uint32_t chunk) {
  clear_error();
  if (!p || !X || !mean) return set_error(MCML_E_INVALID, "bad argument");
  MlpGuard gd(p->device);
  const char *fz = std::getenv("MCML_MLP_FUSED");
  if (fused_eligible(p) && !(fz && fz[0] == '0')) return fused_predict(p, X, n, mean, spread);
  if (chunk == 0) chunk = 131072;
  int rc = ensure_cap(p, (int)std::min<uint64_t>(chunk, n));
  if (rc) return rc;
  const long long cap = p->cap;
  for (uint64_t r0 = 0; r0 < n; r0 += cap) {
    const int rows = (int)std::min<uint64_t>(cap, n - r0);
    gather_x_kernel<<<dim3((unsigned)((rows * p->in_pad + 255) / 256), 1, 1), 256, 0, p->stream>>>(
        X + r0 * p->in_dim, nullptr, rows, p->in_dim, p->in_pad, p->d_xmean, p->d_xinv, 0, p->d_x,
        cap * p->in_pad, nullptr);
    MLP_TRY(cudaGetLastError());
    rc = forward(p, rows, false, true);
    if (rc) return rc;
    ensemble_kernel<<<(unsigned)(((long long)rows * p->out_dim + 255) / 256), 256, 0, p->stream>>>(
        p->d_y, cap * p->out_dim, p->E, (long long)rows * p->out_dim, p->d_tmean, p->d_tstd,
        p->out_dim, mean + r0 * p->out_dim, spread ? spread + r0 * p->out_dim : nullptr);
    MLP_TRY(cudaGetLastError());
  }
  return MCML_OK;
}

int mcml_mlp_sync(mcml_mlp *p) {
  clear_error();
  if (!p) return set_error(MCML_E_INVALID, "null mlp");
  MlpGuard gd(p->device);
  MLP_TRY(cudaStreamSynchronize(p->stream));
  return check_status(p);
}

void mcml_mlp_destroy(mcml_mlp *p) { delete p; }

}  // extern "C"
