// probes.cu -- the walk's own device functions exercised one at a time, for
// known-answer tests of the physics (test support).
//
//   spin probe:    Photon going straight down, spin() with anisotropy g;
//                  sums of cos(theta) and cos^2(theta) -- Henyey-Greenstein
//                  gives E[cos] = g and E[cos^2] = (1 + 2 g^2) / 3.
//   reflect probe: Photon reaching an interface n1 -> n2 with incidence
//                  cosine c; reflect() decides.  Returns the reflected
//                  fraction (Fresnel's unpolarised R; 1 beyond the critical
//                  angle, ((n1-n2)/(n1+n2))^2 at normal incidence) and the
//                  mean |dz| of transmitted photons (Snell's law).
// Each thread keeps its own XORWOW subsequence and adds its sums into FP64
// accumulators with one atomic per thread.
#include <cuda_runtime.h>

#include <string>

#include "../../include/mcml_b200.h"
#include "internal.h"
#include "photon.cuh"

namespace mcml {
namespace {

__global__ void spin_probe_kernel(float g, uint64_t n, uint64_t seed, double *out) {
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  curandStateXORWOW st;
  curand_init(seed, tid, 0, &st);
  double s1 = 0.0, s2 = 0.0;
  for (uint64_t i = tid; i < n; i += stride) {
    Photon p{};
    p.dz = 1.0f;
    spin(p, g, &st);
    s1 += p.dz;
    s2 += (double)p.dz * p.dz;
  }
  atomicAdd(&out[0], s1);
  atomicAdd(&out[1], s2);
}

__global__ void reflect_probe_kernel(float n1, float n2, float cos_i, uint64_t n, uint64_t seed,
                                     double *out) {
  __shared__ SmemTables t;
  if (threadIdx.x == 0) {
    t.lay2[0] = make_float2(0.0f, n2);  // the medium above: n2
    t.lay2[1] = make_float2(0.0f, n1);  // the photon's layer: n1
  }
  __syncthreads();
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  curandStateXORWOW st;
  curand_init(seed, tid, 0, &st);
  double refl = 0.0, dz_t = 0.0;
  const float sin_i = sqrtf(fmaxf(0.0f, 1.0f - cos_i * cos_i));
  for (uint64_t i = tid; i < n; i += stride) {
    Photon p{};
    p.layer = 1;
    p.dx = sin_i;
    p.dz = -cos_i;  // moving up, towards layer 0
    if (reflect(p, 0, &st, t))
      refl += 1.0;
    else
      dz_t += fabsf(p.dz);
  }
  atomicAdd(&out[0], refl);
  atomicAdd(&out[1], dz_t);
}

}  // namespace
}  // namespace mcml

using namespace mcml;

namespace {

// Zeroed FP64 pair on `device`, the kernel launched by `launch`, the sums
// copied back and divided by n.
template <class Launch>
int run_probe(int device, uint64_t n, double *out, const char *what, Launch launch) {
  int prev = -1;
  cudaGetDevice(&prev);
  if (cudaSetDevice(device) != cudaSuccess) {
    cudaGetLastError();
    return set_error(MCML_E_INVALID, "bad device");
  }
  double *d = nullptr;
  cudaError_t e = cudaMalloc(&d, 2 * sizeof(double));
  if (e == cudaSuccess) e = cudaMemset(d, 0, 2 * sizeof(double));
  if (e == cudaSuccess) {
    launch(d);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(out, d, 2 * sizeof(double), cudaMemcpyDeviceToHost);
  if (d) cudaFree(d);
  if (prev >= 0) cudaSetDevice(prev);
  if (e != cudaSuccess)
    return set_error(MCML_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  out[0] /= (double)n;
  out[1] /= (double)n;
  return MCML_OK;
}

constexpr int kProbeGrid = 592, kProbeBlock = 256;

}  // namespace

extern "C" int mcml_probe_spin(int device, float g, uint64_t n, uint64_t seed, double *out) {
  clear_error();
  if (!out || n == 0 || !(g > -1.0f && g < 1.0f)) return set_error(MCML_E_INVALID, "bad argument");
  return run_probe(device, n, out, "spin probe", [&](double *d) {
    spin_probe_kernel<<<kProbeGrid, kProbeBlock>>>(g, n, seed, d);
  });
}

extern "C" int mcml_probe_reflect(int device, float n1, float n2, float cos_i, uint64_t n,
                                  uint64_t seed, double *out) {
  clear_error();
  if (!out || n == 0 || !(n1 >= 1.0f) || !(n2 >= 1.0f) || !(cos_i > 0.0f && cos_i <= 1.0f))
    return set_error(MCML_E_INVALID, "bad argument");
  return run_probe(device, n, out, "reflect probe", [&](double *d) {
    reflect_probe_kernel<<<kProbeGrid, kProbeBlock>>>(n1, n2, cos_i, n, seed, d);
  });
}
