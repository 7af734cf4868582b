// order.cu -- detection records, replay rows and interaction counts put in
// file order on the device before they are copied to the host.
//
// The reference's host collects detections thread by thread and writes
// each SDS's rows in that order (transport.cu:301-325); with a fixed
// photon-to-slot mapping the deterministic equivalent is photon order.
// Records arrive in atomic-append order, so the host would otherwise sort
// D indices with an indirect comparison; here one radix sort of the
// 49-bit keys (sds << 44 | photon) and one gather do it on the GPU.
#include <cub/device/device_radix_sort.cuh>
#include <cuda_runtime.h>

#include "kernels.h"

namespace mcml {
namespace {

constexpr int kPhotonBits = 44;

__global__ void record_keys_kernel(const DetRecord *rec, uint64_t D, uint64_t *keys,
                                   uint32_t *idx) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < D;
       i += (uint64_t)gridDim.x * blockDim.x) {
    keys[i] = ((uint64_t)rec[i].sds << kPhotonBits) | rec[i].photon;
    idx[i] = (uint32_t)i;
  }
}

// One thread per output position: record j of the sorted order and its
// row (L + 2 floats) and counts (L words).
__global__ void gather_kernel(const uint32_t *perm, uint64_t D, const DetRecord *rec,
                              DetRecord *rec_out, const float *rows, float *rows_out,
                              const uint32_t *inter, uint32_t *inter_out, int L) {
  for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < D;
       j += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t i = perm[j];
    rec_out[j] = rec[i];
    if (rows) {
      const int rl = L + 2;
      for (int k = 0; k < rl; ++k) rows_out[j * rl + k] = rows[i * rl + k];
      for (int k = 0; k < L; ++k) inter_out[j * L + k] = inter[i * L + k];
    }
  }
}

}  // namespace

cudaError_t sort_records_for_output(const DetRecord *rec, uint64_t D, const float *rows,
                                    const uint32_t *inter, int L, DetRecord *rec_out,
                                    float *rows_out, uint32_t *inter_out, int sm_count,
                                    cudaStream_t stream) {
  if (D == 0) return cudaSuccess;
  if (D >= (1ull << 31)) return cudaErrorInvalidValue;
  uint64_t *keys = nullptr;
  uint32_t *idx = nullptr;
  void *temp = nullptr;
  size_t temp_bytes = 0;
  cudaError_t e = cub::DeviceRadixSort::SortPairs(nullptr, temp_bytes, keys, keys, idx, idx,
                                                  (int)D, 0, kPhotonBits + 5, stream);
  if (e == cudaSuccess) e = cudaMallocAsync(&keys, 2 * D * sizeof(uint64_t), stream);
  if (e == cudaSuccess) e = cudaMallocAsync(&idx, 2 * D * sizeof(uint32_t), stream);
  if (e == cudaSuccess) e = cudaMallocAsync(&temp, temp_bytes, stream);
  if (e == cudaSuccess) {
    const int grid = 4 * sm_count;
    record_keys_kernel<<<grid, 256, 0, stream>>>(rec, D, keys, idx);
    e = cudaGetLastError();
    if (e == cudaSuccess)
      e = cub::DeviceRadixSort::SortPairs(temp, temp_bytes, keys, keys + D, idx, idx + D, (int)D,
                                          0, kPhotonBits + 5, stream);
    if (e == cudaSuccess) {
      gather_kernel<<<grid, 256, 0, stream>>>(idx + D, D, rec, rec_out, rows, rows_out, inter,
                                              inter_out, L);
      e = cudaGetLastError();
    }
  }
  if (temp) cudaFreeAsync(temp, stream);
  if (idx) cudaFreeAsync(idx, stream);
  if (keys) cudaFreeAsync(keys, stream);
  return e;
}

}  // namespace mcml
