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

size_t align256(size_t n) { return (n + 255) & ~size_t(255); }

size_t cub_temp_bytes(uint64_t D) {
  size_t bytes = 0;
  uint64_t *k = nullptr;
  uint32_t *v = nullptr;
  cub::DeviceRadixSort::SortPairs(nullptr, bytes, k, k, v, v, (int)D, 0, kPhotonBits + 5);
  return bytes;
}

}  // namespace

size_t order_scratch_bytes(uint64_t D, int L, bool rows) {
  if (D == 0) return 0;
  size_t b = align256(2 * D * sizeof(uint64_t)) + align256(2 * D * sizeof(uint32_t)) +
             align256(cub_temp_bytes(D)) + align256(D * sizeof(DetRecord));
  if (rows) b += align256(D * (L + 2) * sizeof(float)) + align256(D * L * sizeof(uint32_t));
  return b;
}

cudaError_t sort_records_for_output(const DetRecord *rec, uint64_t D, const float *rows,
                                    const uint32_t *inter, int L, void *scratch,
                                    size_t scratch_bytes, OrderedOutput *out, int sm_count,
                                    cudaStream_t stream) {
  *out = OrderedOutput{};
  if (D == 0) return cudaSuccess;
  if (D >= (1ull << 31)) return cudaErrorInvalidValue;
  if (scratch_bytes < order_scratch_bytes(D, L, rows != nullptr)) return cudaErrorInvalidValue;
  char *p = static_cast<char *>(scratch);
  auto take = [&](size_t n) {
    char *q = p;
    p += align256(n);
    return q;
  };
  uint64_t *keys = reinterpret_cast<uint64_t *>(take(2 * D * sizeof(uint64_t)));
  uint32_t *idx = reinterpret_cast<uint32_t *>(take(2 * D * sizeof(uint32_t)));
  size_t temp_bytes = cub_temp_bytes(D);
  void *temp = take(temp_bytes);
  out->records = reinterpret_cast<DetRecord *>(take(D * sizeof(DetRecord)));
  if (rows) {
    out->rows = reinterpret_cast<float *>(take(D * (L + 2) * sizeof(float)));
    out->interactions = reinterpret_cast<uint32_t *>(take(D * L * sizeof(uint32_t)));
  }
  const int grid = 4 * sm_count;
  record_keys_kernel<<<grid, 256, 0, stream>>>(rec, D, keys, idx);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cub::DeviceRadixSort::SortPairs(temp, temp_bytes, keys, keys + D, idx, idx + D, (int)D, 0,
                                        kPhotonBits + 5, stream);
  if (e == cudaSuccess) {
    gather_kernel<<<grid, 256, 0, stream>>>(idx + D, D, rec, out->records, rows, out->rows, inter,
                                            out->interactions, L);
    e = cudaGetLastError();
  }
  return e;
}

}  // namespace mcml
