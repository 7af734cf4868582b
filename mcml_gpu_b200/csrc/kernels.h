// kernels.h -- host-visible declarations of the device kernels' launchers.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "photon.cuh"

namespace mcml {

// Slots of the per-context counter block (unsigned long long each).
enum : int {
  kCntSlot = 0,     // next slot to hand out (walk)
  kCntRecords = 1,  // detection records appended (may exceed capacity)
  kCntSteps = 2,    // walk steps
  kCntReplay = 3,   // next record to replay
  kCntStatus = 4,   // kernel status bits (int in the low word)
  kCntWords = 8
};

enum : int { kStatusBudget = 1 };

constexpr int kReplayBlock = 128;

struct WalkArgs {
  const uint2 *slot_state;       // num_slots x 3 uint2: (d,v0) (v1,v2) (v3,v4)
  unsigned long long *counters;  // kCntWords
  DetRecord *records;
  unsigned long long rec_cap;
  unsigned long long slot_end;   // lanes stop taking slots here (<= num_slots)
};

struct ReplayArgs {
  const DetRecord *records;
  const unsigned long long *rec_count;
  unsigned long long rec_cap;
  unsigned long long *cursor;
  float *rows;              // rec_cap x (L+2)
  uint32_t *interactions;   // rec_cap x L, may be null
  unsigned long long *A_rz; // S x nz x nr
  unsigned long long *A0_z; // S x nz
  unsigned long long budget;
  int *status;
};

cudaError_t launch_seed_slots(uint64_t seed, uint64_t slot_begin, uint64_t num_slots, uint2 *out,
                              int sm_count, cudaStream_t stream);
cudaError_t launch_walk(const DevParams &P, const WalkArgs &A, bool src_obl, bool det_obl,
                        int block, int min_blocks, int grid, cudaStream_t stream);
// The walk kernel of a launch shape; glass: some tissue layer has
// mutr == FLT_MAX (has_glass_layer), which needs the conditional draw.
const void *walk_kernel_ptr(int block, int min_blocks, bool src_obl, bool det_obl, bool glass);
bool has_glass_layer(const DevParams &P);
cudaError_t launch_replay(const DevParams &P, const ReplayArgs &A, bool src_obl, bool det_obl,
                          bool ref_grid, int grid, cudaStream_t stream);
// The first D records -- and, when rows is not null, their replay rows
// (L + 2 floats) and interaction counts (L words) -- ordered by SDS, then
// photon index, in caller-provided device scratch of at least
// order_scratch_bytes(D, L, rows != nullptr) bytes (order.cu).  The
// ordered arrays are placed in the scratch; *out points at them.
struct OrderedOutput {
  DetRecord *records = nullptr;
  float *rows = nullptr;
  uint32_t *interactions = nullptr;
};
size_t order_scratch_bytes(uint64_t D, int L, bool rows);
cudaError_t sort_records_for_output(const DetRecord *rec, uint64_t D, const float *rows,
                                    const uint32_t *inter, int L, void *scratch,
                                    size_t scratch_bytes, OrderedOutput *out, int sm_count,
                                    cudaStream_t stream);
cudaError_t launch_reduce_records(const DetRecord *rec, const unsigned long long *rec_count,
                                  unsigned long long rec_cap, unsigned n_sds,
                                  unsigned long long *det_count, double *wsum, double *wsq,
                                  int sm_count, cudaStream_t stream);
cudaError_t launch_uniform_stream(uint64_t seed, uint64_t subsequence, uint64_t count, float *out,
                                  cudaStream_t stream);

}  // namespace mcml
