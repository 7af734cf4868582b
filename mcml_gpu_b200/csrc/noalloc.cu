// noalloc.cu -- a first pass that allocates no device memory.
//
// Some callers cannot call cudaMalloc at the moment they want photons
// walked: a real-time pipeline whose device memory is fixed at start-up and
// must not block in the allocator (cudaMalloc can synchronise the device)
// mid-run, or a process whose GPU memory is already reserved by another
// framework's memory pool, so that an allocation of its own would fail or
// steal from that pool.  mcml_run_noalloc serves them: the walk's scratch
// memory (slot cursor, per-SDS accumulators and the XORWOW slot states)
// lives in the fixed array below, compiled into the library, and the caller
// passes its inputs by value and a device buffer for the outputs.  Nothing
// here calls cudaMalloc, cudaFree or any allocating routine.
//
// The array is MCML_NOALLOC_SCRATCH_BYTES (8 MiB) on every GPU that loads
// the library, held until the process exits; it fits the reference's
// one-photon-per-thread layout on a B200 (303104 slots).  All calls share
// it and it keeps the last call's contents: each call clears the part that
// must start at zero, and calls that overlap on the GPU (two streams, two
// host threads) race on it -- serialise them.
//
// The walk is the same step function (walk_step, photon.cuh) as the
// allocating first pass; only where a detection goes differs (summed per
// SDS here, appended as a record there).
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include <cuda.h>  // CUcontext / CUresult types; the functions are looked up at run time

#include "../../include/mcml_b200.h"
#include "internal.h"
#include "kernels.h"
#include "params.h"
#include "photon.cuh"

namespace mcml {
namespace {

constexpr size_t kScratchBytes = MCML_NOALLOC_SCRATCH_BYTES;
constexpr size_t kHeaderBytes = 1024;  // cursor, steps, per-SDS accumulators
constexpr uint64_t kMaxSlots = (kScratchBytes - kHeaderBytes) / 24;

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

struct Header {
  unsigned long long cursor;
  unsigned long long steps;
  unsigned long long detected[kMaxSds + 2];
  double wsum[kMaxSds + 2];
  double wsq[kMaxSds + 2];
};
static_assert(sizeof(Header) <= kHeaderBytes, "scratch header");

// Clears the header and seeds the slot states (one slot per thread).
__global__ void noalloc_seed_kernel(unsigned char *scratch, uint64_t seed, uint64_t num_slots) {
  Header *h = reinterpret_cast<Header *>(scratch);
  uint2 *states = reinterpret_cast<uint2 *>(scratch + kHeaderBytes);
  const uint64_t s = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s == 0) {
    h->cursor = 0;
    h->steps = 0;
    for (int i = 0; i < kMaxSds + 2; ++i) {
      h->detected[i] = 0;
      h->wsum[i] = 0.0;
      h->wsq[i] = 0.0;
    }
  }
  if (s >= num_slots) return;
  curandStateXORWOW st;
  curand_init(seed, s, 0, &st);
  states[s * 3 + 0] = make_uint2(st.d, st.v[0]);
  states[s * 3 + 1] = make_uint2(st.v[1], st.v[2]);
  states[s * 3 + 2] = make_uint2(st.v[3], st.v[4]);
}

__device__ __forceinline__ void tally(Header *h, int sds, float w) {
  atomicAdd(&h->detected[sds], 1ull);
  atomicAdd(&h->wsum[sds], (double)w);
  atomicAdd(&h->wsq[sds], (double)w * (double)w);
}

// The first pass (walk_step) with detections summed per SDS in place of
// appended records.
template <bool kSrcOblique, bool kDetOblique, bool kGlass>
__global__ void __launch_bounds__(128) noalloc_walk_kernel(const __grid_constant__ DevParams P,
                                                           unsigned char *scratch) {
  __shared__ SmemTables t;
  load_tables(t, P);
  __syncthreads();
  Header *h = reinterpret_cast<Header *>(scratch);
  const uint2 *states = reinterpret_cast<const uint2 *>(scratch + kHeaderBytes);
  const uint64_t S = P.num_slots;
  const uint64_t q = P.num_photons / S;
  const uint64_t rem = P.num_photons % S;
  const int n_layers = (int)P.n_layers;
  const int n_sds = (int)P.n_sds;
  curandStateXORWOW st;
  st.boxmuller_flag = 0;
  st.boxmuller_flag_double = 0;
  st.boxmuller_extra = 0.0f;
  st.boxmuller_extra_double = 0.0;
  Photon p;
  uint32_t k = 0, quota = 0, steps_acc = 0;

  auto next_slot = [&]() -> bool {
    const uint64_t s = atomicAdd(&h->cursor, 1ull);
    if (s >= S) return false;
    const uint2 a = states[s * 3 + 0], b = states[s * 3 + 1], c = states[s * 3 + 2];
    st.d = a.x;
    st.v[0] = a.y;
    st.v[1] = b.x;
    st.v[2] = b.y;
    st.v[3] = c.x;
    st.v[4] = c.y;
    k = 0;
    quota = (uint32_t)(q + (s < rem ? 1 : 0));
    return true;
  };

  if (!next_slot()) return;
  launch_photon<kSrcOblique>(p, &st, t, P.start_weight);
  for (;;) {
    const bool alive = walk_step<kDetOblique, kGlass>(p, st, t, n_layers, n_sds, P.det_reflectance,
                                              [&](int i, float w) { tally(h, i, w); });
    if (!alive) {
      steps_acc += (uint32_t)p.steps;
      if (++k >= quota || steps_acc >= 0x40000000u) {
        atomicAdd(&h->steps, (unsigned long long)steps_acc);
        steps_acc = 0;
      }
      if (k >= quota && !next_slot()) break;
      launch_photon<kSrcOblique>(p, &st, t, P.start_weight);
    }
  }
}

// Copies the accumulators to the caller's buffer (mcml_noalloc_result).
__global__ void noalloc_finish_kernel(const unsigned char *scratch, unsigned n_sds,
                                      mcml_noalloc_result *out) {
  const Header *h = reinterpret_cast<const Header *>(scratch);
  const unsigned i = threadIdx.x;
  if (i < MCML_MAX_SDS) {
    const bool on = i < n_sds;
    out->detected[i] = on ? h->detected[i + 1] : 0ull;
    out->weight_sum[i] = on ? h->wsum[i + 1] : 0.0;
    out->weight_sumsq[i] = on ? h->wsq[i + 1] : 0.0;
  }
  if (i == 0) out->steps = h->steps;
}

// Per-device set-up: the device address of g_scratch (its host-side name is
// only a stand-in: a kernel given it would fault or, where the GPU can reach
// host memory, silently use the wrong memory) and the walk's launch shape.
// It runs on the first call on a device, and again on the first call after
// that device's context was replaced (cudaDeviceReset ends a context; the
// next one loads the library's module anew, possibly at another address).
struct DeviceSetup {
  bool done = false;
  unsigned long long ctx_id = 0;  // context the address belongs to (0: unknown)
  unsigned char *scratch = nullptr;
  int grid[8] = {0, 0, 0, 0, 0, 0, 0, 0};
};
constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
DeviceSetup g_setup[kMaxDevices];

// Unique id of the calling thread's current CUDA context (cuCtxGetId ids
// are never reused within a process), or 0 when there is none yet or the
// driver lacks the call.  The driver functions are looked up through the
// runtime, so the library does not link libcuda directly.
unsigned long long current_context_id() {
  using GetCurrent = CUresult (*)(CUcontext *);
  using GetId = CUresult (*)(CUcontext, unsigned long long *);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  static bool looked_up = false;
  if (!looked_up) {
    cudaDriverEntryPointQueryResult q1, q2;
    void *f1 = nullptr, *f2 = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1) == cudaSuccess &&
        q1 == cudaDriverEntryPointSuccess &&
        cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2) == cudaSuccess &&
        q2 == cudaDriverEntryPointSuccess) {
      get_current = reinterpret_cast<GetCurrent>(f1);
      get_id = reinterpret_cast<GetId>(f2);
    }
    cudaGetLastError();
    looked_up = true;
  }
  if (!get_current || !get_id) return 0;
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (get_current(&ctx) != CUDA_SUCCESS || ctx == nullptr) return 0;
  if (get_id(ctx, &id) != CUDA_SUCCESS) return 0;
  return id;
}

// variant: glass*4 + src_oblique*2 + det_oblique
const void *walk_fn(int variant) {
  switch (variant) {
    case 0: return (const void *)noalloc_walk_kernel<false, false, false>;
    case 1: return (const void *)noalloc_walk_kernel<false, true, false>;
    case 2: return (const void *)noalloc_walk_kernel<true, false, false>;
    case 3: return (const void *)noalloc_walk_kernel<true, true, false>;
    case 4: return (const void *)noalloc_walk_kernel<false, false, true>;
    case 5: return (const void *)noalloc_walk_kernel<false, true, true>;
    case 6: return (const void *)noalloc_walk_kernel<true, false, true>;
    default: return (const void *)noalloc_walk_kernel<true, true, true>;
  }
}

// Called with `device` current.
int setup_device(int device, DeviceSetup **out) {
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  DeviceSetup &d = g_setup[device];
  const unsigned long long ctx = current_context_id();
  if (!d.done || (ctx != 0 && ctx != d.ctx_id)) {
    d.done = false;
    void *ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_scratch);
    if (e != cudaSuccess)
      return set_error(MCML_E_CUDA, std::string("cudaGetSymbolAddress(scratch): ") +
                                        cudaGetErrorString(e));
    int sms = 0;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess)
      return set_error(MCML_E_CUDA, std::string("cudaDeviceGetAttribute: ") + cudaGetErrorString(e));
    for (int v = 0; v < 8; ++v) {
      int nb = 0;
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, walk_fn(v), 128, 0);
      if (e != cudaSuccess)
        return set_error(MCML_E_CUDA, std::string("occupancy: ") + cudaGetErrorString(e));
      d.grid[v] = (nb < 1 ? 1 : nb) * sms;
    }
    d.scratch = static_cast<unsigned char *>(ptr);
    // the symbol lookup created the context if there was none yet
    d.ctx_id = ctx != 0 ? ctx : current_context_id();
    d.done = true;
  }
  *out = &d;
  return MCML_OK;
}

}  // namespace
}  // namespace mcml

extern "C" int mcml_run_noalloc(const mcml_sim *sim, uint64_t seed, uint64_t slots, int device,
                                void *stream, mcml_noalloc_result *out) {
  using namespace mcml;
  clear_error();
  if (!out) return set_error(MCML_E_INVALID, "mcml_run_noalloc: null output buffer");
  int rc = validate_sim(sim);
  if (rc) return rc;
  mcml_derived der;
  rc = derive(sim, &der);
  if (rc) return rc;
  const uint64_t N = sim->number_photons;
  uint64_t S = slots ? slots : (N < kMaxSlots ? N : kMaxSlots);
  if (S > kMaxSlots)
    return set_error(MCML_E_INVALID,
                     "mcml_run_noalloc: " + std::to_string(S) + " slots exceed the fixed scratch "
                     "capacity of " + std::to_string(kMaxSlots) + " slots (" +
                     std::to_string(kScratchBytes) + " bytes)");
  if (S > N) S = N;
  if (N / S >= 0xFFFFFFFFull)
    return set_error(MCML_E_INVALID, "mcml_run_noalloc: too many photons per slot");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return set_error(MCML_E_NODEV, "no CUDA device");
  }
  if (device < 0 || device >= ndev || device >= kMaxDevices)
    return set_error(MCML_E_INVALID, "GPU selection ERROR!");
  int prev = -1;
  cudaGetDevice(&prev);
  if (prev != device && cudaSetDevice(device) != cudaSuccess)
    return set_error(MCML_E_CUDA, "cudaSetDevice failed");
  DeviceSetup *d = nullptr;
  rc = setup_device(device, &d);
  if (rc == MCML_OK) {
    DevParams P;
    fill_dev_params(*sim, der, N, S, P);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int variant = (has_glass_layer(P) ? 4 : 0) + (sim->source_probe_oblique ? 2 : 0) +
                        (sim->detector_probe_oblique ? 1 : 0);
    noalloc_seed_kernel<<<(unsigned)((S + 255) / 256), 256, 0, s>>>(d->scratch, seed, S);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) {
      void *args[] = {(void *)&P, (void *)&d->scratch};
      e = cudaLaunchKernel(walk_fn(variant), dim3(d->grid[variant]), dim3(128), args, 0, s);
    }
    if (e == cudaSuccess) {
      noalloc_finish_kernel<<<1, 32, 0, s>>>(d->scratch, sim->num_sds, out);
      e = cudaGetLastError();
    }
    if (e != cudaSuccess)
      rc = set_error(MCML_E_CUDA, std::string("mcml_run_noalloc launch: ") + cudaGetErrorString(e));
  }
  if (prev >= 0 && prev != device) cudaSetDevice(prev);
  return rc;
}
