// noalloc.cu -- a first pass that allocates no device memory.
//
// Some callers cannot call cudaMalloc at the moment they want photons
// walked: code that is recording a CUDA graph (an allocation is not allowed
// while a stream is being captured, and it would synchronise the device), a
// real-time pipeline whose device memory is fixed at start-up and must not
// block in the allocator mid-run, or a process whose GPU memory is already
// reserved by another framework's memory pool.  mcml_run_noalloc serves
// them: the walk's scratch memory (slot cursor, per-SDS accumulators and
// the XORWOW slot states) lives in the fixed array below, compiled into the
// library, and the caller passes its inputs by value and a device buffer
// for the outputs.  Nothing here calls cudaMalloc, cudaFree or any
// allocating routine.
//
// The array is MCML_NOALLOC_SCRATCH_BYTES (8 MiB) on every GPU that loads
// the library, held until the process exits; it fits the reference's
// one-photon-per-thread layout on a B200 (303104 slots).  All calls share
// it and it keeps the last call's contents: each call clears the part that
// must start at zero, and calls that overlap on the GPU (two streams, two
// host threads) race on it -- serialise them.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/mcml_b200.h"
#include "internal.h"
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

// The first pass of kernels.cu's walk_kernel with detections summed per
// SDS in place of appended records.
template <bool kSrcOblique, bool kDetOblique>
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
    float s;
    const int new_layer = hop(p, s, &st, t);
    p.steps++;
    clamp_z(p, t, p.layer);
    if (new_layer != p.layer) {
      const int temp_layer = p.layer;
      s = 0.0f;
      if (!reflect(p, new_layer, &st, t)) {
        if (new_layer == 0) {
          bool detected = false;
          if (kDetOblique) {
            unsigned mask = fiber_mask(p, t, n_sds);
            detected = mask != 0u;
            while (mask) {
              const int i = __ffs(mask) - 1;
              mask &= mask - 1u;
              tally(h, i, p.w);
            }
          } else {
            const float uz_angle = acosf(fabsf(p.dz));
            const float distance = radius_xy(p);
            for (int i = 1; i <= n_sds; i++) {
              float wd;
              if (ring_hit(p, t, i, uz_angle, distance, wd)) {
                tally(h, i, wd);
                detected = true;
              }
            }
          }
          if (detected) {
            p.w = 0;
          } else if (uni(&st) > P.det_reflectance) {
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
      drop_weight_walk(p, L.w);
      spin(p, t.hg[p.layer], &st);
    }
    if (!survive<true>(p, &st)) {
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
// only a stand-in) and the walk's launch shape.
struct DeviceSetup {
  bool done = false;
  unsigned char *scratch = nullptr;
  int grid[4] = {0, 0, 0, 0};
};
constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
DeviceSetup g_setup[kMaxDevices];

const void *walk_fn(int variant) {
  switch (variant) {
    case 0: return (const void *)noalloc_walk_kernel<false, false>;
    case 1: return (const void *)noalloc_walk_kernel<false, true>;
    case 2: return (const void *)noalloc_walk_kernel<true, false>;
    default: return (const void *)noalloc_walk_kernel<true, true>;
  }
}

int setup_device(int device, DeviceSetup **out) {
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  DeviceSetup &d = g_setup[device];
  if (!d.done) {
    void *ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_scratch);
    if (e != cudaSuccess)
      return set_error(MCML_E_CUDA, std::string("cudaGetSymbolAddress(scratch): ") +
                                        cudaGetErrorString(e));
    int sms = 0;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess)
      return set_error(MCML_E_CUDA, std::string("cudaDeviceGetAttribute: ") + cudaGetErrorString(e));
    for (int v = 0; v < 4; ++v) {
      int nb = 0;
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, walk_fn(v), 128, 0);
      if (e != cudaSuccess)
        return set_error(MCML_E_CUDA, std::string("occupancy: ") + cudaGetErrorString(e));
      d.grid[v] = (nb < 1 ? 1 : nb) * sms;
    }
    d.scratch = static_cast<unsigned char *>(ptr);
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
    std::memset(&P, 0, sizeof(P));
    const int L = (int)sim->num_layers;
    for (int l = 0; l <= L + 1; ++l) {
      P.z_min[l] = der.z_min[l];
      P.z_max[l] = der.z_max[l];
      P.mutr[l] = der.mutr[l];
      if (l >= 1 && l <= L) {
        P.mua[l] = sim->mua[l - 1];
        P.g[l] = sim->g[l - 1];
        P.n[l] = sim->n[l - 1];
      }
    }
    P.n[0] = sim->upper_n;
    P.n[L + 1] = sim->lower_n;
    P.det_radius[0] = sim->source_radius;
    P.det_NA[0] = sim->source_NA;
    P.det_angle[0] = der.det_angle_rad[0];
    for (unsigned i = 0; i < sim->num_sds; ++i) {
      P.det_radius[i + 1] = sim->det_radius[i];
      P.det_NA[i + 1] = sim->det_NA[i];
      P.det_pos[i + 1] = sim->det_pos[i];
      P.det_angle[i + 1] = der.det_angle_rad[i + 1];
      P.crit[i + 1] = der.critical_angle[i + 1];
    }
    P.n_layers = sim->num_layers;
    P.n_sds = sim->num_sds;
    P.start_weight = der.start_weight;
    P.det_reflectance = sim->detector_reflectance;
    P.num_photons = N;
    P.num_slots = S;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int variant = (sim->source_probe_oblique ? 2 : 0) + (sim->detector_probe_oblique ? 1 : 0);
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
