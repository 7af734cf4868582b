// mcml_oracle.cpp -- CPU restatement of the reference MCML walk.
//
// TEST INFRASTRUCTURE ONLY.  This file is the correctness oracle and the
// timed CPU baseline; the library never links, loads or calls it.
//
// It restates, in plain C++, the per-photon algorithm of the reference
// (MCML_GPU K3.02): launch (transport.cu:624-719), hop / boundary / move
// (transport.cu:372-395), Fresnel reflect/refract (transport.cu:790-853),
// detection on exit (transport.cu:403-427, 872-1000), weight drop
// (transport.cu:430-437), Henyey-Greenstein spin (transport.cu:742-786),
// roulette (transport.cu:855-870), the replay tallies
// (transport.cu:506-613) and the derived constants (io.cpp:168-238).
//
// Two precisions: float (the reference's types, libm functions standing in
// for the GPU's __logf/__fdividef/__sincosf/rsqrtf) and double (the FP64
// statistical oracle).  Two random sources:
//   * a recorded stream of uniforms -- the exact draws curand_uniform
//     produces for one XORWOW subsequence, generated on the GPU -- so that
//     one photon can be walked with the reference's own random numbers;
//   * PCG32 (M. E. O'Neill, "PCG: A Family of Simple Fast Space-Efficient
//     Statistically Good Algorithms for Random Number Generation", 2014),
//     one stream per photon, for statistical runs and the CPU baseline.
// OpenMP parallelises statistical runs over photons.
#include <algorithm>
#include <cfenv>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/mcml_b200.h"

namespace {

constexpr double kPId = 3.141592654;  // PI of header.h:40, as the float 3.141592654f
constexpr float kPIf = 3.141592654f;
constexpr float kRPIf = 0.318309886f;  // header.h:41
constexpr unsigned kWEIGHTI = 429497u; // header.h:57
constexpr int kMaxScatter = 10000;     // header.h:62

// ---- random sources --------------------------------------------------------
struct StreamRng {
  const float *u;
  uint64_t n;
  uint64_t i = 0;
  bool exhausted = false;
  double next() {
    if (i < n) return (double)u[i++];
    exhausted = true;
    return 0.5;
  }
};

struct Pcg32 {
  uint64_t state = 0, inc = 1;
  uint32_t step() {
    const uint64_t old = state;
    state = old * 6364136223846793005ULL + inc;
    const uint32_t xorshifted = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    const uint32_t rot = (uint32_t)(old >> 59u);
    return (xorshifted >> rot) | (xorshifted << ((32u - rot) & 31u));
  }
  void seed(uint64_t initstate, uint64_t initseq) {
    state = 0u;
    inc = (initseq << 1u) | 1u;
    step();
    state += initstate;
    step();
  }
  // Uniform in (0, 1] with 24-bit resolution.
  double next() { return (double)((step() >> 8) + 1u) * (1.0 / 16777216.0); }
  bool exhausted = false;
};

// ---- precision policy ------------------------------------------------------
template <typename R>
struct Tab {
  R z_min[MCML_MAX_LAYERS + 2], z_max[MCML_MAX_LAYERS + 2], mutr[MCML_MAX_LAYERS + 2];
  R mua[MCML_MAX_LAYERS + 2], g[MCML_MAX_LAYERS + 2], n[MCML_MAX_LAYERS + 2];
  R det_pos[MCML_MAX_SDS + 1], det_r[MCML_MAX_SDS + 1], det_crit[MCML_MAX_SDS + 1];
  R det_cos[MCML_MAX_SDS + 1], det_sin[MCML_MAX_SDS + 1];
  R src_sin, src_cos, src_theta, src_radius, src_NA;
  R start_weight, det_refl;
  int n_layers, n_sds;
  bool src_obl, det_obl;
};

uint32_t sat_u32(double x) {  // float->unsigned conversion of the GPU: saturating
  if (!(x > 0.0)) return 0u;
  if (x >= 4294967295.0) return 0xFFFFFFFFu;
  return (uint32_t)x;
}
uint32_t rn_u32(double x) {  // __float2uint_rn: nearest-even, saturating
  return sat_u32(std::nearbyint(x));
}

// Derived constants, io.cpp:168-238, in float as the reference stores them.
void derive_float(const mcml_sim &s, mcml_derived &d) {
  std::memset(&d, 0, sizeof(d));
  const int L = (int)s.num_layers;
  d.det_angle_rad[0] = s.source_angle_deg * kPIf / 180;
  for (unsigned i = 0; i < s.num_sds; ++i) {
    d.det_angle_rad[i + 1] = s.det_angle_deg[i] * kPIf / 180;
    d.critical_angle[i + 1] = std::asin(s.det_NA[i] / s.upper_n);
  }
  float zmin = 0, zmax = 0;
  for (int l = 1; l <= L; ++l) {
    const float h = l < L ? s.height[l - 1] : 0.0f;
    zmax += h;
    d.z_min[l] = zmin;
    d.z_max[l] = zmax;
    d.mutr[l] = 1.0f / (s.mua[l - 1] + s.mus[l - 1]);
    zmin += h;
  }
  if (d.z_max[L] < 10.0f) d.z_max[L] = 10.0f;
  const double n1 = s.upper_n, n2 = s.n[0];
  double r = (n1 - n2) / (n1 + n2);
  r = r * r;
  d.start_weight = (unsigned int)((double)0xffffffff * (1 - r));
}

template <typename R>
void make_tab(const mcml_sim &s, Tab<R> &t) {
  mcml_derived d;
  derive_float(s, d);
  std::memset(&t, 0, sizeof(t));
  const int L = (int)s.num_layers;
  t.n_layers = L;
  t.n_sds = (int)s.num_sds;
  for (int l = 1; l <= L; ++l) {
    t.z_min[l] = d.z_min[l];
    t.z_max[l] = d.z_max[l];
    t.mua[l] = s.mua[l - 1];
    t.g[l] = s.g[l - 1];
    t.n[l] = s.n[l - 1];
    if (sizeof(R) == sizeof(float))
      t.mutr[l] = d.mutr[l];
    else
      t.mutr[l] = (R)(1.0 / ((double)s.mua[l - 1] + (double)s.mus[l - 1]));
  }
  t.n[0] = s.upper_n;
  t.n[L + 1] = s.lower_n;
  for (int i = 1; i <= t.n_sds; ++i) {
    const R a = (R)d.det_angle_rad[i];
    t.det_pos[i] = s.det_pos[i - 1];
    t.det_r[i] = s.det_radius[i - 1];
    t.det_crit[i] = d.critical_angle[i];
    t.det_cos[i] = std::cos(a);
    t.det_sin[i] = std::sin(a);
  }
  t.src_sin = std::sin((R)d.det_angle_rad[0]);
  t.src_cos = std::cos((R)d.det_angle_rad[0]);
  t.src_theta = std::asin((R)s.source_NA / (R)s.upper_n);
  t.src_radius = s.source_radius;
  t.src_NA = s.source_NA;
  t.start_weight = d.start_weight;
  t.det_refl = s.detector_reflectance;
  t.src_obl = s.source_probe_oblique != 0;
  t.det_obl = s.detector_probe_oblique != 0;
}

template <typename R>
struct Ph {
  R x, y, z, dx, dy, dz, w;
  int layer, steps;
};

template <typename R, typename Rng>
R uni(Rng &g) {
  return (R)g.next();
}

// transport.cu:624-719
template <typename R, typename Rng>
void launch(Ph<R> &p, Rng &g, const Tab<R> &t) {
  const R PI = (R)kPId;
  if (t.src_obl) {
    p.x = p.y = p.z = 0;
    p.dx = t.src_sin;
    p.dy = 0;
    p.dz = t.src_cos;
  } else {
    if (t.src_radius == 0) {
      p.x = p.y = p.z = 0;
    } else {
      const R rp = uni<R>(g), ra = uni<R>(g);
      const R lr = t.src_radius * rp;
      const R az = 2 * PI * ra;
      p.x = lr * std::sin(az);
      p.y = lr * std::cos(az);
      p.z = 0;
    }
    if (t.src_NA == 0) {
      p.dx = 0;
      p.dy = 0;
      p.dz = 1;
    } else {
      const R rd = uni<R>(g), rr = uni<R>(g);
      const R th = t.src_theta * rd;
      const R rot = 2 * PI * rr;
      p.dz = std::cos(th);
      p.dx = std::sin(th) * std::cos(rot);
      p.dy = std::sin(th) * std::sin(rot);
    }
  }
  p.layer = 1;
  p.steps = 0;
  p.w = t.start_weight;
}

// transport.cu:790-853; true = reflected.
template <typename R, typename Rng>
bool reflect(Ph<R> &p, int new_layer, Rng &g, const Tab<R> &t) {
  const R n1 = t.n[p.layer], n2 = t.n[new_layer];
  const R c = std::fabs(p.dz);
  if (n1 == n2) {
    p.layer = new_layer;
    return false;
  }
  if (n1 > n2 && n2 * n2 < n1 * n1 * (1 - c * c)) {
    p.dz = -p.dz;
    return true;
  }
  R r;
  if (c == 1) {
    r = (n1 - n2) / (n1 + n2);
    if (uni<R>(g) <= r * r) {
      p.dz = -p.dz;
      return true;
    }
    p.layer = new_layer;
    return false;
  }
  R e = (n1 * n1) / (n2 * n2) * (1 - c * c);
  r = 2 * std::sqrt((1 - c * c) * (1 - e) * e * c * c);
  e = e + (c * c) * (1 - 2 * e);
  r = e * ((1 - e - r) / ((1 - e + r) * (e + r)));
  if (uni<R>(g) <= r) {
    p.dz = -p.dz;
    return true;
  }
  r = n1 / n2;
  e = r * r * (1 - c * c);
  p.dx *= r;
  p.dy *= r;
  p.dz = std::copysign(std::sqrt(1 - e), p.dz);
  p.layer = new_layer;
  return false;
}

// transport.cu:742-786
template <typename R, typename Rng>
void spin(Ph<R> &p, R g, Rng &rng) {
  const R PI = (R)kPId;
  R cost, temp;
  if (g == 0) {
    cost = 2 * uni<R>(rng) - 1;
  } else {
    temp = (1 - g * g) / (1 - g + 2 * g * uni<R>(rng));
    cost = (1 + g * g - temp * temp) / (2 * g);
  }
  const R sint = std::sqrt(1 - cost * cost);
  const R psi = 2 * PI * uni<R>(rng);
  const R sinp = std::sin(psi), cosp = std::cos(psi);
  temp = std::sqrt(1 - p.dz * p.dz);
  if (temp == 0) {
    p.dx = sint * cosp;
    p.dy = sint * sinp;
    p.dz = std::copysign(cost, p.dz * cost);
  } else {
    const R cxp = sint * (p.dx * p.dz * cosp - p.dy * sinp) / temp + p.dx * cost;
    const R cyp = sint * (p.dy * p.dz * cosp + p.dx * sinp) / temp + p.dy * cost;
    p.dz = -sint * cosp * temp + p.dz * cost;
    p.dx = cxp;
    p.dy = cyp;
  }
  temp = 1 / std::sqrt(p.dx * p.dx + p.dy * p.dy + p.dz * p.dz);
  p.dx *= temp;
  p.dy *= temp;
  p.dz *= temp;
}

// transport.cu:855-870
template <typename R, typename Rng>
bool survive(Ph<R> &p, Rng &g, bool cap) {
  if (cap && p.steps >= kMaxScatter) return false;
  if (p.w > (R)kWEIGHTI) return true;
  if (p.w == 0) return false;
  if (uni<R>(g) < (R)0.1f) {
    p.w = (R)rn_u32((double)(p.w / (R)0.1f));
    return true;
  }
  return false;
}

// transport.cu:433-435
template <typename R>
uint32_t drop(Ph<R> &p, const Tab<R> &t) {
  const R wq = (R)sat_u32((double)p.w);
  const uint32_t wt = rn_u32((double)(t.mua[p.layer] * t.mutr[p.layer] * wq));
  p.w = p.w - (R)wt;
  return wt;
}

// transport.cu:372-395; returns new_layer, s by reference.
template <typename R, typename Rng>
int hop(Ph<R> &p, R &s, Rng &g, const Tab<R> &t) {
  const int l = p.layer;
  s = -std::log(uni<R>(g)) * t.mutr[l];
  int nl = l;
  if (p.z + s * p.dz < t.z_min[l]) {
    nl--;
    s = (t.z_min[l] - p.z) / p.dz;
  }
  if (p.z + s * p.dz > t.z_max[l]) {
    nl++;
    s = (t.z_max[l] - p.z) / p.dz;
  }
  p.x += p.dx * s;
  p.y += p.dy * s;
  p.z += p.dz * s;
  return nl;
}

template <typename R>
void clampz(Ph<R> &p, const Tab<R> &t) {
  if (p.z > t.z_max[p.layer]) p.z = t.z_max[p.layer];
  if (p.z < t.z_min[p.layer]) p.z = t.z_min[p.layer];
}

// transport.cu:883-888 / 904-929 for detector i; weight out through wd.
template <typename R>
bool det_hit(const Ph<R> &p, const Tab<R> &t, int i, R &wd) {
  if (t.det_obl) {
    const R a = (p.x - t.det_pos[i]) * t.det_cos[i];
    if (a * a + p.y * p.y <= t.det_r[i] * t.det_r[i]) {
      const R uz = p.dx * t.det_sin[i] + std::fabs(p.dz * t.det_cos[i]);
      if (std::acos(std::fabs(uz)) <= t.det_crit[i]) {
        wd = p.w;
        return true;
      }
    }
    return false;
  }
  const R ang = std::acos(std::fabs(p.dz));
  const R dist = std::sqrt(p.x * p.x + p.y * p.y);
  if (ang <= t.det_crit[i]) {
    const R pos = t.det_pos[i], rad = t.det_r[i];
    if (dist >= pos - rad && dist <= pos + rad) {
      R c = (dist * dist + pos * pos - rad * rad) / (2 * dist * pos);
      if (c > 1) c = 1;
      wd = p.w * std::acos(c) * (R)kRPIf;
      return true;
    }
  }
  return false;
}

struct Detection {
  int sds;
  double w;
};

// First pass of one photon (one MCd photon, transport.cu:370-454).
// Appends every detection to det; returns the number of steps.
template <typename R, typename Rng>
int walk_first(Rng &g, const Tab<R> &t, Detection *det, int *n_det) {
  Ph<R> p;
  launch(p, g, t);
  *n_det = 0;
  for (;;) {
    R s;
    const int nl = hop(p, s, g, t);
    p.steps++;
    clampz(p, t);
    if (nl != p.layer) {
      const int temp_layer = p.layer;
      s = 0;
      if (!reflect(p, nl, g, t)) {
        if (nl == 0) {
          bool any = false;
          for (int i = 1; i <= t.n_sds; ++i) {
            R wd;
            if (det_hit(p, t, i, wd)) {
              det[(*n_det)++] = Detection{i, (double)wd};
              any = true;
            }
          }
          if (any)
            p.w = 0;
          else if (uni<R>(g) > t.det_refl)
            p.w = 0;
          else {
            p.dz = -p.dz;
            p.z = -p.z;
            p.layer = temp_layer;
          }
        }
        if (nl > t.n_layers) p.w = 0;
      }
    }
    if (s > 0) {
      drop(p, t);
      spin(p, t.g[p.layer], g);
    }
    if (!survive(p, g, true)) return p.steps;
    if (g.exhausted) return -1;
  }
}

// Energy bookkeeping of one photon's first pass (a known-answer test of
// the walk's weight arithmetic): every quantum of the start weight ends up
// absorbed, leaving through the top or the bottom, still held at the step
// cap, or removed / added by roulette -- up to the rounding of the float
// weight in `w - w_t`, which is tracked exactly (weights are integers, so
// each rounding is an integer).  roulette = false replaces the roulette by
// "live while w > 0" (the step cap still ends every photon).
struct Energy {
  double start, absorbed, top, bottom, capped, roulette_lost, roulette_gained, rounding;
};

template <typename R, typename Rng>
void walk_energy(Rng &g, const Tab<R> &t, bool roulette, Energy &e) {
  Ph<R> p;
  launch(p, g, t);
  e.start += (double)p.w;
  for (;;) {
    R s;
    const int nl = hop(p, s, g, t);
    p.steps++;
    clampz(p, t);
    if (nl != p.layer) {
      const int temp_layer = p.layer;
      s = 0;
      if (!reflect(p, nl, g, t)) {
        if (nl == 0) {
          bool any = false;
          for (int i = 1; i <= t.n_sds; ++i) {
            R wd;
            if (det_hit(p, t, i, wd)) any = true;
          }
          if (any || uni<R>(g) > t.det_refl) {
            e.top += (double)p.w;
            p.w = 0;
          } else {
            p.dz = -p.dz;
            p.z = -p.z;
            p.layer = temp_layer;
          }
        }
        if (nl > t.n_layers) {
          e.bottom += (double)p.w;
          p.w = 0;
        }
      }
    }
    if (s > 0) {
      const double before = (double)p.w;
      const uint32_t wt = drop(p, t);
      e.absorbed += (double)wt;
      e.rounding += (double)p.w - (before - (double)wt);
      spin(p, t.g[p.layer], g);
    }
    if (p.steps >= kMaxScatter) {
      e.capped += (double)p.w;
      return;
    }
    if (!roulette) {
      if (p.w == 0) return;
      continue;
    }
    const double before = (double)p.w;
    if (!survive(p, g, false)) {
      e.roulette_lost += before;
      return;
    }
    e.roulette_gained += (double)p.w - before;
  }
}

struct Grid {
  uint64_t *A_rz = nullptr;  // nz x nr of one SDS (may be null)
  uint64_t *A0_z = nullptr;  // nz of one SDS (may be null)
  uint32_t nr = 1000, nz = 500;
  float dr = 0.01f, dz = 0.01f;
};

// Replay of one photon for SDS sds (MCd_replay, transport.cu:506-613).
// row gets [weight, PL_1..PL_L, steps]; inter gets per-layer interaction
// counts.  Returns false if the draws ran out.
template <typename R, typename Rng>
bool walk_replay(Rng &g, const Tab<R> &t, int sds, double *row, uint32_t *inter,
                 const Grid &grid, double *w_exit = nullptr) {
  const int L = t.n_layers;
  Ph<R> p;
  launch(p, g, t);
  std::vector<R> pl(L, (R)0);
  std::fill(inter, inter + L, 0u);
  bool first = true;
  uint64_t idx_old = 0;
  uint32_t w_run = 0;
  int steps = 0;
  R w_det = 0;
  for (;;) {
    if (g.exhausted) return false;
    R s;
    const int nl = hop(p, s, g, t);
    steps++;
    pl[p.layer - 1] += s;
    clampz(p, t);
    if (nl != p.layer) {
      const int temp_layer = p.layer;
      s = 0;
      if (!reflect(p, nl, g, t)) {
        if (nl == 0) {
          R wd;
          if (det_hit(p, t, sds, wd)) {
            w_det = wd;
            if (w_exit) *w_exit = (double)p.w;  // the weight the detector weighs
            break;
          }
          if (uni<R>(g) > t.det_refl) break;
          p.dz = -p.dz;
          p.z = -p.z;
          p.layer = temp_layer;
        }
        if (nl > L) break;
      }
    }
    if (s > 0) {
      const uint32_t wt = drop(p, t);
      inter[p.layer - 1]++;
      const int iz = std::min((int)std::trunc((double)(p.z / (R)grid.dz)), (int)grid.nz - 1);
      if (first) {
        if (grid.A0_z) grid.A0_z[iz] += wt;
        first = false;
      } else {
        const R rr = std::sqrt(p.x * p.x + p.y * p.y);
        const int ir = std::min((int)std::trunc((double)(rr / (R)grid.dr)), (int)grid.nr - 1);
        const uint64_t index = (uint64_t)iz * grid.nr + ir;
        if (index == idx_old) {
          w_run += wt;
        } else {
          if (w_run && grid.A_rz) grid.A_rz[idx_old] += w_run;
          idx_old = index;
          w_run = wt;
        }
      }
      spin(p, t.g[p.layer], g);
    }
    if (!survive(p, g, false)) break;
  }
  if (w_run && grid.A_rz) grid.A_rz[idx_old] += w_run;
  if (g.exhausted) return false;
  row[0] = (double)w_det;
  for (int l = 0; l < L; ++l) row[1 + l] = (double)pl[l];
  row[L + 1] = (double)steps;
  return true;
}

}  // namespace

extern "C" {

// Derived constants (io.cpp:168-238).
int oracle_derive(const mcml_sim *sim, mcml_derived *out) {
  if (!sim || !out) return -1;
  derive_float(*sim, *out);
  return 0;
}

// First pass of one photon driven by recorded uniforms u[0..n_u).
// det_sds/det_w get up to 30 detections.  Returns the photon's step count,
// or -1 if the stream ran out.  *used = draws consumed.
int oracle_walk_stream(const mcml_sim *sim, int fp64, const float *u, uint64_t n_u,
                       int *n_det, int *det_sds, double *det_w, uint64_t *used) {
  StreamRng g{u, n_u};
  Detection det[MCML_MAX_SDS];
  int steps;
  if (fp64) {
    Tab<double> t;
    make_tab(*sim, t);
    steps = walk_first(g, t, det, n_det);
  } else {
    Tab<float> t;
    make_tab(*sim, t);
    steps = walk_first(g, t, det, n_det);
  }
  for (int i = 0; i < *n_det; ++i) {
    det_sds[i] = det[i].sds;
    det_w[i] = det[i].w;
  }
  if (used) *used = g.i;
  return g.exhausted ? -1 : steps;
}

// Replay of one photon for SDS sds (1-based) driven by recorded uniforms.
// row[L+2], inter[L]; A_rz (nz*nr) / A0_z (nz) of this SDS may be null.
// w_exit (may be NULL): the photon's weight as it leaves through the
// detector, before the ring weighting (transport.cu:1000-1002).
int oracle_replay_stream(const mcml_sim *sim, int fp64, int sds, const float *u, uint64_t n_u,
                         double *row, uint32_t *inter, uint64_t *A_rz, uint64_t *A0_z,
                         uint64_t *used, double *w_exit) {
  StreamRng g{u, n_u};
  Grid grid;
  grid.A_rz = A_rz;
  grid.A0_z = A0_z;
  bool ok;
  if (fp64) {
    Tab<double> t;
    make_tab(*sim, t);
    ok = walk_replay(g, t, sds, row, inter, grid, w_exit);
  } else {
    Tab<float> t;
    make_tab(*sim, t);
    ok = walk_replay(g, t, sds, row, inter, grid, w_exit);
  }
  if (used) *used = g.i;
  return ok ? 0 : -1;
}

typedef struct oracle_stats {
  uint64_t photons;
  uint64_t steps;
  uint64_t detected[MCML_MAX_SDS];
  double wsum[MCML_MAX_SDS];
  double wsq[MCML_MAX_SDS];
} oracle_stats;

// Statistical first pass: photons [first, first+count) with PCG32 stream
// (seed, photon).  Detection lists (photon, sds, weight) go to the caller's
// arrays up to cap entries; *n_out gets the total.  threads<=0: all cores.
int oracle_run(const mcml_sim *sim, int fp64, uint64_t seed, uint64_t first, uint64_t count,
               int threads, oracle_stats *stats, uint64_t *det_photon, int32_t *det_sds,
               double *det_w, uint64_t cap, uint64_t *n_out) {
  if (!sim || !stats) return -1;
  std::memset(stats, 0, sizeof(*stats));
  Tab<float> tf;
  Tab<double> td;
  make_tab(*sim, tf);
  make_tab(*sim, td);
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#endif
  uint64_t n_det_total = 0;
  const int S = (int)sim->num_sds;
#pragma omp parallel
  {
    oracle_stats loc;
    std::memset(&loc, 0, sizeof(loc));
    std::vector<uint64_t> lp;
    std::vector<int32_t> ls;
    std::vector<double> lw;
#pragma omp for schedule(dynamic, 256)
    for (int64_t k = 0; k < (int64_t)count; ++k) {
      const uint64_t ph = first + (uint64_t)k;
      Pcg32 g;
      g.seed(seed, ph);
      Detection det[MCML_MAX_SDS];
      int nd = 0;
      const int steps = fp64 ? walk_first(g, td, det, &nd) : walk_first(g, tf, det, &nd);
      loc.steps += (uint64_t)steps;
      for (int i = 0; i < nd; ++i) {
        const int s = det[i].sds - 1;
        loc.detected[s]++;
        loc.wsum[s] += det[i].w;
        loc.wsq[s] += det[i].w * det[i].w;
        lp.push_back(ph);
        ls.push_back(det[i].sds);
        lw.push_back(det[i].w);
      }
    }
#pragma omp critical
    {
      stats->steps += loc.steps;
      for (int s = 0; s < S; ++s) {
        stats->detected[s] += loc.detected[s];
        stats->wsum[s] += loc.wsum[s];
        stats->wsq[s] += loc.wsq[s];
      }
      for (size_t i = 0; i < lp.size(); ++i) {
        if (n_det_total < cap && det_photon) {
          det_photon[n_det_total] = lp[i];
          det_sds[n_det_total] = ls[i];
          det_w[n_det_total] = lw[i];
        }
        ++n_det_total;
      }
    }
  }
  stats->photons = count;
  if (n_out) *n_out = n_det_total;
  return 0;
}

// Statistical replay of detections from oracle_run: rows (n x (L+2)),
// inter (n x L), and per-SDS tallies A_rz (S x nz x nr), A0_z (S x nz),
// any of which may be null.
int oracle_replay(const mcml_sim *sim, int fp64, uint64_t seed, uint64_t n,
                  const uint64_t *det_photon, const int32_t *det_sds, int threads, double *rows,
                  uint32_t *inter, uint64_t *A_rz, uint64_t *A0_z, uint32_t nr, uint32_t nz,
                  float dr, float dz) {
  if (!sim) return -1;
  Tab<float> tf;
  Tab<double> td;
  make_tab(*sim, tf);
  make_tab(*sim, td);
  const int L = (int)sim->num_layers;
  const int S = (int)sim->num_sds;
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#endif
  int bad = 0;
#pragma omp parallel
  {
    std::vector<uint64_t> arz(A_rz ? (size_t)S * nz * nr : 0), a0z(A0_z ? (size_t)S * nz : 0);
    std::vector<double> row(L + 2);
    std::vector<uint32_t> ni(L);
#pragma omp for schedule(dynamic, 16)
    for (int64_t k = 0; k < (int64_t)n; ++k) {
      Pcg32 g;
      g.seed(seed, det_photon[k]);
      const int s = det_sds[k];
      Grid grid;
      grid.nr = nr;
      grid.nz = nz;
      grid.dr = dr;
      grid.dz = dz;
      grid.A_rz = A_rz ? arz.data() + (size_t)(s - 1) * nz * nr : nullptr;
      grid.A0_z = A0_z ? a0z.data() + (size_t)(s - 1) * nz : nullptr;
      const bool ok = fp64 ? walk_replay(g, td, s, row.data(), ni.data(), grid)
                           : walk_replay(g, tf, s, row.data(), ni.data(), grid);
      if (!ok) {
#pragma omp atomic
        bad++;
      }
      if (rows)
        for (int j = 0; j < L + 2; ++j) rows[(size_t)k * (L + 2) + j] = row[j];
      if (inter)
        for (int l = 0; l < L; ++l) inter[(size_t)k * L + l] = ni[l];
    }
#pragma omp critical
    {
      for (size_t i = 0; i < arz.size(); ++i) A_rz[i] += arz[i];
      for (size_t i = 0; i < a0z.size(); ++i) A0_z[i] += a0z[i];
    }
  }
  return bad ? -1 : 0;
}

// Energy bookkeeping (walk_energy) of photons [0, count) with PCG32
// streams of `seed`; out: start, absorbed, top, bottom, capped,
// roulette_lost, roulette_gained, rounding (weight quanta, FP64 sums of
// integers).  Single-threaded so the sums are exact.
int oracle_energy(const mcml_sim *sim, int fp64, uint64_t seed, uint64_t count, int roulette,
                  double *out) {
  if (!sim || !out) return -1;
  Energy e{};
  Tab<float> tf;
  Tab<double> td;
  make_tab(*sim, tf);
  make_tab(*sim, td);
  for (uint64_t k = 0; k < count; ++k) {
    Pcg32 g;
    g.seed(seed, k);
    if (fp64)
      walk_energy(g, td, roulette != 0, e);
    else
      walk_energy(g, tf, roulette != 0, e);
  }
  const double v[8] = {e.start, e.absorbed, e.top, e.bottom, e.capped, e.roulette_lost,
                       e.roulette_gained, e.rounding};
  std::memcpy(out, v, sizeof(v));
  return 0;
}

}  // extern "C"
