// params.h -- building the kernel parameter block of one simulation.
#pragma once

#include <cstring>

#include "../../include/mcml_b200.h"
#include "photon.cuh"

namespace mcml {

// The reference's __constant__ tables (header.h:205-214, filled by InitDCMem,
// transport.cu:1002-1035) as one by-value kernel argument.  Layers 0 and
// L+1 carry only their refractive index, as in the reference.
inline void fill_dev_params(const mcml_sim &s, const mcml_derived &d, uint64_t photons,
                            uint64_t slots, DevParams &P) {
  std::memset(&P, 0, sizeof(P));
  const int L = (int)s.num_layers;
  for (int l = 0; l <= L + 1; ++l) {
    P.z_min[l] = d.z_min[l];
    P.z_max[l] = d.z_max[l];
    P.mutr[l] = d.mutr[l];
    if (l >= 1 && l <= L) {
      P.mua[l] = s.mua[l - 1];
      P.g[l] = s.g[l - 1];
      P.n[l] = s.n[l - 1];
    }
  }
  P.n[0] = s.upper_n;
  P.n[L + 1] = s.lower_n;
  P.det_radius[0] = s.source_radius;
  P.det_NA[0] = s.source_NA;
  P.det_pos[0] = 0.0f;
  P.det_angle[0] = d.det_angle_rad[0];
  for (unsigned i = 0; i < s.num_sds; ++i) {
    P.det_radius[i + 1] = s.det_radius[i];
    P.det_NA[i + 1] = s.det_NA[i];
    P.det_pos[i + 1] = s.det_pos[i];
    P.det_angle[i + 1] = d.det_angle_rad[i + 1];
    P.crit[i + 1] = d.critical_angle[i + 1];
  }
  P.n_layers = s.num_layers;
  P.n_sds = s.num_sds;
  P.start_weight = d.start_weight;
  P.det_reflectance = s.detector_reflectance;
  P.num_photons = photons;
  P.num_slots = slots;
}

}  // namespace mcml
