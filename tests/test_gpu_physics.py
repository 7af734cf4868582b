"""Known-answer tests of the walk's own device functions on the GPU
(mcml_probe_spin / mcml_probe_reflect run spin() and reflect() of the
product kernels):

  * Henyey-Greenstein: E[cos] = g, E[cos^2] = (1 + 2 g^2) / 3; g = 0 is
    the isotropic 2u - 1 branch (E[cos^2] = 1/3);
  * Fresnel at normal incidence: R = ((n1 - n2)/(n1 + n2))^2, transmitted
    photons keep |dz| = 1;
  * oblique incidence: the unpolarised Fresnel R, transmitted |dz| from
    Snell's law;
  * total internal reflection beyond the critical angle (R = 1 exactly);
    matched indices pass everything unchanged.
Statistical checks use 5 standard errors of the sample mean."""
import math

import numpy as np
import pytest

import mcml_gpu_b200 as m

N = 8_000_000


@pytest.mark.gpu
@pytest.mark.parametrize("g", [0.0, 0.5, 0.9, -0.3])
def test_henyey_greenstein_moments(g, gpu_available):
    c1, c2 = m.probe_spin(g, N, seed=11)
    var = (1 + 2 * g * g) / 3 - g * g
    assert abs(c1 - g) < 5 * math.sqrt(var / N), (c1, g)
    # cos^2 has variance below 1/4 on [0, 1]
    assert abs(c2 - (1 + 2 * g * g) / 3) < 5 * math.sqrt(0.25 / N), (c2, g)


def fresnel(n1, n2, c):
    s = n1 / n2 * math.sqrt(1 - c * c)
    if s >= 1:
        return 1.0, None
    ct = math.sqrt(1 - s * s)
    rs = ((n1 * c - n2 * ct) / (n1 * c + n2 * ct)) ** 2
    rp = ((n1 * ct - n2 * c) / (n1 * ct + n2 * c)) ** 2
    return 0.5 * (rs + rp), ct


@pytest.mark.gpu
@pytest.mark.parametrize("n1,n2,c", [
    (1.4, 1.457, 1.0),   # tissue -> probe glass, normal incidence
    (1.4, 1.0, 1.0),     # tissue -> air, normal incidence
    (1.4, 1.0, 0.9),
    (1.0, 1.4, 0.3),
    (1.4, 1.457, 0.5),
    (1.4, 1.0, 0.75),    # just inside the critical angle (cos 0.6999)
    (1.4, 1.0, 0.5),     # total internal reflection
    (1.4, 1.4, 0.6),     # matched indices
])
def test_fresnel_and_snell(n1, n2, c, gpu_available):
    n1f, n2f, cf = (float(np.float32(v)) for v in (n1, n2, c))
    frac, dz_t = m.probe_reflect(n1f, n2f, cf, N, seed=5)
    if n1 == n2:
        assert frac == 0.0 and abs(dz_t - cf) < 1e-6
        return
    R, ct = fresnel(n1f, n2f, cf)
    if ct is None:
        assert frac == 1.0 and dz_t == 0.0
        return
    assert abs(frac - R) < 5 * math.sqrt(max(R * (1 - R), 1e-12) / N) + 1e-7, (frac, R)
    # every transmitted photon has the Snell cosine; dz_t is its mean times (1 - frac)
    assert abs(dz_t / (1 - frac) - ct) < 2e-6, (dz_t / (1 - frac), ct)
    if c == 1.0:
        assert abs(R - ((n1f - n2f) / (n1f + n2f)) ** 2) < 1e-12
