"""White Monte Carlo relabelling (mcml_wmc_rescale).

* numerics: the kernel equals the float64 formula on the same replay rows
  to 5e-5 relative: the FP32 exponent sums terms of size up to ~300
  (dmu_t * PL), so it carries an absolute error of ~2e-5, which exp2
  turns into that relative error;
* identity: unchanged coefficients give back the replay's own reflectance;
* physics: reflectance relabelled from one baseline replay to other
  (mua, mus) agrees with plain MC walked at those coefficients within
  4 combined standard errors.
"""
import numpy as np
import pytest

from conftest import load_case

import mcml_gpu_b200 as m
from mcml_gpu_b200 import wmc

SEED = 4242


def baseline(case, photons):
    sim = load_case(case)
    sim.number_photons = photons
    with m.Simulation(sim, seed=SEED) as run:
        r = run.run()
        run.replay()
        rows = [run.rows(s) for s in range(1, sim.num_sds + 1)]
    return sim, r, rows


def combos_around(sim, n, rng, spread=0.3):
    L = sim.num_layers
    mua = np.array(sim.mua[:L], np.float64)
    mus = np.array(sim.mus[:L], np.float64)
    fa = rng.uniform(1 - spread, 1 + spread, (n, L))
    fs = rng.uniform(1 - spread / 3, 1 + spread / 3, (n, L))
    return np.hstack([mua * fa, mus * fs]).astype(np.float32)


@pytest.mark.gpu
def test_wmc_matches_float64_formula(gpu_available):
    sim, r, rows = baseline("ring5", 303104)
    L = sim.num_layers
    rng = np.random.default_rng(1)
    combos = combos_around(sim, 3000, rng)
    for sds in range(sim.num_sds):
        R, inter = rows[sds]
        got = wmc.rescale(R, inter, sim.mua[:L], sim.mus[:L], combos, sim.number_photons).cpu().numpy()
        ref = wmc.rescale_reference(R, inter, sim.mua[:L], sim.mus[:L], combos, sim.number_photons)
        np.testing.assert_allclose(got, ref, rtol=5e-5)


@pytest.mark.gpu
def test_wmc_identity_gives_replay_reflectance(gpu_available):
    sim, r, rows = baseline("fiber3", 303104)
    L = sim.num_layers
    same = np.array([list(sim.mua[:L]) + list(sim.mus[:L])], np.float32)
    for sds in range(sim.num_sds):
        R, inter = rows[sds]
        got = float(wmc.rescale(R, inter, sim.mua[:L], sim.mus[:L], same, sim.number_photons)[0])
        np.testing.assert_allclose(got, r.reflectance[sds], rtol=1e-6)


@pytest.mark.gpu
def test_wmc_agrees_with_plain_mc(gpu_available):
    sim, r, rows = baseline("ring5", 4_000_000)
    L = sim.num_layers
    rng = np.random.default_rng(7)
    combos = combos_around(sim, 4, rng, spread=0.25)
    for c in combos:
        target = load_case("ring5")
        target.number_photons = 4_000_000
        for l in range(L):
            target.mua[l] = float(c[l])
            target.mus[l] = float(c[L + l])
        with m.Simulation(target, seed=SEED + 1) as run:
            direct = run.run()
        for sds in range(sim.num_sds):
            R, inter = rows[sds]
            got = float(wmc.rescale(R, inter, sim.mua[:L], sim.mus[:L], c[None, :], sim.number_photons)[0])
            se = np.hypot(direct.std_error[sds], r.std_error[sds])
            assert abs(got - direct.reflectance[sds]) <= 4 * se, (sds, got, direct.reflectance[sds], se)
