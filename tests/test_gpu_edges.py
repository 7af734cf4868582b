"""Edge cases of the walk on the GPU: the largest configuration the
formats allow (10 layers, 30 ring SDS) and a single layer, each against
the CPU restatement's FP64 statistics (within 4 standard errors of the
difference); tiny and ragged photon counts (1, 2, 7 photons, counts that
do not divide into the slots), where every photon must be walked exactly
once and the replay must reproduce every detection."""
import math

import numpy as np
import pytest

import mcml_gpu_b200 as m
import oracle


def ring_sim(n_layers, n_sds, photons):
    rng = np.random.default_rng(n_layers * 100 + n_sds)
    layers = []
    for l in range(n_layers):
        layers.append((float(rng.uniform(0.05, 0.3)), float(rng.uniform(0.05, 0.5)),
                       float(rng.uniform(20, 120)), 1.4, 0.85))
    dets = [(0.1 + 0.06 * i, 0.8, 0.03, 0.0) for i in range(n_sds)]
    return m.make_sim(layers, dets, photons=photons, source_oblique=False,
                      detector_oblique=False, source=(0.0, 0.0, 0.0))


def compare_with_oracle(sim, photons, seed):
    sim.number_photons = photons
    with m.Simulation(sim, seed=seed) as run:
        r = run.run()
    st, *_ = oracle.run(sim, photons, seed + 1, fp64=True)
    S = int(sim.num_sds)
    scale = float(0xFFFFFFFF) * photons
    checked = 0
    for s in range(S):
        g_mean, g_se = r.reflectance[s], r.std_error[s]
        o_mean = st.wsum[s] / scale
        o_var = max(st.wsq[s] / photons - (st.wsum[s] / photons) ** 2, 0.0)
        o_se = math.sqrt(o_var / (photons - 1)) / float(0xFFFFFFFF)
        se = math.hypot(g_se, o_se)
        if se > 0:
            assert abs(g_mean - o_mean) <= 4 * se, (s, g_mean, o_mean, se)
            checked += 1
    return checked


@pytest.mark.gpu
def test_ten_layers_thirty_sds_match_oracle_statistics(gpu_available):
    sim = ring_sim(m.MAX_LAYERS, m.MAX_SDS, 0)
    assert compare_with_oracle(sim, 400_000, 21) >= 25


@pytest.mark.gpu
def test_single_layer_matches_oracle_statistics(gpu_available):
    sim = ring_sim(1, 4, 0)
    assert compare_with_oracle(sim, 400_000, 5) == 4


@pytest.mark.gpu
@pytest.mark.parametrize("photons,slots", [(1, 0), (2, 0), (7, 0), (1000, 7), (4099, 64), (100003, 0)])
def test_tiny_and_ragged_photon_counts(photons, slots, gpu_available):
    sim = ring_sim(3, 3, photons)
    with m.Simulation(sim, seed=9, slots=slots) as run:
        r = run.run()
        assert int(r.photons) == photons
        if slots:
            assert int(r.slots) == slots
        else:
            assert int(r.slots) == photons  # below the reference's thread count: one per slot
        assert int(r.steps) >= photons  # every photon took at least one step
        run.replay()
        for s in range(1, 4):
            ids, w = run.detections(s)
            rows, _ = run.rows(s)
            assert len(ids) == len(rows) == int(r.detected[s - 1])
            assert np.all(ids < photons)
            assert np.array_equal(rows[:, 0], w.astype(np.float32))
