"""End to end: White-MC labels from replayed baselines -> MLP ensemble trained
on the GPU -> served predictions, compared with plain MC.

The network is configuration C3's: 25 inputs -> 4 hidden layers of 256,
GELU -> 3 log-reflectances, an ensemble of 4, BF16 tensor-core training.
The held-out tissues are drawn like the labels (a baseline's scattering
within a few percent, clipped to 50-250 /cm, absorption anywhere in
range).  The network must (a) agree with plain MC walked at 2e7 photons
per tissue within 2 % median relative error (the references' own standard
error is about 0.4 %), and (b) beat plain MC given the same GPU time as the
network's inference -- the gain the trained network brings over the
method without it.  Queries outside the training hull go to plain MC.
"""
import time

import numpy as np
import pytest
import torch

from conftest import CONFIGS

import mcml_gpu_b200 as m
import mcml_gpu_b200.surrogate as sg


def base_sim():
    d = CONFIGS / "surrogate"
    return m.parse_config(d / "sim_set.json", d / "input.txt")[0]


def held_out(labels, count, rng, mua_range=(0.05, 0.5), jitter=0.05):
    out = []
    L = int(labels.baselines[0].num_layers)
    for k in range(count):
        b = labels.baselines[k % len(labels.baselines)]
        s = m.Sim.from_buffer_copy(b)
        for l in range(L):
            s.mua[l] = float(rng.uniform(*mua_range))
            s.mus[l] = float(np.clip(b.mus[l] * rng.uniform(1 - jitter, 1 + jitter), 50.0, 250.0))
        out.append(s)
    return out


@pytest.mark.gpu
def test_surrogate_beats_equal_cost_plain_mc(gpu_available):
    base = base_sim()
    labels = sg.make_labels(base, n_baselines=8, photons=5_000_000, combos_per_baseline=4000,
                            seed=3)
    sur = sg.Surrogate.train(labels, epochs=40, batch=1024, lr=2e-3, hidden=256, depth=4,
                             ensemble=4, seed=1, max_spread=1.0)
    assert sur.history[-1].mean() < sur.history[0].mean()
    rng = np.random.default_rng(11)
    tissues = held_out(labels, 12, rng)
    # surrogate answers (all inside the hull, so no fallback)
    X = sg.features(tissues)
    t0 = time.perf_counter()
    logR, spread = sur.predict(X)
    t_sur = time.perf_counter() - t0
    R_sur = np.exp(logR)
    # plain MC references at 2e7 photons per tissue
    refs = []
    for t in tissues:
        s = m.Sim.from_buffer_copy(t)
        s.number_photons = 20_000_000
        refs.append(s)
    with m.Batch(refs, seed=99) as b:
        res = b.run()
    R_ref = np.array([r.reflectance[:3] for r in res])
    se = np.array([r.std_error[:3] for r in res])
    rel = np.abs(R_sur - R_ref) / R_ref
    # plain MC with the network's cost: photons that fit in the same time
    rate = sum(int(s.number_photons) for s in refs) / (res[0].walk_ms / 1e3)
    cheap_photons = max(1000, int(rate * max(t_sur, 1e-3) / len(tissues)))
    cheap = []
    for t in tissues:
        s = m.Sim.from_buffer_copy(t)
        s.number_photons = cheap_photons
        cheap.append(s)
    with m.Batch(cheap, seed=7, photons_per_slot=8) as b:
        cres = b.run()
    R_cheap = np.array([r.reflectance[:3] for r in cres])
    rel_cheap = np.abs(R_cheap - R_ref) / R_ref
    print("surrogate median rel err", np.median(rel), "MC SE/R", np.median(se / R_ref),
          "equal-cost MC photons", cheap_photons, "its median rel err", np.median(rel_cheap))
    assert np.median(rel) < 0.02
    assert np.median(rel) < np.median(rel_cheap)
    # out-of-hull queries fall back to plain MC
    far = m.Sim.from_buffer_copy(tissues[0])
    far.mua[0] = 2.0
    R_fb, used_mc = sur.serve([tissues[1], far])
    assert list(used_mc) == [False, True]
    assert np.all(R_fb[1] >= 0)
