"""Batched multi-set launch (mcml_batch_*): every set of a batch gives what
the same set gives alone with the same seed and slot count -- detected
counts exactly, FP64 weight sums to 1e-12 (atomic summation order) -- with
and without CUDA-graph capture, over repeated runs, and for the reference's
one-photon-per-thread layout the reference's own detected counts."""
import numpy as np
import pytest

from conftest import GOLDEN, load_case

import mcml_gpu_b200 as m


def same(a, b, S):
    assert [int(v) for v in a.detected[:S]] == [int(v) for v in b.detected[:S]]
    np.testing.assert_allclose(list(a.weight_sum[:S]), list(b.weight_sum[:S]), rtol=1e-12)
    assert int(a.steps) == int(b.steps)


@pytest.mark.gpu
@pytest.mark.parametrize("graph", [True, False])
def test_batch_sets_equal_single_runs(graph, gpu_available):
    base = load_case("fiber3")
    sims = m.sample_sets(base, 12, seed=5, photons=(2e4, 2e5))
    pps = 16
    seed = 777
    with m.Batch(sims, seed=seed, photons_per_slot=pps, graph=graph) as b:
        res = b.run()
        again = b.run()
    for i, sim in enumerate(sims):
        N = int(sim.number_photons)
        with m.Simulation(sim, seed=seed + i, slots=-(-N // pps)) as s:
            ref = s.run()
        same(res[i], ref, sim.num_sds)
        same(again[i], ref, sim.num_sds)


@pytest.mark.gpu
def test_batch_reproduces_reference_counts(gpu_available):
    g = np.load(GOLDEN / "golden_fiber3.npz")
    sim = load_case("fiber3")
    T = int(g["threads"])
    sim.number_photons = T
    other = load_case("fiber3")
    other.number_photons = 5000
    # the golden set is set 0 (seed = seed + 0); one photon per slot
    with m.Batch([sim, other], seed=int(g["seed"]), photons_per_slot=1) as b:
        res = b.run()
    assert [int(v) for v in res[0].detected[:3]] == [int(v) for v in g["detected"]]


@pytest.mark.gpu
def test_batch_autotune_keeps_results_valid(gpu_available):
    base = load_case("ring5")
    sims = m.sample_sets(base, 16, seed=9, photons=(1e4, 1e5))
    with m.Batch(sims, seed=3) as b:
        t = b.autotune(0.25)
        assert t.photons_per_slot in (4, 8, 32) and t.block_size in (128, 256)
        res = b.run()
    for r, s in zip(res, sims):
        assert int(r.photons) == int(s.number_photons)
        assert int(r.slots) == -(-int(s.number_photons) // t.photons_per_slot)
        assert r.steps > 0
