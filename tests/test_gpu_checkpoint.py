"""Checkpoint / resume of the first pass (mcml_run_checkpointed).

A run stopped after a few launches and resumed in a fresh context from its
checkpoint file must detect the same photons as one uninterrupted
mcml_run with the same seed and slots: the same per-SDS counts, the same
replayed pathlength rows bit for bit, the same u64 absorbance tallies.
Interruption is made on the host (max_chunks), not by failing the GPU.
"""
import numpy as np
import pytest

from conftest import load_case

import mcml_gpu_b200 as m

SEED = 4242


def outputs(run, S):
    rows = [run.rows(s)[0].copy() for s in range(1, S + 1)]
    a_rz, a0_z = run.tallies()
    return rows, a_rz.copy(), a0_z.copy()


def reference_run(sim, slots):
    with m.Simulation(sim, seed=SEED, slots=slots) as run:
        first = run.run()
        run.replay()
        return first, outputs(run, sim.num_sds)


@pytest.mark.gpu
@pytest.mark.parametrize("case,photons,slots,chunk,capacity", [
    ("ring5", 1_000_000, 125_000, 20_000, 0),
    ("fiber3", 2_000_000, 250_000, 64_000, 0),
    ("ring5", 400_000, 50_000, 7_000, 16),   # record buffer regrown inside a launch
])
def test_resumed_run_equals_uninterrupted(case, photons, slots, chunk, capacity, tmp_path,
                                          gpu_available):
    sim = load_case(case)
    sim.number_photons = photons
    S = sim.num_sds
    first, (rows, a_rz, a0_z) = reference_run(sim, slots)
    path = tmp_path / "walk.ckpt"
    with m.Simulation(sim, seed=SEED, slots=slots, record_capacity=capacity) as run:
        assert run.run_checkpointed(path, chunk_slots=chunk, max_chunks=2) is None
    info = m.checkpoint_info(path)
    assert (info.launches, info.slots_done, info.slots, info.seed) == (2, 2 * chunk, slots, SEED)
    with m.Simulation(sim, seed=SEED, slots=slots, record_capacity=capacity) as run:
        assert run.run_checkpointed(path, chunk_slots=chunk, max_chunks=1) is None
        res = run.run_checkpointed(path, chunk_slots=chunk)
        assert res is not None
        info = m.checkpoint_info(path)
        assert info.slots_done == slots and info.launches == -(-slots // chunk)
        assert info.steps == res.steps == first.steps
        assert [int(v) for v in res.detected[:S]] == [int(v) for v in first.detected[:S]]
        np.testing.assert_allclose(res.weight_sum[:S], first.weight_sum[:S], rtol=1e-12)
        run.replay()
        rows2, a_rz2, a0_z2 = outputs(run, S)
    for a, b in zip(rows, rows2):
        assert a.tobytes() == b.tobytes()
    assert np.array_equal(a_rz, a_rz2) and np.array_equal(a0_z, a0_z2)
    # a finished checkpoint resumes to the same result without walking
    with m.Simulation(sim, seed=SEED, slots=slots) as run:
        again = run.run_checkpointed(path)
        assert [int(v) for v in again.detected[:S]] == [int(v) for v in first.detected[:S]]


@pytest.mark.gpu
def test_checkpoint_of_another_run_is_rejected(tmp_path, gpu_available):
    sim = load_case("ring5")
    sim.number_photons = 200_000
    path = tmp_path / "walk.ckpt"
    with m.Simulation(sim, seed=1, slots=20_000) as run:
        assert run.run_checkpointed(path, chunk_slots=5000, max_chunks=1) is None
    before = path.read_bytes()
    for kw, edit in [({"seed": 2, "slots": 20_000}, None), ({"seed": 1, "slots": 25_000}, None),
                     ({"seed": 1, "slots": 20_000}, "mua")]:
        other = m.Sim.from_buffer_copy(sim)
        if edit:
            other.mua[0] *= 1.5
        with m.Simulation(other, **kw) as run:
            with pytest.raises(m.MCMLError) as e:
                run.run_checkpointed(path, chunk_slots=5000)
            assert e.value.status == -10
    assert path.read_bytes() == before
