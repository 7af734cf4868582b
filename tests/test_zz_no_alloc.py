"""mcml_run_noalloc: the first pass for callers that cannot allocate device
memory (pipelines whose device memory is fixed at start-up, where cudaMalloc
could block mid-run, or processes whose GPU memory another framework's pool
owns), with its scratch memory in a fixed array inside the library.

Called through the C ABI, twice in a row on the same fixed scratch array,
it must give what mcml_run gives for the same seed and slot count: the
per-SDS detected counts exactly and the FP64 weight sums to 1e-12
(only the order of the floating-point atomic additions differs).  The file
is named to be collected last, so a stop-at-first-failure run has already
run every other test; it also passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import load_case

import mcml_gpu_b200 as m

MAX_SLOTS = ((8 << 20) - 1024) // 24


def run_noalloc(sim, seed, slots):
    import torch
    lib = m.load_library()
    out = torch.zeros(C.sizeof(m.NoallocResult), dtype=torch.uint8, device="cuda:0")
    stream = torch.cuda.current_stream(0).cuda_stream
    rc = lib.mcml_run_noalloc(C.byref(sim), seed, slots, 0, C.c_void_p(stream),
                              C.c_void_p(out.data_ptr()))
    assert rc == 0, lib.mcml_last_error()
    torch.cuda.synchronize(0)
    return m.NoallocResult.from_buffer_copy(out.cpu().numpy().tobytes())


def check_same(ref, got, S):
    assert [int(v) for v in got.detected[:S]] == [int(v) for v in ref.detected[:S]]
    np.testing.assert_allclose(list(got.weight_sum[:S]), list(ref.weight_sum[:S]), rtol=1e-12)
    np.testing.assert_allclose(list(got.weight_sumsq[:S]), list(ref.weight_sumsq[:S]), rtol=1e-12)
    assert int(got.steps) == int(ref.steps)


@pytest.mark.gpu
@pytest.mark.parametrize("case,photons,slots", [
    ("fiber3", 303104, 303104),    # the reference's one-photon-per-thread layout
    ("ring5", 303104, 0),          # slots = 0: min(N, capacity)
    ("mismatch", 2_000_000, 250000),
])
def test_noalloc_matches_mcml_run_twice(case, photons, slots, gpu_available):
    sim = load_case(case)
    sim.number_photons = photons
    seed = 20261203
    used_slots = slots or min(photons, MAX_SLOTS)
    with m.Simulation(sim, seed=seed, slots=used_slots) as s:
        ref = s.run()
    S = sim.num_sds
    first = run_noalloc(sim, seed, slots)
    second = run_noalloc(sim, seed, slots)
    check_same(ref, first, S)
    check_same(ref, second, S)


@pytest.mark.gpu
def test_noalloc_rejects_more_slots_than_its_scratch(gpu_available):
    import torch
    sim = load_case("fiber3")
    sim.number_photons = 10 * MAX_SLOTS
    lib = m.load_library()
    out = torch.zeros(C.sizeof(m.NoallocResult), dtype=torch.uint8, device="cuda:0")
    rc = lib.mcml_run_noalloc(C.byref(sim), 1, MAX_SLOTS + 1, 0, None, C.c_void_p(out.data_ptr()))
    assert rc == -1
    assert b"exceed the fixed scratch capacity" in lib.mcml_last_error()
