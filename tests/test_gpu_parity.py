"""Parity of the CUDA walk and replay with the reference's own outputs.

The golden fixtures (tests/golden/golden_<case>.npz, made by
tests/golden/make_golden.py from the reference built for sm_100a) hold
what the reference wrote with a pinned seed and N equal to its thread
count (one photon per thread, deterministic).  With the same seed and the
same slot layout the library must reproduce:
  * the per-SDS detected counts exactly (SDS_detected_number);
  * every pathlength_SDS_#.bin row bit for bit (weight, per-layer
    pathlength, steps) -- the required tolerance for pathlengths is
    1e-5 relative, the walk here meets 0;
  * A0_z_SDS_#.bin exactly and A_rz_SDS_#.bin by SHA-256;
  * average_pathlength.txt byte for byte (same rows, same FP64 formula);
  * the FP64 weight sums within 1e-12 of the exact sum of the reference's
    rows; output.txt within 6-digit print precision of that sum, and
    within the reference's float32 summation error of its own output.txt
    (it sums detected weights in float, this library in double).
"""
import hashlib
import os
import tempfile
from pathlib import Path

import numpy as np
import pytest

from conftest import GOLDEN, load_case

import mcml_gpu_b200 as m

GOLDEN_DIR = Path(os.environ.get("MCML_GOLDEN_DIR", GOLDEN))
CASES = ["fiber3", "ring5", "mismatch", "ringpt", "three_layer", "surrogate", "hw8a",
         "head_model"]
STAT_CASES = ["fiber3", "ring5", "mismatch", "ringpt", "surrogate", "hw8a", "head_model"]


def same_or_both_nan(a: float, b: float, tol: float) -> bool:
    """|a - b| <= tol, or both NaN: the reference's ring detector at pos = 0
    (example/HW8_A) divides by 2*d*pos = 0 and records NaN weights
    (transport.cu:915), which every sum over that SDS carries."""
    if np.isnan(a) or np.isnan(b):
        return bool(np.isnan(a) and np.isnan(b))
    return abs(a - b) <= tol


def golden(case):
    p = GOLDEN_DIR / f"golden_{case}.npz"
    if not p.exists():
        pytest.fail(f"missing golden fixture {p}")
    return np.load(p)


def run_case(case, g):
    sim = load_case(case)
    T = int(g["threads"])
    sim.number_photons = T
    s = m.Simulation(sim, seed=int(g["seed"]), slots=T)
    first = s.run()
    replay = s.replay()
    return sim, s, first, replay


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES)
def test_detected_counts_and_rows_bit_exact(case, gpu_available):
    g = golden(case)
    sim, s, first, _ = run_case(case, g)
    with s:
        S, L = sim.num_sds, sim.num_layers
        assert [int(v) for v in first.detected[:S]] == [int(v) for v in g["detected"]]
        for sds in range(1, S + 1):
            rows, inter = s.rows(sds)
            ref = g[f"rows_{sds}"]
            assert rows.shape == ref.shape
            # bit-exact float32 rows (weight, PL_1..PL_L, steps)
            assert np.array_equal(rows.view(np.uint32), ref.view(np.uint32)), (
                f"SDS {sds}: {np.count_nonzero(rows != ref)} differing values")
            # interaction counts never exceed the step count
            assert np.all(inter.sum(axis=1) <= rows[:, L + 1])


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES)
def test_tallies_and_files_match_reference(case, gpu_available):
    g = golden(case)
    sim, s, _, rep = run_case(case, g)
    with s, tempfile.TemporaryDirectory() as td:
        S = sim.num_sds
        flags = m.OUT_REPLAY | m.OUT_ABSORBANCE | m.OUT_PATHLENGTH | m.OUT_AVERAGE_PL | m.OUT_BINARY
        s.write_outputs(td, str(Path(td) / "output.txt"), flags, 1.0, 1.0)
        for sds in range(1, S + 1):
            a0 = np.fromfile(Path(td) / f"A0_z_SDS_{sds}.bin", dtype=np.float32)
            assert np.array_equal(a0.view(np.uint32), g[f"A0_z_{sds}"].view(np.uint32))
            digest = hashlib.sha256((Path(td) / f"A_rz_SDS_{sds}.bin").read_bytes()).hexdigest()
            if digest != bytes(g[f"A_rz_sha_{sds}"]).decode():
                arz = np.fromfile(Path(td) / f"A_rz_SDS_{sds}.bin", dtype=np.float32)
                rs = arz.reshape(500, 1000).astype(np.float64).sum(axis=1)
                bad = np.nonzero(rs != g[f"A_rz_rowsum_{sds}"])[0]
                pytest.fail(f"A_rz SDS {sds} differs; rows {bad[:10]} nnz {np.count_nonzero(arz)}"
                            f" vs {int(g[f'A_rz_nnz_{sds}'])}")
            pl = np.fromfile(Path(td) / f"pathlength_SDS_{sds}.bin", dtype=np.float32)
            assert pl.tobytes() == g[f"rows_{sds}"].tobytes()
        avg = (Path(td) / "average_pathlength.txt").read_bytes()
        assert avg == bytes(g["average_pathlength_txt"])
        # output.txt: this library sums detected weights in float64, the
        # reference in float32 (error up to n * 2^-24 relative for n rows),
        # and both print 6 significant digits (up to 5e-6 relative).
        out = [float(v) for v in (Path(td) / "output.txt").read_text().split()]
        ref = [float(v) for v in bytes(g["output_txt"]).decode().split()]
        scale = 4294967295.0 * int(g["threads"])
        exact = [float(np.sum(g[f"rows_{s}"][:, 0].astype(np.float64))) / scale
                 for s in range(1, S + 1)]
        np.testing.assert_allclose(out, exact, rtol=5e-6, atol=0)
        for i in range(S):
            n = g[f"rows_{i + 1}"].shape[0]
            assert same_or_both_nan(out[i], ref[i], (n * 2.0 ** -24 + 1e-5) * abs(ref[i])), \
                (i, out[i], ref[i])
        for i in range(S):
            assert same_or_both_nan(rep.weight_sum[i], exact[i] * scale,
                                    1e-12 * abs(exact[i]) * scale), (i, rep.weight_sum[i])


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES)
def test_text_mode_files_match_reference(case, gpu_available):
    g = golden(case)
    sim, s, _, _ = run_case(case, g)
    with s, tempfile.TemporaryDirectory() as td:
        flags = m.OUT_REPLAY | m.OUT_ABSORBANCE | m.OUT_PATHLENGTH
        s.write_outputs(td, str(Path(td) / "output.txt"), flags, 1.0, 1.0)
        for sds in range(1, sim.num_sds + 1):
            for stem in ("pathlength_SDS_", "A_rz_SDS_", "A0_z_SDS_"):
                digest = hashlib.sha256((Path(td) / f"{stem}{sds}.txt").read_bytes()).hexdigest()
                assert digest == bytes(g[f"{stem}{sds}_txt_sha"]).decode(), f"{stem}{sds}.txt"


@pytest.mark.gpu
@pytest.mark.parametrize("case", STAT_CASES)
def test_reflectance_within_3_se_of_reference_at_4x_threads(case, gpu_available):
    """At N = 4 x threads the reference's photon split is timing-dependent;
    reflectance must agree within 3 combined standard errors."""
    g = golden(case)
    sim = load_case(case)
    N = int(g["stat_photons"])
    sim.number_photons = N
    with m.Simulation(sim, seed=int(g["seed"]) + 1, slots=int(g["threads"])) as s:
        r = s.run()
    ref_R = [float(v) for v in bytes(g["stat_output_txt"]).decode().split()]
    for i in range(sim.num_sds):
        se = r.std_error[i] * np.sqrt(2.0)  # both estimates carry the same SE
        assert same_or_both_nan(r.reflectance[i], ref_R[i], 3 * se + 1e-15), \
            (i, r.reflectance[i], ref_R[i], se)


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["fiber3", "ring5", "mismatch"])
@pytest.mark.parametrize("shape", [(64, 1), (128, 1), (128, 10), (256, 4), (256, 6)])
def test_rows_independent_of_launch_shape(case, shape, gpu_available):
    """Every compiled walk variant (block size x register cap) rounds the
    same way, so each reproduces the reference's rows bit for bit."""
    g = golden(case)
    sim = load_case(case)
    T = int(g["threads"])
    sim.number_photons = T
    block, minb = shape
    with m.Simulation(sim, seed=int(g["seed"]), slots=T, block_size=block,
                      blocks_per_sm=minb) as s:
        first = s.run()
        s.replay()
        assert [int(v) for v in first.detected[:sim.num_sds]] == [int(v) for v in g["detected"]]
        for sds in range(1, sim.num_sds + 1):
            rows, _ = s.rows(sds)
            assert rows.tobytes() == g[f"rows_{sds}"].tobytes(), f"SDS {sds}"


@pytest.mark.gpu
@pytest.mark.parametrize("case", STAT_CASES)
def test_reflectance_within_3_se_of_fp64_host_build(case, gpu_available):
    """The CUDA walk (FP32, XORWOW) against the FP64 host build of the same
    walk (the oracle: double precision throughout, its own PCG32 stream per
    photon) at 4 x threads photons each: per-SDS reflectance within 3
    combined standard errors, each side's SE from its per-photon
    detected-weight variance."""
    import oracle
    g = golden(case)
    sim = load_case(case)
    N = int(g["stat_photons"])
    sim.number_photons = N
    with m.Simulation(sim, seed=int(g["seed"]) + 3, slots=int(g["threads"])) as s:
        r = s.run()
    st, *_ = oracle.run(sim, N, 97, fp64=True)
    W = 4294967295.0
    for i in range(sim.num_sds):
        R64 = st.wsum[i] / (W * N)
        mean = st.wsum[i] / N
        se64 = np.sqrt(max(st.wsq[i] / N - mean * mean, 0.0) / (N - 1)) / W
        se = np.hypot(r.std_error[i], se64)
        assert same_or_both_nan(r.reflectance[i], R64, 3 * se + 1e-15), \
            (i, r.reflectance[i], R64, se)


def superset(case):
    p = GOLDEN_DIR / f"superset_{case}.npz"
    if not p.exists():
        pytest.fail(f"missing golden fixture {p}")
    return np.load(p)


SUPERSET_CASES = ["five_layer", "three_layer"]


@pytest.mark.gpu
@pytest.mark.parametrize("case", SUPERSET_CASES)
def test_benchmark_tissue_rows_of_reference_found_bit_exact(case, gpu_available):
    """The benchmark tissues with their three oblique fibres: config 1 (5
    layers, g = 0.9) at 1e9 photons, config 0 (3 layers, g = 0) at 1e10.
    The reference walked them on T threads (about N/T photons
    each; which thread takes the last photons depends on timing, but each
    thread's sequence of photons -- subsequence t, one photon after another
    -- does not).  This library walks the same T subsequences with 1.5 N/T
    photons each (slots = T), more than any reference thread walked, so:
      * every pathlength row the reference wrote is among this run's rows,
        bit for bit (weight, per-layer pathlengths, steps);
      * every detection of this run among the first N/(4T) photons of its
        slot -- photons every reference thread walked -- is among the
        reference's rows.
    This pins the multi-photon-per-slot walk (each photon starting where the
    previous one's draws ended) on the benchmark tissue itself."""
    g = superset(case)
    T, Nref, seed = int(g["threads"]), int(g["photons"]), int(g["seed"])
    q = -(-3 * Nref // (2 * T))
    sim = load_case(case)
    sim.number_photons = q * T
    matched = early = 0
    with m.Simulation(sim, seed=seed, slots=T) as s:
        s.run()
        s.replay()
        for sds in range(1, sim.num_sds + 1):
            rows, _ = s.rows(sds)
            ids, _ = s.detections(sds)
            assert rows.shape[0] == ids.size
            k = ids % q  # photon index within its slot (N = q*T: every slot has q)
            ours = {r.tobytes(): int(kk) for r, kk in zip(rows, k)}
            ref = g[f"rows_{sds}"]
            refset = {r.tobytes() for r in ref}
            missing = [i for i, r in enumerate(ref) if r.tobytes() not in ours]
            assert not missing, f"SDS {sds}: reference rows {missing[:5]} not found"
            matched += len(ref)
            for r, kk in zip(rows, k):
                if kk < Nref // (4 * T):
                    assert r.tobytes() in refset, f"SDS {sds}: photon {kk} of its slot missing"
                    early += 1
    assert matched >= 50, f"only {matched} reference rows to compare"
    assert early >= 5


@pytest.mark.gpu
@pytest.mark.parametrize("case", SUPERSET_CASES)
def test_benchmark_tissue_reflectance_within_3_se_of_reference(case, gpu_available):
    """The benchmark tissue at the reference's photon count with this
    library's own slot layout (the benchmark's): per-SDS reflectance within 3
    combined standard errors of the reference's output.txt."""
    g = superset(case)
    Nref = int(g["photons"])
    sim = load_case(case)
    sim.number_photons = Nref
    with m.Simulation(sim, seed=int(g["seed"]) + 7) as s:
        r = s.run()
    ref_R = [float(v) for v in bytes(g["output_txt"]).decode().split()]
    for i in range(sim.num_sds):
        se = r.std_error[i] * np.sqrt(2.0)
        assert abs(r.reflectance[i] - ref_R[i]) <= 3 * se + 1e-15, (i, r.reflectance[i], ref_R[i], se)
