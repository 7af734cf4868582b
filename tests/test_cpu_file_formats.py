"""The reference's output files, written on the host from host arrays
(mcml_write_host_outputs), against a Python restatement of the reference's
writers (io.cpp:11-33, 281-469) and of its average-pathlength reduction
(transport.cu:274-297).  No GPU: the inputs are synthetic detections, rows
and u64 tallies of the shapes a run produces.

Text values follow iostream's default formatting, which is printf's %g
(6 significant digits); Python's '%g' is the same conversion.  Binary files
hold float32.  Absorbance scales are evaluated in double in the reference's
order, with PI and the grid steps being float constants.
"""
import ctypes as C
import json
import math
from pathlib import Path

import numpy as np
import pytest

from conftest import load_case

PI_F = float(np.float32(3.141592654))  # header.h:40, a float literal


def _fmt(v) -> str:
    return "%g" % float(v)


def _synthetic(sim, seed, nr, nz):
    rng = np.random.default_rng(seed)
    S, L = int(sim.num_sds), int(sim.num_layers)
    rows = []
    for s in range(S):
        n = [7, 0, 3, 5][s % 4]
        r = (rng.random((n, L + 2)) * 3).astype(np.float32)
        r[:, 0] = rng.integers(1, 2**32 - 1, n).astype(np.float32)  # weights in quanta
        r[:, L + 1] = rng.integers(1, 10000, n).astype(np.float32)  # steps
        rows.append(np.ascontiguousarray(r))
    a_rz = rng.integers(0, 2**45, (S, nz, nr), dtype=np.uint64)
    a_rz[0, 0, :3] = 0
    a0_z = rng.integers(0, 2**45, (S, nz), dtype=np.uint64)
    return rows, a_rz, a0_z


def _write(sim, photons, rows, a_rz, a0_z, wsum, grid, d: Path, flags, sim_s, replay_s, gpu):
    import mcml_gpu_b200 as m
    lib = m.load_library()
    S = int(sim.num_sds)
    det = np.array([len(r) for r in rows], np.uint64)
    ptrs = (C.c_void_p * S)(*[r.ctypes.data for r in rows])
    h = m.HostData()
    h.photons = photons
    h.detected = det.ctypes.data
    h.weight_sum = wsum.ctypes.data
    h.rows = C.cast(ptrs, C.c_void_p)
    h.A_rz, h.A0_z = a_rz.ctypes.data, a0_z.ctypes.data
    h.grid_nr, h.grid_nz, h.grid_dr, h.grid_dz = grid
    h.gpu_name = gpu.encode()
    rc = lib.mcml_write_host_outputs(C.byref(sim), C.byref(h), str(d).encode(),
                                     str(d / "output.txt").encode(), flags, sim_s, replay_s)
    assert rc == 0, lib.mcml_last_error()


def _scale2(scale1, r, dr, dz):
    # io.cpp:400 / 447: scale1 * 2 * PI*(r + 0.5)*record_dr*record_dr*record_dz
    dr, dz = float(np.float32(dr)), float(np.float32(dz))
    return scale1 * 2 * PI_F * (r + 0.5) * dr * dr * dz


@pytest.mark.parametrize("case", ["ring5", "fiber3"])
def test_host_writer_matches_the_reference_formats(case, tmp_path):
    import mcml_gpu_b200 as m
    sim = load_case(case)
    S, L = int(sim.num_sds), int(sim.num_layers)
    nr, nz, dr, dz = 9, 4, 0.01, 0.02
    photons = 12_345_678
    rows, a_rz, a0_z = _synthetic(sim, 5, nr, nz)
    wsum = np.array([math.fsum(r[:, 0].astype(np.float64)) for r in rows])
    scale1 = float(0xFFFFFFFF) * float(photons)
    everything = m.OUT_REPLAY | m.OUT_ABSORBANCE | m.OUT_PATHLENGTH | m.OUT_AVERAGE_PL
    text_dir, bin_dir = tmp_path / "text", tmp_path / "bin"
    text_dir.mkdir()
    bin_dir.mkdir()
    # text files open in append mode: two writes give two copies
    for _ in range(2):
        _write(sim, photons, rows, a_rz, a0_z, wsum, (nr, nz, dr, dz), text_dir, everything,
               1.5, 0.25, "B200 test")
    _write(sim, photons, rows, a_rz, a0_z, wsum, (nr, nz, dr, dz), bin_dir,
           everything | m.OUT_BINARY, 1.5, 0.25, "B200 test")

    # output.txt (io.cpp:11-33): R_s = sum W / (0xFFFFFFFF N), each followed by ' '
    line = "".join(_fmt(w / scale1) + " " for w in wsum) + "\n"
    assert (text_dir / "output.txt").read_text() == line * 2

    for s in range(S):
        # pathlength rows (io.cpp:302-323): float32 rows; text: value '\t' ... '\n'
        assert (bin_dir / f"pathlength_SDS_{s + 1}.bin").read_bytes() == rows[s].tobytes()
        txt = "".join("".join(_fmt(v) + "\t" for v in row) + "\n" for row in rows[s])
        assert (text_dir / f"pathlength_SDS_{s + 1}.txt").read_text() == txt * 2

        # A_rz (io.cpp:383-434): [z][r], divided by the ring volume of r
        vals = [[int(a_rz[s, z, r]) / _scale2(scale1, r, dr, dz) for r in range(nr)]
                for z in range(nz)]
        want_bin = np.array(vals, np.float64).astype(np.float32).tobytes()
        assert (bin_dir / f"A_rz_SDS_{s + 1}.bin").read_bytes() == want_bin
        txt = "".join("".join(_fmt(v) + "\t" for v in row) + "\n" for row in vals)
        assert (text_dir / f"A_rz_SDS_{s + 1}.txt").read_text() == txt * 2

        # A0_z (io.cpp:436-469): r = 0 volume, one value per line in text
        v0 = [int(a0_z[s, z]) / _scale2(scale1, 0, dr, dz) for z in range(nz)]
        assert (bin_dir / f"A0_z_SDS_{s + 1}.bin").read_bytes() == \
            np.array(v0, np.float64).astype(np.float32).tobytes()
        assert (text_dir / f"A0_z_SDS_{s + 1}.txt").read_text() == \
            "".join(_fmt(v) + "\n" for v in v0) * 2

    # average_pathlength.txt (transport.cu:274-297, io.cpp:331-343)
    inv_w = float(np.float32(1) / np.float32(m.derive(sim).start_weight))
    parts = []
    for s in range(S):
        for l in range(1, L + 1):
            changed = 0.001 * float(np.float32(sim.mua[l - 1]))
            a = b = 0.0
            for row in rows[s]:
                e = float(row[0]) * inv_w
                a += e
                e *= math.exp(-1 * changed * float(row[l]))
                b += e
            parts.append(_fmt(math.log(a / b) / changed) if b else None)
    got = (text_dir / "average_pathlength.txt").read_text().split("\n")
    assert got[2] == "" and got[0] == got[1]
    fields = got[0].split("\t")
    assert fields[-1] == "" and len(fields) == S * L + 1
    for want, have in zip(parts, fields):
        if want is not None:  # an SDS without rows gives 0/0, printed as nan
            assert have == want
        else:
            assert "nan" in have

    # summary.json (io.cpp:345-381): keys in the reference's order
    text = (bin_dir / "summary.json").read_text()
    d = json.loads(text)
    assert list(d) == ["MCML_version_K", "num_photon", "sim_time", "replay_time",
                       "sim_speed(photons/s)", "sim_GPU", "each_photon_weight",
                       "number_layers", "detect_mode", "num_SDS", "SDS_detected_number"]
    assert d["MCML_version_K"] == 3.02 and d["num_photon"] == photons
    assert d["sim_time"] == 1.5 and d["replay_time"] == 0.25
    assert f'"sim_speed(photons/s)": {_fmt(photons / 1.75)},' in text
    assert f'"each_photon_weight": {_fmt(scale1)},' in text
    assert d["sim_GPU"] == "B200 test" and d["number_layers"] == L and d["num_SDS"] == S
    assert d["detect_mode"] == ("fiber" if sim.source_probe_oblique else "ring")
    assert d["SDS_detected_number"] == [len(r) for r in rows]
    assert '"SDS_detected_number": [ ' + " , ".join(str(len(r)) for r in rows) + " ]\n}" in text


def test_large_text_file_keeps_row_order_across_write_rounds(tmp_path):
    """A pathlength text file is formatted in rounds of up to 32 threads x
    4 MB and written while the next round is formatted.  With 2.5e6 rows
    (several rounds on any host) the file must equal the rows formatted in
    order, twice after two appends; the single-threaded row formatter of the
    library gives the expected bytes."""
    import mcml_gpu_b200 as m
    lib = m.load_library()
    sim = load_case("ring5")
    S, L = int(sim.num_sds), int(sim.num_layers)
    rng = np.random.default_rng(11)
    n = 2_500_000
    big = (rng.random((n, L + 2)) * 5).astype(np.float32)
    big[:, 0] = np.arange(1, n + 1, dtype=np.float32)  # row order is visible
    rows = [big] + [np.zeros((0, L + 2), np.float32) for _ in range(S - 1)]
    a_rz = np.zeros((S, 2, 2), np.uint64)
    a0_z = np.zeros((S, 2), np.uint64)
    wsum = np.zeros(S)
    for _ in range(2):
        _write(sim, 10**8, rows, a_rz, a0_z, wsum, (2, 2, 0.01, 0.01), tmp_path,
               m.OUT_REPLAY | m.OUT_PATHLENGTH, 1.0, 1.0, "")
    need = C.c_uint64(0)
    assert lib.mcml_format_rows_text(big.ctypes.data, n, L + 2, None, 0, C.byref(need)) == 0
    want = C.create_string_buffer(need.value)
    assert lib.mcml_format_rows_text(big.ctypes.data, n, L + 2, want, need.value,
                                     C.byref(need)) == 0
    got = (tmp_path / "pathlength_SDS_1.txt").read_bytes()
    assert len(got) == 2 * need.value
    assert got == want.raw * 2
    assert (tmp_path / "pathlength_SDS_2.txt").read_bytes() == b""
