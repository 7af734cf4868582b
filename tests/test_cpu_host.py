"""Host-side logic without a GPU: the C ABI's exports, the configuration
reader (read_mua_mus, io.cpp:35-256), the derived constants
(io.cpp:168-238), the CLI's flag rules (main.cu:31-100) and the errors a
caller gets without a device."""
import json
import math
import re
import subprocess
import tempfile
from pathlib import Path

import numpy as np
import pytest

from conftest import CONFIGS, ROOT, load_case

import mcml_gpu_b200 as m

HEADER = ROOT / "include" / "mcml_b200.h"
CLI = ROOT / "mcml_gpu_b200" / "bin" / "MCML_GPU"


def declared_entry_points():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"\b(mcml_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_entry_point():
    lib = m.load_library()
    names = declared_entry_points()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    # the Python bindings cover the whole header
    from mcml_gpu_b200 import surrogate, wmc
    assert set(names) == set(m.exported_symbols()) | set(wmc.BOUND) | set(surrogate.BOUND)


def test_version_and_strerror():
    lib = m.load_library()
    assert b"K3.02" in lib.mcml_version()
    assert lib.mcml_strerror(-4) == b"detection record buffer overflow"
    assert lib.mcml_strerror(0) == b"ok"


def test_parse_reference_example():
    sim = load_case("three_layer")
    assert sim.num_layers == 3 and sim.num_sds == 3
    assert sim.number_photons == 1000000
    assert sim.source_probe_oblique == 1 and sim.detector_probe_oblique == 1
    np.testing.assert_array_equal(np.array(sim.mua[:3], np.float32),
                                  np.array([0.3201, 0.2954, 0.2747], np.float32))
    assert np.float32(sim.det_pos[1]) == np.float32(1.5)


def test_derived_constants():
    sim = load_case("three_layer")
    d = m.derive(sim)
    # Fresnel start weight at normal incidence, 1.457 -> 1.4 (io.cpp:230-237)
    r = ((1.457 - 1.4) / (1.457 + 1.4)) ** 2
    n0, n1 = float(np.float32(1.457)), float(np.float32(1.4))
    r = ((n0 - n1) / (n0 + n1)) ** 2
    assert d.start_weight == np.float32(int(0xFFFFFFFF * (1 - r)))
    # layer stack with the 10 cm floor (io.cpp:107, 210-225)
    assert np.float32(d.z_min[1]) == 0.0 and np.float32(d.z_max[1]) == np.float32(0.27)
    assert np.float32(d.z_max[3]) == np.float32(10.0)
    # 1/(mua+mus) in float
    assert np.float32(d.mutr[1]) == np.float32(1.0) / (np.float32(0.3201) + np.float32(35.2861))
    # critical angle asin(NA/upper_n) (io.cpp:196)
    assert abs(d.critical_angle[1] - math.asin(0.13 / 1.457)) < 1e-6


def _write_case(td, sim_json, input_txt):
    (Path(td) / "s.json").write_text(json.dumps(sim_json))
    (Path(td) / "in.txt").write_text(input_txt)
    return Path(td) / "s.json", Path(td) / "in.txt"


BASE = json.loads((CONFIGS / "three_layer" / "sim_set.json").read_text())
GOOD_INPUT = (CONFIGS / "three_layer" / "input.txt").read_text()


@pytest.mark.parametrize("edit,text,message", [
    ({"source_probe_oblique": 2}, GOOD_INPUT, "source_probe_oblique: 2is not 1 or 0!"),
    ({"detector_reflectance": 1.5}, GOOD_INPUT, "Detector reflectance: 1.5 is out of range !"),
    ({"number_layers": 11}, GOOD_INPUT, "Number of layer is too large!"),
    ({"probes": dict(BASE["probes"], num_SDS=2)}, GOOD_INPUT,
     "Number of SDS : 2 not match the probe setting : 3 !"),
    ({}, "0.27 0.3 35 1.4 0 0.65 0.3 30 1.4 0 0.27 0 1.4 0", "Mus for simulation 0 layer 2"),
    ({}, "0.27 0.3 35 1.4 0 0.65 0.3 30 1.4 0 0.27 130 1.0 0", "n for simulation 0 layer 2"),
    ({}, "0.27 0.3 35 1.4 0 0.65 0.3 30 1.4 0 0.27 130 1.4 1.5", "g for simulation 0 layer 2"),
    ({}, "0.27 0.3 35", "Mus for simulation 0 layer 2 Error with value 0 !"),
])
def test_config_errors_carry_reference_messages(edit, text, message):
    with tempfile.TemporaryDirectory() as td:
        sj, it = _write_case(td, dict(BASE, **edit), text)
        with pytest.raises(m.MCMLError) as e:
            m.parse_config(sj, it)
        assert message in e.value.message


def test_multi_simulation_file():
    with tempfile.TemporaryDirectory() as td:
        sj, it = _write_case(td, dict(BASE, number_simulation=2),
                             GOOD_INPUT.strip() + "\n" + GOOD_INPUT.replace("0.3201", "0.5"))
        sims = m.parse_config(sj, it)
        assert len(sims) == 2
        assert np.float32(sims[1].mua[0]) == np.float32(0.5)


def test_create_without_gpu_fails_cleanly():
    if m.device_count() > 0:
        pytest.skip("a GPU is present")
    sim = load_case("three_layer")
    with pytest.raises(m.MCMLError) as e:
        m.Simulation(sim)
    assert e.value.status == -9  # MCML_E_NODEV


def test_invalid_sim_rejected_before_device_use():
    sim = load_case("three_layer")
    sim.num_layers = 11
    with pytest.raises(m.MCMLError) as e:
        m.Simulation(sim)
    assert e.value.status == -1


def run_cli(*args, cwd=None):
    return subprocess.run([str(CLI), *args], capture_output=True, text=True, cwd=cwd, timeout=60)


def test_cli_usage_and_flag_rules():
    r = run_cli()
    assert r.returncode == 0 and "Usage:" in r.stderr
    sj, it = CONFIGS / "three_layer" / "sim_set.json", CONFIGS / "three_layer" / "input.txt"
    for flags, msg in [(["-P"], "-P option only work with -R option!"),
                       (["-A"], "-A option only work with -R option!"),
                       (["-AP"], "-AP option only work with -R option!"),
                       (["-R", "-B"], None),
                       (["-B"], "-B option only work with -P or -A option!"),
                       (["-batch", "-R"], "-batch option does not work with -R or -CK option!"),
                       (["-batch", "-CK", "x.ckpt"],
                        "-batch option does not work with -R or -CK option!")]:
        r = run_cli(str(sj), str(it), "out.txt", *flags, cwd=tempfile.gettempdir())
        if msg:
            assert r.returncode == 0 and msg in r.stdout, (flags, r.stdout)
    r = run_cli(str(sj), str(it), "out.txt", "-G", "-1")
    assert r.returncode == 0 and "GPU selection ERROR!" in r.stdout


@pytest.mark.parametrize("flags,msg", [
    (["-S", "12ab"], "-S option needs a seed"),
    (["-S", "-5"], "-S option needs a seed"),
    (["-S"], "-S option needs a seed"),
    (["-T", "many"], "-T option needs a slot count"),
    (["-grid", "200", "200", "0.005"], "-grid option needs nr nz dr dz"),
    (["-grid", "0", "200", "0.005", "0.005"], "-grid option needs nr nz dr dz"),
    (["-grid", "200", "200", "-0.005", "0.005"], "-grid option needs nr nz dr dz"),
    (["-grid", "200", "200", "0.005", "x"], "-grid option needs nr nz dr dz"),
    (["-R", "-CK"], "-CK option needs a checkpoint file name"),
])
def test_cli_rejects_malformed_option_values(flags, msg, tmp_path):
    """This CLI's own options (-S, -T, -grid, -CK) report a malformed or
    missing value, before any configuration is read or GPU used."""
    sj, it = CONFIGS / "three_layer" / "sim_set.json", CONFIGS / "three_layer" / "input.txt"
    r = run_cli(str(sj), str(it), "out.txt", *flags, cwd=str(tmp_path))
    assert r.returncode == 0 and msg in r.stdout, (flags, r.stdout)
    assert not any(tmp_path.iterdir())


def test_cli_bad_config_exits_1():
    with tempfile.TemporaryDirectory() as td:
        sj, it = _write_case(td, dict(BASE, detector_reflectance=2.0), GOOD_INPUT)
        r = run_cli(str(sj), str(it), "out.txt", cwd=td)
        assert r.returncode == 1
        assert "Something wrong with read_simulation_data!" in r.stdout


def _fnv1a(data: bytes, h: int = 14695981039346656037) -> int:
    for b in data:
        h = ((h ^ b) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    return h


def _checkpoint_bytes(records: bytes, **f) -> bytes:
    import struct
    n = len(records) // 40
    head = b"MCMLCKP1" + struct.pack("<II", 1, 40) + struct.pack(
        "<10Q", f.get("digest", 7), f.get("seed", 5), 0, f.get("photons", 1000),
        f.get("slots", 100), f.get("done", 40), n, f.get("steps", 123456), f.get("launches", 2),
        _fnv1a(records))
    return head + struct.pack("<Q", _fnv1a(head)) + bytes(24) + records


def test_checkpoint_header_is_checked_on_the_host(tmp_path):
    """The checkpoint layout documented in include/mcml_b200.h, written by
    hand: read back field by field; a damaged header, a truncated record
    area or another file is rejected with MCML_E_CHECKPOINT."""
    import mcml_gpu_b200 as m
    recs = bytes(range(200)) * 2  # ten 40-byte records
    p = tmp_path / "a.ckpt"
    p.write_bytes(_checkpoint_bytes(recs, seed=99, done=60, launches=3))
    info = m.checkpoint_info(p)
    assert (info.seed, info.photons, info.slots, info.slots_done, info.records, info.steps,
            info.launches) == (99, 1000, 100, 60, 10, 123456, 3)
    good = p.read_bytes()
    bad = [good[:8] + bytes([2]) + good[9:],          # version
           good[:30] + bytes([good[30] ^ 1]) + good[31:],  # header digest
           good[:-1],                                  # truncated records
           b"not a checkpoint" + good[16:]]
    for b in bad:
        p.write_bytes(b)
        with pytest.raises(m.MCMLError) as e:
            m.checkpoint_info(p)
        assert e.value.status == -10
    p.write_bytes(_checkpoint_bytes(recs, done=101))  # slots_done beyond slots
    with pytest.raises(m.MCMLError) as e:
        m.checkpoint_info(p)
    assert e.value.status == -10
    with pytest.raises(m.MCMLError) as e:
        m.checkpoint_info(tmp_path / "missing.ckpt")
    assert e.value.status == -5


def test_row_text_matches_iostream_default_format():
    """pathlength_SDS_#.txt text: every float as iostream prints it by
    default (printf "%g", 6 significant digits), tab after each value,
    newline after each row -- checked against Python's %g over random bit
    patterns of every float class and the values rows really hold."""
    import mcml_gpu_b200 as m
    rng = np.random.default_rng(3)
    bits = rng.integers(0, 2**32, size=(20000, 7), dtype=np.uint64).astype(np.uint32)
    rows = bits.view(np.float32).copy()
    rows[np.isnan(rows)] = 1.5
    special = np.array([[0.0, -0.0, np.inf, -np.inf, 4294967295.0, 1e-45, 3.4028235e38],
                        [123456.5, 999999.5, 9999995.0, 0.0001, 1e-5, 100000.0, 1e6]],
                       np.float32)
    rows = np.vstack([rows, special])
    want = "".join("".join("%g\t" % float(v) for v in r) + "\n" for r in rows).encode()
    assert m.format_rows_text(rows) == want
    assert m.format_rows_text(np.zeros((0, 7), np.float32)) == b""


def test_device_tensor_checks_reject_host_memory():
    """Tensors handed to kernels must be CUDA tensors: a host tensor's
    address would be read by the GPU as a device address."""
    import torch
    from mcml_gpu_b200 import _device_ptr
    with pytest.raises(TypeError):
        _device_ptr(np.zeros((4, 25), np.float32), "X", device=0)
    with pytest.raises(ValueError, match="cuda:0"):
        _device_ptr(torch.zeros((4, 25)), "X", device=0, shape=(None, 25))
