"""The command line as a drop-in for the reference's binary.

For every golden case, `MCML_GPU sim_set.json input.txt output.txt` runs in
a fresh directory with the reference's flags and N equal to the
reference's thread count T, seeded like the golden run (-S, -T: this
library's additive flags for what the reference takes from time(NULL) and
its launch shape).  Every file the reference wrote must come out the same
(io.cpp:11-33, 258-469):
  * pathlength_SDS_#.bin, A0_z_SDS_#.bin, average_pathlength.txt byte for
    byte, A_rz_SDS_#.bin and the text-mode files by SHA-256;
  * output.txt within the reference's float32 summation error (it sums
    detected weights in float, this library in double);
  * summary.json line by line in the reference's key order, the timing
    values (sim_time, replay_time, sim_speed) masked.
"""
import hashlib
import json
import math
import subprocess
from pathlib import Path

import numpy as np
import pytest

from conftest import CONFIGS, GOLDEN

import mcml_gpu_b200 as m

CLI = Path(m.__file__).resolve().parent / "bin" / "MCML_GPU"
CASES = ["fiber3", "ring5", "mismatch", "ringpt", "three_layer", "surrogate", "hw8a",
         "head_model"]
TIME_KEYS = ('"sim_time"', '"replay_time"', '"sim_speed(photons/s)"')


def golden(case):
    p = GOLDEN / f"golden_{case}.npz"
    if not p.exists():
        pytest.fail(f"missing golden fixture {p}")
    return np.load(p)


def run_cli(d: Path, case: str, T: int, seed: int, flags: list) -> None:
    conf = json.loads((CONFIGS / case / "sim_set.json").read_text())
    conf["number_photons"] = T
    d.mkdir(parents=True, exist_ok=True)
    (d / "sim_set.json").write_text(json.dumps(conf, indent=2))
    (d / "input.txt").write_text((CONFIGS / case / "input.txt").read_text())
    r = subprocess.run([str(CLI), "sim_set.json", "input.txt", "output.txt", *flags,
                        "-S", str(seed), "-T", str(T)], cwd=d, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr


def summary_lines(text: str) -> list:
    out = []
    for ln in text.splitlines():
        key = ln.split(":", 1)[0]
        out.append(key + ": <time>" if key in TIME_KEYS else ln)
    return out


def sha(p: Path) -> str:
    return hashlib.sha256(p.read_bytes()).hexdigest()


def floats_match(ours: list, ref: list, rows: list) -> None:
    assert len(ours) == len(ref)
    for i, (a, b) in enumerate(zip(ours, ref)):
        if math.isnan(b):
            assert math.isnan(a), (i, a, b)
            continue
        n = rows[i]
        assert abs(a - b) <= (n * 2.0 ** -24 + 1e-5) * abs(b), (i, a, b)


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES)
def test_cli_binary_outputs_match_reference(case, tmp_path, gpu_available):
    g = golden(case)
    if "summary_json" not in g.files:
        pytest.fail(f"golden_{case}.npz predates the stored summary.json")
    T, seed = int(g["threads"]), int(g["seed"])
    run_cli(tmp_path, case, T, seed, ["-R", "-A", "-P", "-AP", "-B"])
    S = len(g["detected"])
    for s in range(1, S + 1):
        assert (tmp_path / f"pathlength_SDS_{s}.bin").read_bytes() == g[f"rows_{s}"].tobytes()
        assert (tmp_path / f"A0_z_SDS_{s}.bin").read_bytes() == g[f"A0_z_{s}"].tobytes()
        assert sha(tmp_path / f"A_rz_SDS_{s}.bin") == bytes(g[f"A_rz_sha_{s}"]).decode()
    assert (tmp_path / "average_pathlength.txt").read_bytes() == bytes(g["average_pathlength_txt"])
    ours = [float(v) for v in (tmp_path / "output.txt").read_text().split()]
    ref = [float(v) for v in bytes(g["output_txt"]).decode().split()]
    floats_match(ours, ref, [g[f"rows_{s}"].shape[0] for s in range(1, S + 1)])
    assert summary_lines((tmp_path / "summary.json").read_text()) == \
        summary_lines(bytes(g["summary_json"]).decode())


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES)
def test_cli_text_outputs_match_reference(case, tmp_path, gpu_available):
    g = golden(case)
    if "summary_json_textmode" not in g.files:
        pytest.fail(f"golden_{case}.npz predates the stored summary.json")
    T, seed = int(g["threads"]), int(g["seed"])
    run_cli(tmp_path, case, T, seed, ["-R", "-A", "-P"])
    S = len(g["detected"])
    for s in range(1, S + 1):
        for stem in ("pathlength_SDS_", "A_rz_SDS_", "A0_z_SDS_"):
            assert sha(tmp_path / f"{stem}{s}.txt") == bytes(g[f"{stem}{s}_txt_sha"]).decode(), \
                f"{stem}{s}.txt"
    ours = [float(v) for v in (tmp_path / "output.txt").read_text().split()]
    ref = [float(v) for v in bytes(g["output_txt_textmode"]).decode().split()]
    floats_match(ours, ref, [g[f"rows_{s}"].shape[0] for s in range(1, S + 1)])
    assert summary_lines((tmp_path / "summary.json").read_text()) == \
        summary_lines(bytes(g["summary_json_textmode"]).decode())
    # -R -P (no -AP): the reference writes no average_pathlength.txt
    assert not (tmp_path / "average_pathlength.txt").exists()
