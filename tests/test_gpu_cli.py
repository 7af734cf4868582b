"""The command line's additive modes on the GPU: a checkpointed first pass
(-CK) writes the same output.txt and pathlength rows as a plain run with
the same seed and slots, also when resumed from a checkpoint left by an
interrupted run; -batch walks every simulation of a multi-simulation file
in one launch and appends one output.txt line per simulation."""
import json
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from conftest import CONFIGS, load_case

import mcml_gpu_b200 as m

CLI = Path(m.__file__).resolve().parent / "bin" / "MCML_GPU"


def cli(cwd, *args):
    r = subprocess.run([str(CLI), "sim_set.json", "input.txt", "output.txt", *args], cwd=cwd,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    return r


def setup_case(d, case, photons, n_sims=1):
    conf = json.loads((CONFIGS / case / "sim_set.json").read_text())
    conf["number_photons"] = photons
    conf["number_simulation"] = n_sims
    (d / "sim_set.json").write_text(json.dumps(conf))
    line = (CONFIGS / case / "input.txt").read_text().strip().splitlines()[0]
    rows = [line]
    for k in range(1, n_sims):  # more tissues: scale the absorption of every layer
        vals = line.split()
        L = conf["number_layers"]
        for l in range(L):
            i = 5 * l + 1 if l < L - 1 else 5 * (L - 1)
            vals[i] = "%.6g" % (float(vals[i]) * (1 + 0.5 * k))
        rows.append("\t".join(vals))
    (d / "input.txt").write_text("\n".join(rows) + "\n")


@pytest.mark.gpu
def test_cli_checkpointed_run_matches_plain_run(tmp_path, gpu_available):
    a, b = tmp_path / "plain", tmp_path / "ck"
    a.mkdir()
    b.mkdir()
    for d in (a, b):
        setup_case(d, "ring5", 600_000)
    flags = ["-S", "77", "-T", "60000", "-R", "-P", "-B"]
    cli(a, *flags)
    # an interrupted checkpointed run leaves a partial checkpoint; the CLI resumes it
    sim = m.parse_config(b / "sim_set.json", b / "input.txt")[0]
    with m.Simulation(sim, seed=77, slots=60000) as run:
        assert run.run_checkpointed(b / "walk.ckpt", chunk_slots=15000, max_chunks=1) is None
    assert m.checkpoint_info(b / "walk.ckpt").slots_done == 15000
    cli(b, *flags, "-CK", "walk.ckpt")
    assert m.checkpoint_info(b / "walk.ckpt").slots_done == 60000
    want = [float(v) for v in (a / "output.txt").read_text().split()]
    got = [float(v) for v in (b / "output.txt").read_text().split()]
    np.testing.assert_allclose(got, want, rtol=1e-12)
    for s in (1, 2, 3):
        name = f"pathlength_SDS_{s}.bin"
        assert (a / name).read_bytes() == (b / name).read_bytes()


@pytest.mark.gpu
def test_cli_batch_writes_one_line_per_simulation(tmp_path, gpu_available):
    setup_case(tmp_path, "ring5", 300_000, n_sims=3)
    r = cli(tmp_path, "-S", "5", "-batch")
    lines = (tmp_path / "output.txt").read_text().strip().splitlines()
    assert len(lines) == 3
    R = np.array([[float(v) for v in ln.split()] for ln in lines])
    assert np.all(R > 0)
    # more absorption, less reflectance
    assert np.all(R[0] > R[1]) and np.all(R[1] > R[2])
    assert (tmp_path / "summary.json").read_text().count('"MCML_version_K"') == 3
