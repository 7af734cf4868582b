"""Generates the golden fixtures of the parity tests from the reference itself.

Run on a machine with a B200 (the reference's thread count there is
148 x 2048 = 303104), after ``make -C oracle ref`` has built the
reference from its own sources into ``oracle/_ref``:

    python tests/golden/make_golden.py [--out tests/golden] [--cases fiber3,...]

For each case under ``configs/`` it runs the reference build with its
seed pinned through the ``time()`` shim (the reference seeds from
time(NULL) and has no seed option) and N equal to its thread count, where
every thread walks exactly one photon and the run is deterministic.  It
stores what the reference wrote: the detected counts, output.txt,
pathlength_SDS_#.bin rows, A0_z_SDS_#.bin, average_pathlength.txt,
digests of A_rz_SDS_#.bin and of the text-mode files.  It also stores,
for a few detected photons of each SDS, the first draws of their XORWOW
subsequence (generated with curand on the GPU through the library's test
entry point), so the CPU oracle can replay those photons with the
reference's own random numbers.  A second, nondeterministic run at 4x the
thread count gives the statistical fixture.  The reference's summary.json
of each run is stored too, for the drop-in test of the command line.

Superset fixtures (``--superset five_layer:1000000000,three_layer:10000000000``,
configs 1 and 0 of the benchmark, whose narrow fibres need that many
photons for detections): the reference
at N well above its thread count T, where each thread walks about N/T
photons and the split between threads depends on timing, but each
thread's sequence of photons does not.  The fixture keeps every
pathlength row the reference wrote; a run of this library with T slots of
more photons than any thread walked must contain each of them bit for
bit.

Cases: fiber3, ring5, mismatch, ringpt (this build's geometries), three_layer
(the 3-layer tissue with the README's fibres), surrogate (the 5-layer
benchmark tissue with ring detectors), hw8a and head_model (the inputs the
reference ships under example/HW8_A and example/head_model).
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import shutil
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402
import mcml_gpu_b200 as mcml  # noqa: E402

SEED = 20261203
PARITY_CASES = ["fiber3", "ring5", "mismatch", "ringpt", "three_layer", "surrogate", "hw8a",
                "head_model"]
SUPERSET_CASES = "five_layer:1000000000,three_layer:10000000000"
STREAM_PHOTONS_PER_SDS = 6


def sha(path: Path) -> str:
    return hashlib.sha256(path.read_bytes()).hexdigest()


def run_reference(case: str, photons: int, flags: list[str], workdir: Path, seed: int) -> Path:
    cfg = HERE / "configs" / case
    sim = json.loads((cfg / "sim_set.json").read_text())
    sim["number_photons"] = photons
    workdir.mkdir(parents=True, exist_ok=True)
    (workdir / "sim_set.json").write_text(json.dumps(sim, indent=2))
    shutil.copy(cfg / "input.txt", workdir / "input.txt")
    env = dict(os.environ)
    env["MCML_FIXED_TIME"] = str(seed)
    env["LD_PRELOAD"] = str(oracle.REF_SHIM)
    res = subprocess.run([str(oracle.REF_BIN), "sim_set.json", "input.txt", "output.txt", *flags],
                         cwd=workdir, env=env, capture_output=True, text=True, timeout=1800)
    (workdir / "stdout.txt").write_text(res.stdout + res.stderr)
    if res.returncode != 0:
        raise RuntimeError(f"reference failed on {case}: {res.returncode}\n{res.stdout[-2000:]}")
    return workdir


def summary_counts(path: Path) -> list[int]:
    txt = path.read_text()
    key = '"SDS_detected_number": ['
    i = txt.index(key) + len(key)
    j = txt.index("]", i)
    return [int(v.strip()) for v in txt[i:j].split(",")]


def superset_fixture(case: str, photons: int, T: int, out: Path, tmp: Path, seed: int) -> None:
    """The reference at `photons` >> T with -R -P -B: counts, output.txt,
    summary.json and every pathlength row, into superset_<case>.npz."""
    cfg = HERE / "configs" / case
    sim = mcml.parse_config(cfg / "sim_set.json", cfg / "input.txt")[0]
    L, S = int(sim.num_layers), int(sim.num_sds)
    wd = run_reference(case, photons, ["-R", "-P", "-B"], tmp / case / "superset", seed)
    fx: dict[str, np.ndarray] = {
        "seed": np.array(seed, dtype=np.uint64),
        "threads": np.array(T, dtype=np.uint64),
        "photons": np.array(photons, dtype=np.uint64),
        "detected": np.array(summary_counts(wd / "summary.json"), dtype=np.uint64),
        "output_txt": np.frombuffer((wd / "output.txt").read_bytes(), dtype=np.uint8),
        "summary_json": np.frombuffer((wd / "summary.json").read_bytes(), dtype=np.uint8),
    }
    for s in range(1, S + 1):
        fx[f"rows_{s}"] = np.fromfile(wd / f"pathlength_SDS_{s}.bin",
                                      dtype=np.float32).reshape(-1, L + 2)
    np.savez_compressed(out / f"superset_{case}.npz", **fx)
    print(f"superset {case} at {photons}: detected {list(fx['detected'])}", flush=True)


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=str(HERE))
    ap.add_argument("--cases", default=",".join(PARITY_CASES))
    ap.add_argument("--seed", type=int, default=SEED)
    ap.add_argument("--keep", default="")
    ap.add_argument("--superset", default=SUPERSET_CASES,
                    help="case:photons[,case:photons...]; empty to skip")
    args = ap.parse_args()
    out = Path(args.out)
    out.mkdir(parents=True, exist_ok=True)
    info = mcml.device_info(0)
    T = int(info.reference_threads)
    print(f"device {info.name.decode()} reference threads {T}", flush=True)
    tmp = Path(args.keep) if args.keep else Path(tempfile.mkdtemp(prefix="golden_"))
    for item in filter(None, args.superset.split(",")):
        case, photons = item.split(":")
        superset_fixture(case, int(float(photons)), T, out, tmp, args.seed + 2)
    for case in filter(None, args.cases.split(",")):
        cfg = HERE / "configs" / case
        sim = mcml.parse_config(cfg / "sim_set.json", cfg / "input.txt")[0]
        L, S = int(sim.num_layers), int(sim.num_sds)
        fx: dict[str, np.ndarray] = {}
        fx["seed"] = np.array(args.seed, dtype=np.uint64)
        fx["threads"] = np.array(T, dtype=np.uint64)
        # binary outputs
        wb = run_reference(case, T, ["-R", "-A", "-P", "-AP", "-B"], tmp / case / "bin", args.seed)
        counts = summary_counts(wb / "summary.json")
        fx["detected"] = np.array(counts, dtype=np.uint64)
        fx["output_txt"] = np.frombuffer((wb / "output.txt").read_bytes(), dtype=np.uint8)
        fx["summary_json"] = np.frombuffer((wb / "summary.json").read_bytes(), dtype=np.uint8)
        fx["average_pathlength_txt"] = np.frombuffer(
            (wb / "average_pathlength.txt").read_bytes(), dtype=np.uint8)
        for s in range(1, S + 1):
            rows = np.fromfile(wb / f"pathlength_SDS_{s}.bin", dtype=np.float32).reshape(-1, L + 2)
            fx[f"rows_{s}"] = rows
            fx[f"A0_z_{s}"] = np.fromfile(wb / f"A0_z_SDS_{s}.bin", dtype=np.float32)
            arz = np.fromfile(wb / f"A_rz_SDS_{s}.bin", dtype=np.float32)
            fx[f"A_rz_sha_{s}"] = np.frombuffer(sha(wb / f"A_rz_SDS_{s}.bin").encode(), np.uint8)
            fx[f"A_rz_rowsum_{s}"] = arz.reshape(500, 1000).astype(np.float64).sum(axis=1)
            fx[f"A_rz_nnz_{s}"] = np.array(int(np.count_nonzero(arz)), dtype=np.uint64)
        # text outputs
        wt = run_reference(case, T, ["-R", "-A", "-P"], tmp / case / "txt", args.seed)
        for s in range(1, S + 1):
            for stem in ("pathlength_SDS_", "A_rz_SDS_", "A0_z_SDS_"):
                p = wt / f"{stem}{s}.txt"
                fx[f"{stem}{s}_txt_sha"] = np.frombuffer(sha(p).encode(), np.uint8)
            head = b"".join((wt / f"pathlength_SDS_{s}.txt").read_bytes().splitlines(True)[:20])
            fx[f"pathlength_SDS_{s}_txt_head"] = np.frombuffer(head, dtype=np.uint8)
        fx["output_txt_textmode"] = np.frombuffer((wt / "output.txt").read_bytes(), np.uint8)
        fx["summary_json_textmode"] = np.frombuffer((wt / "summary.json").read_bytes(), np.uint8)
        # draws of a few detected photons, located with the library at N == T
        sim.number_photons = T
        with mcml.Simulation(sim, seed=args.seed, slots=T) as run:
            run.run()
            for s in range(1, S + 1):
                ids, _ = run.detections(s)
                fx[f"ids_{s}"] = ids
                rows = fx[f"rows_{s}"]
                take = min(STREAM_PHOTONS_PER_SDS, ids.size, rows.shape[0])
                for k in range(take):
                    steps = int(rows[k, L + 1]) if rows.shape[0] > k else 2000
                    count = steps * 5 + 256
                    fx[f"stream_{s}_{k}"] = mcml.uniform_stream(args.seed, int(ids[k]), count)
                    fx[f"stream_{s}_{k}_id"] = np.array(int(ids[k]), dtype=np.uint64)
        # statistical run: 4x the thread count (nondeterministic photon split)
        ws = run_reference(case, 4 * T, ["-R", "-AP"], tmp / case / "stat", args.seed + 1)
        fx["stat_photons"] = np.array(4 * T, dtype=np.uint64)
        fx["stat_detected"] = np.array(summary_counts(ws / "summary.json"), dtype=np.uint64)
        fx["stat_output_txt"] = np.frombuffer((ws / "output.txt").read_bytes(), np.uint8)
        np.savez_compressed(out / f"golden_{case}.npz", **fx)
        print(f"{case}: detected {counts} stat {list(fx['stat_detected'])}", flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
