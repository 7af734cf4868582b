#!/usr/bin/env python
"""Throughput of the MCML photon-transport hot path on B200.

One step = one pass of the hot path over the 5-layer benchmark tissue
(tests/golden/configs/five_layer: heights 0.3/0.7/0.2/0.4/semi-infinite cm,
mua ~ U(0.05,0.5)/cm, mus ~ U(50,250)/cm drawn by seed, g=0.9, n=1.4,
three oblique fibres at 0.8/1.5/3.0 cm): walk 1e8 photons, then replay
every detected photon with per-layer pathlengths and the A_rz / A0_z
tallies (the reference's `-R -A -B` path).  Metric: photons/s.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl mcml|reference]

`value` times the device pipeline with inputs resident (CUDA events on the
launching stream, L2 flushed between steps); `e2e` times the same work
through the public API from host structs to host result buffers.  The
reference arm (`--impl reference`) times the CPU restatement of the
reference algorithm (the reference has no CPU implementation) on all host
cores over a bounded photon sample; it loads the oracle only, never this
library.  Under torchrun each rank walks its own subsequence range (weak
scaling) and rank 0 prints one JSON line.

Beside the timed region, the line carries two baselines: `cpu_baseline`
(the CPU restatement on the host cores) and `reference_cuda` (the
reference's own CUDA build and this library's command line, each run as a
whole process on the same input, `-R -A -B`, wall clock from start to
exit).  Both are comparators; neither is part of the measured path.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

CONFIG = ROOT / "tests" / "golden" / "configs" / "five_layer"
METRIC = "photons/s (plain MC)"
WORKLOAD = "plain MC + replay, 5-layer tissue, 1e8 photons, -R -A -B"

# Per-step work of the walk, counted by hand from the step's arithmetic for
# the common step (hop + weight drop + Henyey-Greenstein spin + roulette
# test; no boundary, no roulette draw):
#   3 XORWOW draws: 9 integer ops, 1 int->float, 1 FMA each      33 lane
#   hop: 2 mul, 2 fma + 2 cmp (boundary), 3 fma (move), steps++,
#        4 clamp, 1 layer cmp                                    15 lane, lg2
#   drop: 2 mul, rint, sub                                        4 lane
#   spin: HG 10, two IEEE sqrt 2x5, sincos 2, rotation 15,
#        renormalise 6, 1 cmp                                    44 lane;
#        rcp x3, rsq x2 (sqrt), sin, cos, rsq                     8 MUFU
#   survive: 2 cmp                                                2 lane
# = 98 FP32/INT32 lane ops and 9 MUFU ops.  7 pairs of those lane ops (the
# x/y halves of the move, of the rotation's five products and sums and of
# the renormalisation) go out as one sm_100 paired FP32 instruction each
# (FFMA2/FMUL2), so a step needs 98 - 7 + 9 = 100 issue slots.  A B200 SM
# issues 128 thread-instructions per clock (4 schedulers x 32 lanes) and 16
# MUFU results, so steps/s <= f_sm * 148 * min(128 / 100, 16 / 9): the
# issue rate binds.  ncu's pipe counters agree that MUFU is not the limit:
# 9.5 XU thread-instructions per step, 91 % of issue slots used.
OPS_LANE = 98
OPS_PAIRED = 7
OPS_MUFU = 9
SM_COUNT = 148


def issue_slots_per_step() -> int:
    return OPS_LANE - OPS_PAIRED + OPS_MUFU


def steps_per_clock_per_sm() -> float:
    return min(128.0 / issue_slots_per_step(), 16.0 / OPS_MUFU)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []
        self._t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self._t = threading.Thread(target=self._read, daemon=True)
        self._t.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self._t:
            self._t.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        load = [v for v in sm if v > 0]
        return {"sm_mhz": statistics.median(load) if load else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def load_sim(photons: int | None):
    import mcml_gpu_b200 as m
    sim = m.parse_config(CONFIG / "sim_set.json", CONFIG / "input.txt")[0]
    if photons:
        sim.number_photons = int(photons)
    return sim


def load_sim_oracle(photons: int | None = None):
    """The benchmark tissue read by the oracle's own configuration reader
    (the CPU legs load no part of this library)."""
    import oracle
    sim = oracle.read_config(CONFIG / "sim_set.json", CONFIG / "input.txt")[0]
    if photons:
        sim.number_photons = int(photons)
    return sim


def cpu_port_rate(sim, seconds: float, threads: int = 0) -> dict:
    """The CPU restatement (oracle, FP32, PCG32) timed on all host cores over a
    photon sample sized to take about `seconds`."""
    import oracle
    pilot = 2000
    t0 = time.perf_counter()
    oracle.run(sim, pilot, 99, first=10**12, threads=threads)
    dt = max(time.perf_counter() - t0, 1e-3)
    n = max(pilot, int(pilot * seconds / dt))
    t0 = time.perf_counter()
    st, *_ = oracle.run(sim, n, 7, first=0, threads=threads)
    dt = time.perf_counter() - t0
    cores = threads if threads > 0 else (os.cpu_count() or 1)
    return {"value": n / dt, "unit": "photons/s", "cores": cores, "kind": "port",
            "sample": f"{n} photons of the benchmark tissue (first pass, FP32, PCG32 per photon), "
                      f"{dt:.1f} s on {cores} threads; {st.steps / max(st.photons, 1):.1f} steps/photon"}


def reference_arm(args) -> int:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    sim = load_sim_oracle(args.photons)
    cores = os.cpu_count() or 1
    # each step: a bounded sample of the workload on all cores
    import oracle
    sample = args.ref_sample
    for _ in range(args.warmup):
        oracle.run(sim, max(sample // 10, 1000), 3, first=10**12)
    times = []
    steps = 0
    for k in range(args.steps):
        t0 = time.perf_counter()
        st, *_ = oracle.run(sim, sample, 1000 + k)
        times.append(time.perf_counter() - t0)
        steps += st.steps
    total = sum(times)
    value = sample * args.steps / total
    line = {
        "metric": METRIC, "value": value, "unit": "photons/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "impl": "reference",
        "config": {"workload": WORKLOAD, "photons_per_step": sample, "note":
                   "CPU restatement of the reference walk (the reference has no CPU path)"},
        "cpu_baseline": {"value": value, "unit": "photons/s", "cores": cores, "kind": "port",
                         "sample": f"{sample} photons per step, FP32, {cores} threads, "
                                   f"{steps / (sample * args.steps):.1f} steps/photon"},
        "e2e": {"value": value, "unit": "photons/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def _timed_cli(cmd: list[str], workdir: Path, env: dict) -> tuple[float, dict]:
    """One run of a MCML_GPU command line in `workdir` (fresh files), wall
    clock from process start to exit; returns (seconds, its summary.json)."""
    for f in workdir.iterdir():
        if f.is_file() and f.name not in ("sim_set.json", "input.txt"):
            f.unlink()
    t0 = time.perf_counter()
    res = subprocess.run(cmd, cwd=workdir, env=env, capture_output=True, text=True, timeout=1200)
    dt = time.perf_counter() - t0
    if res.returncode != 0:
        raise RuntimeError(f"{cmd[0]} exited {res.returncode}: {(res.stdout + res.stderr)[-500:]}")
    summ = {}
    p = workdir / "summary.json"
    if p.exists():
        txt = p.read_text()
        for key in ("sim_time", "replay_time"):
            k = txt.find(f'"{key}": ')
            if k >= 0:
                summ[key] = float(txt[k + len(key) + 4:].split(",")[0])
        k = txt.find('"SDS_detected_number": [')
        if k >= 0:
            body = txt[k + 24:txt.index("]", k)]
            summ["detected"] = [int(v) for v in body.replace(",", " ").split()]
    return dt, summ


def reference_cuda_leg(photons: int, runs: int, seed: int) -> dict:
    """The reference's own CUDA build against this library's command line,
    like for like: `MCML_GPU sim_set.json input.txt output.txt -R -A -B` on
    the benchmark tissue at `photons`, one process per run in a fresh
    directory, wall clock from process start to exit (CUDA start-up, first
    pass, replay and every output file included), one untimed run of each
    first.  The reference (oracle/_ref/MCML_GPU, compiled from its own
    sources for sm_100a) is seeded through the time() shim because it seeds
    from time(NULL); this library's CLI takes -S.  `first_pass_s` is each
    program's own sim_time from summary.json (the reference's is CPU
    clock(), which its busy-waiting host loop keeps close to wall time)."""
    import oracle
    ours = ROOT / "mcml_gpu_b200" / "bin" / "MCML_GPU"
    if not oracle.REF_BIN.exists() or not oracle.REF_SHIM.exists():
        return {"unavailable": "oracle/_ref is not built"}
    if not ours.exists():
        return {"unavailable": "mcml_gpu_b200/bin/MCML_GPU is not built"}
    conf = json.loads((CONFIG / "sim_set.json").read_text())
    conf["number_photons"] = int(photons)
    out = {"photons": int(photons), "runs": runs, "flags": "-R -A -B",
           "timing": "wall clock per process, start to exit, after one untimed run"}
    with tempfile.TemporaryDirectory() as td:
        for name, cmd, env in (
                ("reference", [str(oracle.REF_BIN)],
                 dict(os.environ, MCML_FIXED_TIME=str(seed), LD_PRELOAD=str(oracle.REF_SHIM))),
                ("this_library", [str(ours)], dict(os.environ))):
            wd = Path(td) / name
            wd.mkdir()
            (wd / "sim_set.json").write_text(json.dumps(conf))
            (wd / "input.txt").write_text((CONFIG / "input.txt").read_text())
            full = cmd + ["sim_set.json", "input.txt", "output.txt", "-R", "-A", "-B"]
            if name == "this_library":
                full += ["-S", str(seed)]
            try:
                _timed_cli(full, wd, env)
                walls, firsts, det = [], [], None
                for _ in range(runs):
                    dt, summ = _timed_cli(full, wd, env)
                    walls.append(dt)
                    if "sim_time" in summ:
                        firsts.append(summ["sim_time"])
                    det = summ.get("detected", det)
            except Exception as e:  # report, do not fail the bench line
                out[name] = {"unavailable": str(e)[:300]}
                continue
            wall = statistics.median(walls)
            out[name] = {"wall_s": wall, "wall_s_runs": walls, "photons_per_s": photons / wall,
                         "first_pass_s": statistics.median(firsts) if firsts else None,
                         "detected": det}
    if "wall_s" in out.get("reference", {}) and "wall_s" in out.get("this_library", {}):
        out["speedup_wall"] = out["reference"]["wall_s"] / out["this_library"]["wall_s"]
        fr, fo = out["reference"]["first_pass_s"], out["this_library"]["first_pass_s"]
        if fr and fo:
            out["speedup_first_pass"] = fr / fo
    return out


def reference_gpu_arm(args) -> int:
    """The reference's own CUDA build (oracle/_ref/MCML_GPU, compiled from its
    sources for sm_100a) on the benchmark workload, wall-clock timed end to
    end per run (process start to exit, its file output included).  Seeded
    through the time() shim; N >= its thread count, as it requires."""
    import shutil
    import subprocess
    import oracle
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    if not oracle.REF_BIN.exists():
        print(json.dumps({"impl": "reference-gpu", "unavailable": "oracle/_ref not built"}))
        return 0
    sim_json = json.loads((CONFIG / "sim_set.json").read_text())
    if args.photons:
        sim_json["number_photons"] = args.photons
    N = int(sim_json["number_photons"])
    times = []
    with tempfile.TemporaryDirectory() as td:
        (Path(td) / "sim_set.json").write_text(json.dumps(sim_json))
        shutil.copy(CONFIG / "input.txt", Path(td) / "input.txt")
        env = dict(os.environ, MCML_FIXED_TIME="1234", LD_PRELOAD=str(oracle.REF_SHIM))
        for k in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            res = subprocess.run([str(oracle.REF_BIN), "sim_set.json", "input.txt", "output.txt",
                                  "-R", "-A", "-B"], cwd=td, env=env, capture_output=True,
                                 text=True, timeout=3600)
            dt = time.perf_counter() - t0
            if res.returncode != 0:
                print(json.dumps({"impl": "reference-gpu", "unavailable": f"exit {res.returncode}"}))
                return 0
            if k >= args.warmup:
                times.append(dt)
    ms = 1000 * sum(times) / len(times)
    print(json.dumps({"metric": METRIC, "impl": "reference-gpu", "value": N / (ms / 1000),
                      "unit": "photons/s", "ms_per_step": ms, "steps": args.steps,
                      "warmup": args.warmup, "photons": N,
                      "note": "reference CUDA build, wall clock per run incl. output files"}),
          flush=True)
    return 0


def batch_arm(args) -> int:
    """Batched parameter sets: 4096 sets of the 5-layer tissue (mua, mus drawn
    from the benchmark tissue's ranges by seed, photons log-uniform 1e5-1e7 per set) in
    one persistent CUDA-graph launch, autotuned; compared with the same sets
    run one after another (a sample of them, rate extrapolated)."""
    import torch
    import mcml_gpu_b200 as m
    base = load_sim(None)
    n_sets = args.sets
    sims = m.sample_sets(base, n_sets, seed=20261203, photons=(args.min_photons, args.max_photons))
    total = sum(int(s.number_photons) for s in sims)
    with m.Batch(sims, seed=args.seed) as b:
        t0 = time.perf_counter()
        tuning = b.autotune(1 / 64)
        tune_s = time.perf_counter() - t0
        for _ in range(max(args.warmup, 1)):
            b.run()
        times = []
        sampler = ClockSampler(0)
        sampler.start()
        for _ in range(args.steps):
            res = b.run()
            times.append(res[0].walk_ms)
        clocks = sampler.stop()
    ms = sum(times) / len(times)
    steps = sum(int(r.steps) for r in res)
    # the same sets one at a time through mcml_run (sample of 32 sets)
    sample = sims[:: max(1, n_sets // 32)][:32]
    seq_photons, seq_ms = 0, 0.0
    for i, s in enumerate(sample):
        with m.Simulation(s, seed=args.seed + i) as run:
            run.run()
            t0 = time.perf_counter()
            run.run()
            seq_ms += 1000 * (time.perf_counter() - t0)
            seq_photons += int(s.number_photons)
    rel = [r.std_error[1] / r.reflectance[1] for r in res if r.reflectance[1] > 0]
    print(json.dumps({
        "metric": "photons/s (batched plain MC)", "impl": "mcml-batch", "value": total / (ms / 1e3),
        "unit": "photons/s", "ms_per_step": ms, "steps": args.steps, "warmup": args.warmup,
        "config": {"workload": "4096 batched 5-layer sets, log-uniform 1e5-1e7 photons per set",
                   "sets": n_sets, "photons_total": total,
                   "photons_per_set": [args.min_photons, args.max_photons],
                   "tuned": {"block": tuning.block_size, "blocks_per_sm": tuning.blocks_per_sm,
                             "photons_per_slot": tuning.photons_per_slot},
                   "tune_s": round(tune_s, 2), "cuda_graph": True},
        "steps_per_s": steps / (ms / 1e3),
        "roofline": issue_roofline(steps / (ms / 1e3), clocks, "batch_walk_kernel"),
        "clocks": clocks,
        "sequential_same_library": {"value": seq_photons / (seq_ms / 1e3), "sets": len(sample)},
        "median_rel_se_sds2": float(np.median(rel)) if rel else None,
    }), flush=True)
    return 0


def issue_roofline(steps_per_s: float, clocks: dict, kernel: str) -> dict:
    """Walk steps/s against the issue bound of the hand-counted step (see
    OPS_LANE / OPS_MUFU) at the median SM clock sampled while it ran."""
    f_sm = clocks.get("sm_mhz") or 1965.0
    peak = f_sm * 1e6 * SM_COUNT * steps_per_clock_per_sm()
    return {"bound": "issue", "achieved": steps_per_s / 1e9, "peak": peak / 1e9,
            "unit": "Gstep/s", "frac": steps_per_s / peak, "kernel": kernel}


def wmc_arm(args) -> int:
    """White-MC relabelling throughput: the replayed photons of one SDS of
    the ring geometry (tests/golden/configs/surrogate, 2e7 photons) under
    4096 (mua', mus') combinations; one term = one (photon, combo) pair:
    K = 2L+2 FMAs, one exp2, one add.  Timed with CUDA events on the
    launching stream after warm-up."""
    import torch
    import mcml_gpu_b200 as m
    import mcml_gpu_b200.wmc as wmc
    cfg = ROOT / "tests" / "golden" / "configs" / "surrogate"
    sim = m.parse_config(cfg / "sim_set.json", cfg / "input.txt")[0]
    sim.number_photons = int(args.photons) if args.photons else 20_000_000
    L = int(sim.num_layers)
    with m.Simulation(sim, seed=args.seed) as run:
        run.run()
        run.replay()
        rows, inter = run.rows(1)
    rng = np.random.default_rng(3)
    C = 4096
    mua0 = np.array([sim.mua[l] for l in range(L)])
    mus0 = np.array([sim.mus[l] for l in range(L)])
    combos = np.hstack([rng.uniform(0.05, 0.5, (C, L)),
                        mus0[None, :] * rng.uniform(0.95, 1.05, (C, L))]).astype(np.float32)
    combos_t = torch.from_numpy(combos).cuda()
    prep = wmc.Prepared(rows, inter)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    for _ in range(max(args.warmup, 1)):
        prep.rescale(mua0, mus0, combos_t, int(sim.number_photons))
    ev1.record()
    torch.cuda.synchronize()
    # one call takes milliseconds: repeat it for about 2 s so that the clock
    # sampler (every 200 ms) sees the timed region
    reps = max(args.steps, int(2000.0 / max(ev0.elapsed_time(ev1) / max(args.warmup, 1), 1e-3)))
    sampler = ClockSampler(0)
    sampler.start()
    ev0.record()
    for _ in range(reps):
        out = prep.rescale(mua0, mus0, combos_t, int(sim.number_photons))
    ev1.record()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    ms = ev0.elapsed_time(ev1) / reps
    D = rows.shape[0]
    terms = D * C / (ms / 1e3)
    K = 2 * L + 2
    # per term: the exponent starts at log2 w and takes 2L FMAs, issued as L
    # paired FMAs (two photons each), then one MUFU exp2 and half a paired
    # add; the 16-byte shared loads (K-2 per 8 terms, plus two 8-byte loads
    # of log2 w) are shared by the 2 photons x 2 combos of a thread.  That
    # is `ops` issue slots; the FP32 lanes still do 2L + 1 operations (a
    # paired instruction saves an issue slot, not a lane: it holds the
    # lanes for two cycles).  Bound per SM and clock: min(128 / ops issue,
    # 128 / (2L + 1) FP32 lanes, 16 MUFU).
    ops = L + 1 + 0.5 + K / 8
    lanes = 2 * L + 1
    f_sm = clocks.get("sm_mhz") or 1965.0
    per_clk = {"issue": 128.0 / ops, "fp32": 128.0 / lanes, "mufu": 16.0}
    bound = min(per_clk, key=per_clk.get)
    peak = f_sm * 1e6 * SM_COUNT * per_clk[bound]
    print(json.dumps({
        "metric": "White-MC terms/s", "impl": "mcml-wmc", "value": terms, "unit": "terms/s",
        "ms_per_step": ms, "steps": reps, "warmup": args.warmup,
        "config": {"workload": f"WMC rescale, ring geometry, {sim.number_photons:.3g} photons, "
                               f"SDS 1: {D} replayed photons x {C} combos, L={L}",
                   "includes": "coefficient and packing kernels of each call (inputs resident)"},
        "roofline": {"bound": bound, "achieved": terms / 1e12, "peak": peak / 1e12,
                     "unit": "Tterm/s", "frac": terms / peak,
                     "model": f"terms/clk/SM <= min(128/{ops:.1f} issue slots, 128/{lanes} FP32 "
                              f"lane ops, 16 MUFU exp2) per term, at the sampled SM clock"},
        "clocks": clocks}), flush=True)
    return 0


def measured_peak(key: str, fallback: float) -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    try:
        return float(json.loads(p.read_text())[key]), "measured"
    except Exception:
        return fallback, "fallback"


def mlp_roofline(queries: int, seconds: float) -> dict:
    """Tensor-core roofline of ensemble inference: algorithmic FLOPs of the
    25 -> 256x4 -> 3 network x 4 members per query (2 x MACs, real widths),
    over the whole predict call (gather, layers, ensemble reduction)."""
    macs = 25 * 256 + 3 * 256 * 256 + 256 * 3
    flops = 2.0 * macs * 4 * queries
    peak, kind = measured_peak("bf16_tflops", 1590.0)
    achieved = flops / seconds / 1e12
    return {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": achieved / peak, "peak_kind": kind, "flop_per_query": 2.0 * macs * 4}


def reference_plain_mc_evals(cfg: Path, sims, photons: int) -> tuple[float | None, str]:
    """Plain-MC evaluations per second of the reference's CUDA build
    (oracle/_ref/MCML_GPU) on the same tissues, one process per tissue (its
    multi-simulation mode ends in a segmentation fault here), wall clock
    from process start to exit.  Returns (rate or None, note)."""
    import oracle
    if not oracle.REF_BIN.exists():
        return None, "oracle/_ref not built"
    conf = json.loads((cfg / "sim_set.json").read_text())
    conf["number_photons"] = photons
    conf["number_simulation"] = 1
    total = 0.0
    for s in sims:
        L = int(s.num_layers)
        vals = []
        for l in range(L):
            if l < L - 1:
                vals.append(s.height[l])
            vals += [s.mua[l], s.mus[l], s.n[l], s.g[l]]
        with tempfile.TemporaryDirectory() as td:
            (Path(td) / "sim_set.json").write_text(json.dumps(conf))
            (Path(td) / "input.txt").write_text("\t".join(f"{float(v):.9g}" for v in vals) + "\n")
            env = dict(os.environ, MCML_FIXED_TIME="1234", LD_PRELOAD=str(oracle.REF_SHIM))
            t0 = time.perf_counter()
            res = subprocess.run([str(oracle.REF_BIN), "sim_set.json", "input.txt", "output.txt"],
                                 cwd=td, env=env, capture_output=True, text=True, timeout=3600)
            total += time.perf_counter() - t0
        if res.returncode != 0:
            tail = (res.stdout + res.stderr).strip().splitlines()[-3:]
            return None, f"exit {res.returncode}: " + " | ".join(tail)
    return len(sims) / total, f"{len(sims)} tissues x {photons:.3g} photons in {total:.2f} s"


MUA_RANGE = (0.05, 0.5)   # 1/cm, the benchmark tissue's range
MUS_RANGE = (50.0, 250.0)  # 1/cm


def surrogate_arm(args) -> int:
    """Surrogate training and serving: White-MC labels from replayed baselines of the 5-layer
    tissue (ring detectors at 0.5/1.0/1.5 cm, tests/golden/configs/surrogate),
    ensemble training on the GPU, serving of 1e6 queries (5 % outside the
    training hull, whose answers come from plain MC at --fallback-photons),
    and the error against plain MC at 1e8 photons on held-out tissues: the
    network's answers inside the hull, the fallback's answers outside it, and
    the two mixed in the proportions the queries have."""
    import torch
    import mcml_gpu_b200 as m
    import mcml_gpu_b200.surrogate as sg
    cfg = ROOT / "tests" / "golden" / "configs" / "surrogate"
    base = m.parse_config(cfg / "sim_set.json", cfg / "input.txt")[0]
    L = int(base.num_layers)
    t0 = time.perf_counter()
    labels = sg.make_labels(base, n_baselines=args.baselines, photons=int(args.label_photons),
                            combos_per_baseline=args.combos // args.baselines, seed=1,
                            mua_range=MUA_RANGE, mus_range=MUS_RANGE,
                            mua_baseline=args.label_mua_baseline, mus_jitter=args.label_mus_jitter)
    label_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    fb_photons = int(args.fallback_photons)
    sur = sg.Surrogate.train(labels, epochs=args.epochs, batch=args.train_batch,
                             lr=args.train_lr, seed=1, max_spread=0.05,
                             fallback_photons=fb_photons)
    train_s = time.perf_counter() - t0
    # training FLOPs: forward + input and weight gradients (3 x the forward's
    # 2 x multiply-adds of the real widths) for every row of every full
    # minibatch, 4 members
    macs = 25 * 256 + 3 * 256 * 256 + 256 * 3
    n_lab = int(labels.X.shape[0])
    train_flop = 3 * 2.0 * macs * 4 * (n_lab // args.train_batch * args.train_batch) * args.epochs
    rng = np.random.default_rng(5)
    # 1e6 queries: mua and mus of every layer uniform over the tissue's ranges;
    # 5 % of them take one coefficient from the 20 %-widened ranges' excess,
    # outside the training hull
    nq = args.queries
    X = np.repeat(sg.features(labels.baselines[:1]), nq, axis=0)
    for l in range(L):
        X[:, 5 * l + 1] = rng.uniform(*MUA_RANGE, nq)
        X[:, 5 * l + 2] = rng.uniform(*MUS_RANGE, nq)
    out = rng.random(nq) < 0.05
    for i in np.nonzero(out)[0]:
        l, which = rng.integers(0, L), rng.integers(1, 3)
        lo, hi = MUA_RANGE if which == 1 else MUS_RANGE
        ext = 0.2 * (hi - lo)
        X[i, 5 * l + which] = (rng.uniform(lo - ext, lo) if rng.random() < 0.5
                               else rng.uniform(hi, hi + ext))
    Xt = torch.from_numpy(X).cuda()
    sur.mlp.predict(Xt)  # warm-up at the full size (buffers sized once, outside the timing)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    mean, spread = sur.mlp.predict(Xt)
    torch.cuda.synchronize()
    mlp_s = time.perf_counter() - t0
    inside = np.all((X >= sur.lo - 1e-6) & (X <= sur.hi + 1e-6), axis=1)
    agree = np.all(spread.cpu().numpy() <= sur.max_spread, axis=1)
    fallback = ~(inside & agree)
    # cost of the fallback: plain MC at fb_photons for a sample of flagged queries
    fb_idx = np.nonzero(fallback)[0][:64]
    fb = []
    for i in fb_idx:
        s = m.Sim.from_buffer_copy(labels.baselines[0])
        for l in range(L):
            s.mua[l], s.mus[l] = float(X[i, 5 * l + 1]), float(X[i, 5 * l + 2])
        s.number_photons = fb_photons
        fb.append(s)
    with m.Batch(fb, seed=3) as b:
        b.run()
        res = b.run()
    fb_per_query_s = res[0].walk_ms / 1e3 / max(len(fb), 1)
    serve_s = mlp_s + fallback.sum() * fb_per_query_s
    # error against plain MC on held-out tissues (drawn like the labels)
    # held-out tissues drawn like the in-hull queries
    held = []
    for k in range(args.heldout):
        s = m.Sim.from_buffer_copy(labels.baselines[0])
        for l in range(L):
            s.mua[l] = float(rng.uniform(*MUA_RANGE))
            s.mus[l] = float(rng.uniform(*MUS_RANGE))
        s.number_photons = int(args.ref_photons)
        held.append(s)
    with m.Batch(held, seed=11) as b:
        ref = b.run()
    mc_rate = sum(int(s.number_photons) for s in held) / (ref[0].walk_ms / 1e3)
    R_ref = np.array([r.reflectance[:3] for r in ref])
    se = np.array([r.std_error[:3] for r in ref]) / R_ref
    logR, _ = sur.predict(sg.features(held))
    rel = np.abs(np.exp(logR) - R_ref) / R_ref
    mc_evals = mc_rate / float(args.ref_photons)
    # the fallback's own error: out-of-hull held-out tissues (one coefficient
    # in the widened ranges' excess, like the flagged queries), plain MC at
    # fb_photons against plain MC at ref_photons
    out_t = []
    for k in range(args.heldout_out):
        s = m.Sim.from_buffer_copy(labels.baselines[0])
        for l in range(L):
            s.mua[l] = float(rng.uniform(*MUA_RANGE))
            s.mus[l] = float(rng.uniform(*MUS_RANGE))
        l, which = rng.integers(0, L), rng.integers(1, 3)
        lo, hi = MUA_RANGE if which == 1 else MUS_RANGE
        ext = 0.2 * (hi - lo)
        v = rng.uniform(lo - ext, lo) if rng.random() < 0.5 else rng.uniform(hi, hi + ext)
        if which == 1:
            s.mua[l] = float(v)
        else:
            s.mus[l] = float(v)
        out_t.append(s)
    rel_fb = np.zeros((0, 3))
    if out_t:
        refs_o, fbs_o = [], []
        for t in out_t:
            a, b2 = m.Sim.from_buffer_copy(t), m.Sim.from_buffer_copy(t)
            a.number_photons, b2.number_photons = int(args.ref_photons), fb_photons
            refs_o.append(a)
            fbs_o.append(b2)
        with m.Batch(refs_o, seed=21) as b:
            ro = b.run()
        with m.Batch(fbs_o, seed=22) as b:
            fo = b.run()
        Ro = np.array([r.reflectance[:3] for r in ro])
        Fo = np.array([r.reflectance[:3] for r in fo])
        rel_fb = np.abs(Fo - Ro) / Ro
    # served error: network answers and fallback answers in the queries' mix
    frac_fb = float(fallback.mean())
    vals = np.concatenate([rel.ravel(), rel_fb.ravel()])
    wts = np.concatenate([np.full(rel.size, (1 - frac_fb) / max(rel.size, 1)),
                          np.full(rel_fb.size, frac_fb / max(rel_fb.size, 1))])
    order = np.argsort(vals)
    cw = np.cumsum(wts[order]) / wts.sum()

    def wq(q):
        return float(vals[order][np.searchsorted(cw, q)])
    ref_evals, ref_note = reference_plain_mc_evals(cfg, held[:2], int(args.ref_photons))
    print(json.dumps({
        "metric": "SDS-reflectance evals/s", "impl": "mcml-surrogate",
        "value": nq / serve_s, "unit": "evals/s",
        "mlp_only_evals_per_s": nq / mlp_s,
        "mlp_roofline": mlp_roofline(nq, mlp_s),
        "plain_mc_evals_per_s_at_ref_photons": mc_evals,
        "speedup_vs_plain_mc": (nq / serve_s) / mc_evals,
        "speedup_vs_plain_mc_inside_hull": (nq / mlp_s) / mc_evals,
        "reference_plain_mc_evals_per_s": ref_evals, "reference_plain_mc_run": ref_note,
        "speedup_vs_reference_plain_mc": (nq / serve_s) / ref_evals if ref_evals else None,
        "fallback_fraction": frac_fb,
        "fallback_photons": fb_photons,
        "fallback_s_per_query": fb_per_query_s,
        "speedup_cap_from_fallback": float(args.ref_photons) / max(frac_fb * fb_photons, 1.0),
        "error_vs_plain_mc": {"median_rel": float(np.median(rel)),
                              "p90_rel": float(np.percentile(rel, 90)),
                              "per_sds_median": [float(v) for v in np.median(rel, axis=0)],
                              "per_sds_p90": [float(v) for v in np.percentile(rel, 90, axis=0)],
                              "mc_rel_se_median": float(np.median(se)),
                              "heldout": args.heldout, "ref_photons": int(args.ref_photons),
                              "note": "network answers, held-out tissues inside the hull"},
        "fallback_error_vs_plain_mc": {
            "median_rel": float(np.median(rel_fb)) if rel_fb.size else None,
            "p90_rel": float(np.percentile(rel_fb, 90)) if rel_fb.size else None,
            "heldout": len(out_t),
            "note": "plain MC at fallback_photons on out-of-hull held-out tissues"},
        "served_error_vs_plain_mc": {"median_rel": wq(0.5), "p90_rel": wq(0.9),
                                     "note": "network and fallback answers weighted by the "
                                             "queries' fallback fraction"},
        "labels": {"count": int(labels.X.shape[0]), "baselines": args.baselines,
                   "photons_per_baseline": int(args.label_photons), "seconds": label_s,
                   "mua_baseline": args.label_mua_baseline, "mus_jitter": args.label_mus_jitter},
        "training": {"epochs": args.epochs, "seconds": train_s, "batch": args.train_batch,
                     "lr": args.train_lr, "tflops": train_flop / train_s / 1e12,
                     "final_loss": [float(v) for v in sur.history[-1]]},
        "config": {"workload": "surrogate: WMC labels, MLP 25->256x4->3 GELU, ensemble 4, "
                               "BF16 tensor-core kernels; ring detectors 0.5/1.0/1.5 cm",
                   "queries": nq},
    }), flush=True)
    return 0


def read_traffic(slots: int) -> float | None:
    """DRAM bytes of one walk launch: the ncu-measured bytes per slot of a
    smaller capture (profiles/walk_kernel_traffic.json) times this run's
    slot count -- the walk's DRAM traffic is the slot-state reads."""
    p = ROOT / "profiles" / "walk_kernel_traffic.json"
    if not p.exists():
        return None
    try:
        return float(json.loads(p.read_text())["dram_bytes_per_slot"]) * slots
    except Exception:
        return None


def mcml_arm(args) -> int:
    import torch
    import mcml_gpu_b200 as m

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    sim = load_sim(args.photons)
    N = int(sim.number_photons)
    info = m.device_info(local)
    slots = args.slots  # 0: the library's automatic slot count
    # A dedicated (non-default) stream: the library launches on it and the
    # CUDA events below are recorded on it.
    stream = torch.cuda.Stream(device=local)
    torch.cuda.set_stream(stream)
    # Each rank walks its own range of RNG subsequences (weak scaling).
    first, _ = m.shard(rank, world, slots or N, weak=True)
    run = m.Simulation(sim, seed=args.seed, slots=slots, slot_begin=first,
                       device=local, stream=stream.cuda_stream, block_size=args.block,
                       blocks_per_sm=args.blocks_per_sm)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")

    def step():
        run.launch_run()
        run.launch_replay()
        if dist:
            # the job's one exchange: u64 tallies summed and rows gathered over
            # NCCL on the device buffers (rank 0 gets the whole run)
            from mcml_gpu_b200.distributed import gather_device
            gather_device(run.device_outputs())

    for _ in range(args.warmup):
        flush.zero_()
        step()
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    walk_ms = []
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    wall0 = time.perf_counter()
    for k in range(args.steps):
        flush.zero_()
        starts[k].record(stream)
        step()
        ends[k].record(stream)
        res = None
    torch.cuda.synchronize()
    wall = time.perf_counter() - wall0
    if dist:
        dist.barrier()
    clocks = sampler.stop()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    res = run.result()  # the last step's first pass
    rep = run.replay()  # (re-runs the replay once, outside the timed region, for the row count)
    total_ms = sum(step_ms)
    if dist:
        t = torch.tensor([total_ms], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    value = world * N * args.steps / (total_ms / 1000.0)

    # e2e through the public API: host struct in, host rows and tallies out
    e2e_steps = max(1, min(args.steps, 3))
    L, S = sim.num_layers, sim.num_sds
    nr, nz = 1000, 500
    arz = np.empty((S, nz, nr), dtype=np.uint64)
    d2h = 0
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        run.set_sim(sim)
        r1 = run.run()
        r2 = run.replay()
        nrows = 0
        for sds in range(1, S + 1):
            rows, inter = run.rows(sds)
            nrows += rows.shape[0]
        a_rz, a0_z = run.tallies()
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    if dist:
        t = torch.tensor([e2e_s], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    d2h = (m.C.sizeof(m.Result) * 2 + nrows * ((L + 2) * 4 + L * 4) + 12 * nrows
           + a_rz.nbytes + a0_z.nbytes)
    h2d = m.C.sizeof(m.Sim)

    steps_per_photon = res.steps / max(res.photons, 1)
    walk_kernel_ms = float(res.walk_ms)
    achieved = res.steps / (walk_kernel_ms / 1000.0)
    f_sm = clocks.get("sm_mhz") or 1965.0
    peak = f_sm * 1e6 * info.sm_count * steps_per_clock_per_sm()
    line = {
        "metric": METRIC, "value": value, "unit": "photons/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "photons": N, "layers": L, "sds": S,
                   "grid": "1000x500 @ 0.01 cm", "slots": int(res.slots),
                   "l2": "flushed between steps (256 MiB write)",
                   "parallelism": (f"replicas x{world}, disjoint RNG subsequences; tallies "
                                   f"all-reduced and rows all-gathered over NCCL in each step"
                                   if world > 1 else "1 GPU"),
                   "steps_per_photon": round(steps_per_photon, 2),
                   "detected": [int(v) for v in res.detected[:S]],
                   "replayed_rows": int(sum(rep.detected[:S]))},
        "e2e": {"value": N * world / e2e_s, "unit": "photons/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": int(d2h)},
        # seeding, walk, record reduction, replay; with ranks to combine also the
        # record ordering (keys + gather; the radix sort between them is CUB's)
        "gpu_launches": (4 + (2 if world > 1 else 0)) * args.steps,
        "roofline": {"bound": "issue", "achieved": achieved / 1e9, "peak": peak / 1e9,
                     "unit": "Gstep/s", "frac": achieved / peak,
                     "traffic": read_traffic(int(res.slots)),
                     "kernel": "walk_kernel",
                     "model": f"steps/s <= f_sm x {info.sm_count} SMs x min(128/({OPS_LANE}-"
                              f"{OPS_PAIRED}+{OPS_MUFU}), 16/{OPS_MUFU}) at the measured median "
                              f"SM clock (issue bound: 128 thread-instructions/clk/SM; "
                              f"{OPS_PAIRED} lane-op pairs issued as paired FP32 instructions); "
                              f"ops counted by hand per common step",
                     "walk_ms": walk_kernel_ms, "seed_ms": float(res.seed_ms),
                     "replay_ms": float(rep.replay_ms)},
        "clocks": clocks,
        "wall_s_timed": wall,
    }
    S = int(sim.num_sds)
    line["reflectance"] = {
        "per_sds": [float(v) for v in res.reflectance[:S]],
        "std_error": [float(v) for v in res.std_error[:S]],
        "detected": [int(v) for v in res.detected[:S]],
        "photons": int(res.photons),
        "note": "first pass of the last timed step: R_s = sum of detected weights / "
                "(0xFFFFFFFF N), SE from the per-photon weight variance"}
    run.close()
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_port_rate(load_sim_oracle(), args.cpu_seconds)
    if rank == 0 and world == 1 and args.ref_cuda_runs > 0:
        line["reference_cuda"] = reference_cuda_leg(N, args.ref_cuda_runs, args.seed)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def main() -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mcml",
                    choices=["mcml", "reference", "reference-gpu", "batch", "surrogate", "wmc"])
    ap.add_argument("--photons", type=int, default=0, help="override N (default: 1e8)")
    ap.add_argument("--slots", type=int, default=0)
    ap.add_argument("--block", type=int, default=0)
    ap.add_argument("--blocks-per-sm", type=int, default=0)
    ap.add_argument("--seed", type=int, default=1234)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-sample", type=int, default=300000)
    ap.add_argument("--ref-cuda-runs", type=int, default=3,
                    help="timed runs of each CLI in the reference_cuda leg (0: skip it)")
    ap.add_argument("--sets", type=int, default=4096)
    ap.add_argument("--min-photons", type=float, default=1e5)
    ap.add_argument("--max-photons", type=float, default=1e7)
    ap.add_argument("--baselines", type=int, default=512)
    ap.add_argument("--label-photons", type=float, default=1e7)
    ap.add_argument("--label-mua-baseline", default="low", choices=["mid", "low"])
    ap.add_argument("--label-mus-jitter", type=float, default=0.05)
    ap.add_argument("--combos", type=int, default=2_000_000)
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--train-batch", type=int, default=8192)
    ap.add_argument("--train-lr", type=float, default=2.8e-3)
    ap.add_argument("--queries", type=int, default=1_000_000)
    ap.add_argument("--heldout", type=int, default=1000)
    ap.add_argument("--heldout-out", type=int, default=40,
                    help="out-of-hull held-out tissues for the fallback's error")
    ap.add_argument("--fallback-photons", type=float, default=2e6)
    ap.add_argument("--ref-photons", type=float, default=1e8)
    args = ap.parse_args()
    if args.impl == "reference":
        return reference_arm(args)
    if args.impl == "reference-gpu":
        return reference_gpu_arm(args)
    if args.impl == "batch":
        return batch_arm(args)
    if args.impl == "surrogate":
        return surrogate_arm(args)
    if args.impl == "wmc":
        return wmc_arm(args)
    return mcml_arm(args)


if __name__ == "__main__":
    sys.exit(main())
