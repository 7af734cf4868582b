"""The final combination of a multi-GPU run, on CPU: two gloo ranks hold
shards (synthetic detections, rows and u64 tallies with the shapes a run
produces) and gather_to_rank0 must give rank 0 exactly what combine()
gives for the same shards in one process; the files written from it by
the host writer (mcml_write_host_outputs) carry the combined numbers.
The slot split itself is checked against the photon-per-slot rule."""
import os
import socket
import tempfile
from pathlib import Path

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import load_case

L, S, NZ, NR = 5, 3, 50, 60


def synthetic_shard(rank):
    from mcml_gpu_b200.distributed import Shard
    rng = np.random.default_rng(100 + rank)
    rows, weights = [], []
    for s in range(S):
        n = int(rng.integers(0, 40)) if not (rank == 1 and s == 2) else 0
        r = rng.random((n, L + 2)).astype(np.float32) * 100
        r[:, 0] = rng.integers(1, 2**31, n).astype(np.float32)
        rows.append(r)
        weights.append(r[:, 0].copy())
    a_rz = rng.integers(0, 2**40, (S, NZ, NR), dtype=np.uint64)
    a0_z = rng.integers(0, 2**40, (S, NZ), dtype=np.uint64)
    return Shard(1000 + rank, weights, rows, a_rz, a0_z, 7 + rank)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    from mcml_gpu_b200.distributed import gather_to_rank0
    got = gather_to_rank0(synthetic_shard(rank))
    if rank == 0:
        out.put((got.photons, got.steps, [w.tolist() for w in got.weights],
                 [r.tobytes() for r in got.rows], got.A_rz.tobytes(), got.A0_z.tobytes()))
    else:
        assert got is None
    dist.barrier()
    dist.destroy_process_group()


def test_gather_to_rank0_equals_local_combine():
    from mcml_gpu_b200.distributed import combine
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    want = combine([synthetic_shard(0), synthetic_shard(1)])
    assert got[0] == want.photons == 2001 and got[1] == want.steps == 15
    assert got[2] == [w.tolist() for w in want.weights]
    assert got[3] == [r.tobytes() for r in want.rows]
    assert got[4] == want.A_rz.tobytes() and got[5] == want.A0_z.tobytes()


def device_layout(shard):
    """A shard as Simulation.device_outputs() lays it out (CPU tensors here):
    records SDS-major with the weight in word 3, rows likewise, int64 tallies."""
    import torch
    rows = np.concatenate(shard.rows)
    rec = np.zeros((rows.shape[0], 10), np.float32)
    rec[:, 3] = rows[:, 0]
    return {"records": torch.from_numpy(rec), "rows": torch.from_numpy(rows),
            "A_rz": torch.from_numpy(shard.A_rz.astype(np.int64)),
            "A0_z": torch.from_numpy(shard.A0_z.astype(np.int64)),
            "detected": [len(r) for r in shard.rows], "photons": shard.photons}


def _rank_main_device(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    from mcml_gpu_b200.distributed import gather_device
    sh = synthetic_shard(rank)
    got = gather_device(device_layout(sh), steps=sh.steps)
    if rank == 0:
        out.put((got.photons, got.steps, [w.tobytes() for w in got.weights],
                 [r.tobytes() for r in got.rows], got.A_rz.tobytes(), got.A0_z.tobytes()))
    else:
        assert got is None
    dist.barrier()
    dist.destroy_process_group()


def test_device_tensor_combine_equals_local_combine():
    """gather_device -- the combine a multi-GPU job runs over NCCL on device
    tensors -- on two gloo ranks with CPU tensors: rank 0 gets, byte for byte,
    what combine() gives for the same shards in one process."""
    from mcml_gpu_b200.distributed import combine
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main_device, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    want = combine([synthetic_shard(0), synthetic_shard(1)])
    assert got[0] == want.photons == 2001 and got[1] == want.steps == 15
    assert got[2] == [w.tobytes() for w in want.weights]
    assert got[3] == [r.tobytes() for r in want.rows]
    assert got[4] == want.A_rz.tobytes() and got[5] == want.A0_z.tobytes()


def test_host_writer_files_carry_the_combined_run():
    import mcml_gpu_b200 as m
    from mcml_gpu_b200.distributed import combine, write_outputs
    sim = load_case("ring5")
    run = combine([synthetic_shard(0), synthetic_shard(1)])
    flags = m.OUT_REPLAY | m.OUT_ABSORBANCE | m.OUT_PATHLENGTH | m.OUT_BINARY
    with tempfile.TemporaryDirectory() as td:
        write_outputs(sim, run, td, os.path.join(td, "output.txt"), flags,
                      grid=(NR, NZ, 0.01, 0.01))
        d = Path(td)
        for s in range(S):
            b = (d / f"pathlength_SDS_{s + 1}.bin").read_bytes()
            assert b == run.rows[s].tobytes()
        vals = [float(v) for v in (d / "output.txt").read_text().split()]
        want = [float(np.cumsum(r[:, 0].astype(np.float64))[-1]) / (0xFFFFFFFF * run.photons)
                if len(r) else 0.0 for r in run.rows]
        np.testing.assert_allclose(vals, want, rtol=1e-5)
        a0 = np.frombuffer((d / "A0_z_SDS_1.bin").read_bytes(), np.float32)
        scale = 0xFFFFFFFF * run.photons * 2 * np.float32(3.141592654) * 0.5 * 0.01 ** 3
        np.testing.assert_allclose(a0, run.A0_z[0] / scale, rtol=1e-5)
        assert '"SDS_detected_number": [ %d , %d , %d ]' % tuple(len(r) for r in run.rows) in \
            (d / "summary.json").read_text()


@pytest.mark.parametrize("photons,slots,world", [(1000, 100, 3), (1000, 1000, 4), (10**8, 12_500_000, 8),
                                                 (997, 100, 2)])
def test_slot_split_keeps_each_slots_photons(photons, slots, world):
    from mcml_gpu_b200.distributed import slot_span
    spans = [slot_span(r, world, slots, photons) for r in range(world)]
    assert spans[0][0] == 0 and sum(c for _, c, _ in spans) == slots
    assert sum(n for _, _, n in spans) == photons
    for (b0, c0, _), (b1, _, _) in zip(spans, spans[1:]):
        assert b0 + c0 == b1
    q, rem = divmod(photons, slots)
    for b, c, n in spans:
        assert n == sum(q + (1 if s < rem else 0) for s in range(b, b + c))
