"""The multi-rank path on CPU: two gloo ranks walk disjoint shards of the
photons (mcml_gpu_b200.shard) and add their per-SDS sums with an
all-reduce; the result equals one run over all photons.  The CPU oracle
stands in for the per-rank GPU walk (its photon streams are per-photon, as
the library's are per-subsequence), so the partition and the reduction are
what is tested."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import load_case

SEED = 99
N = 60000


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, weak, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    import mcml_gpu_b200 as m
    import oracle
    sim = load_case("fiber3")
    first, n = m.shard(rank, world, N // world if weak else N, weak=weak)
    st, ids, sds, w = oracle.run(sim, n, SEED, first=first, threads=2)
    S = sim.num_sds
    t = torch.tensor([float(st.detected[i]) for i in range(S)] +
                     [st.wsum[i] for i in range(S)] + [float(n)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    ids_t = torch.tensor(ids.astype(np.int64))
    sizes = [torch.zeros(1, dtype=torch.int64) for _ in range(world)]
    dist.all_gather(sizes, torch.tensor([ids_t.numel()]))
    if rank == 0:
        out.put(t.numpy().tolist())
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("weak", [True, False])
def test_two_gloo_ranks_equal_one_run(weak):
    import mcml_gpu_b200 as m
    import oracle
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, weak, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    sim = load_case("fiber3")
    total = N  # weak: two ranks of N/2 each; strong: N split in two
    st, *_ = oracle.run(sim, total, SEED, first=0, threads=2)
    S = sim.num_sds
    assert got[-1] == total
    assert got[:S] == [float(st.detected[i]) for i in range(S)]
    np.testing.assert_allclose(got[S:2 * S], [st.wsum[i] for i in range(S)], rtol=1e-12)


def test_shard_ranges_are_disjoint_and_cover():
    import mcml_gpu_b200 as m
    for world in (1, 2, 3, 8):
        for photons in (1, 7, 1000, 303104):
            spans = [m.shard(r, world, photons, weak=False) for r in range(world)]
            assert sum(n for _, n in spans) == photons
            ends = [f + n for f, n in spans]
            assert all(spans[r + 1][0] == ends[r] for r in range(world - 1))
            weak = [m.shard(r, world, photons, weak=True) for r in range(world)]
            assert all(weak[r + 1][0] >= weak[r][0] + weak[r][1] for r in range(world - 1))
