"""Runs over several GPUs: replicas on disjoint slot ranges, combined once.

Photons are independent and a slot's photons depend only on (seed, slot),
so rank r walks slots [r*S/W, (r+1)*S/W) of the whole run (mcml_opts
.slot_begin) with no collective while it walks.  The combination is one
step at the end, the reference's host collection (transport.cu:152-272)
across ranks instead of across threads:

  * u64 absorbance tallies: summed (an all-reduce of int64 quanta);
  * detected weights and replay rows: gathered to rank 0 in rank order,
    which is slot order, i.e. the photon order of one run over all slots;
  * the per-SDS FP64 weight sums are taken on rank 0 over the gathered
    rows in that order, so the files equal those of a single run with the
    same seed and slots byte for byte.

`combine` does the same for shards held in one process (tests; one GPU
walking the shards one after another).  `gather_device` is the combine of
a multi-GPU job: it runs the collectives on the tensors where they lie --
under NCCL on each GPU's own device memory (Simulation.device_outputs), so
the 12 MB of tallies and the rows cross NVLink, not the host -- and only
rank 0's result comes to the host, for the writers.  `gather_to_rank0`
is the host-array form (a gloo group).  Nothing here runs on the oracle.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

from . import HostData, Sim, Simulation, _check, load_library

__all__ = ["Shard", "slot_span", "run_shard", "combine", "gather_to_rank0", "gather_device",
           "write_outputs"]


@dataclass
class Shard:
    """What one rank contributes: its photon count, per SDS the detected
    weights (quanta, photon order) and, after a replay, the pathlength rows;
    the u64 tallies; steps walked."""
    photons: int
    weights: list            # per SDS: float32 (n_s,)
    rows: Optional[list]     # per SDS: float32 (n_s, L+2), or None without replay
    A_rz: Optional[np.ndarray]
    A0_z: Optional[np.ndarray]
    steps: int = 0


def slot_span(rank: int, world: int, slots: int, photons: int) -> tuple[int, int, int]:
    """(slot_begin, slot_count, photon_count) of `rank` when a run of
    `photons` photons on `slots` slots is split over `world` ranks.  The
    split keeps each slot's photon count what the whole run gives it
    (q or q+1, the first photons % slots slots taking one more), so the
    shards together walk exactly the photons of the whole run."""
    if world < 1 or not 0 <= rank < world or slots < 1 or photons < slots:
        raise ValueError("need 0 <= rank < world, 1 <= slots <= photons")
    q, rem = divmod(photons, slots)
    base, extra = divmod(slots, world)
    begin = rank * base + min(rank, extra)
    count = base + (1 if rank < extra else 0)

    def photons_before(s):
        return s * q + min(s, rem)
    return begin, count, photons_before(begin + count) - photons_before(begin)


def run_shard(sim: Sim, *, rank: int, world: int, seed: int, slots: int, replay: bool = True,
              device: int = 0, **opts) -> Shard:
    """Walk (and replay) this rank's slots.  With n photons on `count`
    slots the library gives its first n % count slots one photon more --
    the same counts the whole run gives those slots, wherever the whole
    run's remainder falls -- so the shards walk the whole run's photons."""
    begin, count, n = slot_span(rank, world, slots, int(sim.number_photons))
    local = Sim.from_buffer_copy(sim)
    local.number_photons = n
    with Simulation(local, seed=seed, slots=count, slot_begin=begin, device=device, **opts) as run:
        res = run.run()
        S = int(sim.num_sds)
        if replay:
            run.replay()
            rows = [run.rows(s)[0].copy() for s in range(1, S + 1)]
            weights = [r[:, 0].copy() for r in rows]
            a_rz, a0_z = (t.copy() for t in run.tallies())
        else:
            rows, a_rz, a0_z = None, None, None
            weights = [run.detections(s)[1].copy() for s in range(1, S + 1)]
        return Shard(n, weights, rows, a_rz, a0_z, int(res.steps))


def combine(shards: Sequence[Shard]) -> Shard:
    """Shards in rank (slot) order -> the whole run."""
    S = len(shards[0].weights)
    replay = shards[0].rows is not None
    rows = [np.concatenate([sh.rows[s] for sh in shards]) for s in range(S)] if replay else None
    weights = [np.concatenate([sh.weights[s] for sh in shards]) for s in range(S)]
    tal = [None, None]
    if shards[0].A_rz is not None:
        tal = [sum(sh.A_rz.astype(np.uint64) for sh in shards),
               sum(sh.A0_z.astype(np.uint64) for sh in shards)]
    return Shard(sum(sh.photons for sh in shards), weights, rows, tal[0], tal[1],
                 sum(sh.steps for sh in shards))


def _gather_rows(t, group, world, rank, dist, torch):
    """Variable-length float32 2-D tensors of every rank to rank 0, in rank order."""
    n = torch.tensor([t.shape[0]], dtype=torch.int64)
    sizes = [torch.zeros(1, dtype=torch.int64) for _ in range(world)]
    dist.all_gather(sizes, n, group=group)
    sizes = [int(v.item()) for v in sizes]
    width = t.shape[1] if t.dim() == 2 else 1
    mx = max(max(sizes), 1)
    pad = torch.zeros((mx, width), dtype=torch.float32)
    pad[:t.shape[0]] = t.reshape(-1, width)
    bufs = [torch.zeros((mx, width), dtype=torch.float32) for _ in range(world)] if rank == 0 else None
    dist.gather(pad, bufs, dst=0, group=group)
    if rank != 0:
        return None
    return [b[:k].numpy().reshape((k,) + tuple(t.shape[1:])) for b, k in zip(bufs, sizes)]


def gather_to_rank0(local: Shard, group=None) -> Optional[Shard]:
    """Every rank calls this once, in the same order, after its shard is
    done; rank 0 gets the whole run, the others None.  The arrays are host
    arrays, so `group` must be a gloo group (under NCCL:
    dist.new_group(backend="gloo")).  Tallies are summed
    with one all-reduce of int64 quanta (below 2^63 for any run this
    library can hold), rows and weights gathered in rank order."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    S = len(local.weights)
    meta = torch.tensor([local.photons, local.steps], dtype=torch.int64)
    dist.all_reduce(meta, group=group)
    tallies = [None, None]
    if local.A_rz is not None:
        flat = torch.from_numpy(np.concatenate([local.A_rz.ravel(), local.A0_z.ravel()])
                                .astype(np.int64))
        dist.all_reduce(flat, group=group)
        k = local.A_rz.size
        tallies = [flat[:k].numpy().astype(np.uint64).reshape(local.A_rz.shape),
                   flat[k:].numpy().astype(np.uint64).reshape(local.A0_z.shape)]
    weights, rows = [], [] if local.rows is not None else None
    for s in range(S):
        g = _gather_rows(torch.from_numpy(np.ascontiguousarray(local.weights[s])).reshape(-1, 1),
                         group, world, rank, dist, torch)
        if rank == 0:
            weights.append(np.concatenate([x.reshape(-1) for x in g]))
        if local.rows is not None:
            g = _gather_rows(torch.from_numpy(np.ascontiguousarray(local.rows[s])), group, world,
                             rank, dist, torch)
            if rank == 0:
                rows.append(np.concatenate(g))
    if rank != 0:
        return None
    return Shard(int(meta[0]), weights, rows, tallies[0], tallies[1], int(meta[1]))


def gather_device(out: dict, steps: int = 0, group=None) -> Optional[Shard]:
    """The combine of a multi-GPU job over the ranks' device tensors.

    Every rank calls this once, in the same order, with its own
    Simulation.device_outputs() (or tensors of the same layout: `records`
    (D, 10) float32 words, weight in word 3; `rows` (D, L+2) float32 or
    None; `A_rz`, `A0_z` int64 or None; `detected` per SDS; `photons`), all
    on one device per rank -- GPU tensors under NCCL, CPU tensors under gloo.
      * A_rz, A0_z: one all-reduce (SUM) of the int64 views of the u64
        quanta -- two's-complement sums are the u64 sums bit for bit;
      * per-SDS counts, photons and steps: one all-gather;
      * rows (without a replay, the records' weights): one all-gather of
        every rank's D entries, padded to the largest D.
    Rank 0 gets the whole run as host arrays in rank (= slot) order, the
    photon order of one run over all slots; the other ranks get None."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    dev = out["records"].device
    S = len(out["detected"])
    meta = torch.tensor(list(out["detected"]) + [int(out["photons"]), int(steps)],
                        dtype=torch.int64, device=dev)
    metas = [torch.empty_like(meta) for _ in range(world)]
    dist.all_gather(metas, meta, group=group)
    counts = torch.stack(metas).cpu().numpy()  # (world, S + 2)
    replay = out["rows"] is not None
    flat = None
    if replay:
        flat = torch.cat([out["A_rz"].reshape(-1), out["A0_z"].reshape(-1)]).to(torch.int64)
        dist.all_reduce(flat, group=group)
    data = out["rows"] if replay else out["records"][:, 3:4]
    D = int(data.shape[0])
    if D != int(counts[rank, :S].sum()):
        raise ValueError(f"rank {rank}: {D} entries but {counts[rank, :S].sum()} detections")
    dmax = max(int(counts[:, :S].sum(axis=1).max()), 1)
    pad = torch.zeros((dmax, data.shape[1]), dtype=torch.float32, device=dev)
    pad[:D] = data
    bufs = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(bufs, pad, group=group)
    if rank != 0:
        return None
    host = [b.cpu().numpy() for b in bufs]
    per_sds = []
    for s in range(S):
        parts = []
        for r in range(world):
            off = int(counts[r, :s].sum())
            parts.append(host[r][off:off + int(counts[r, s])])
        per_sds.append(np.concatenate(parts))
    tallies = [None, None]
    if replay:
        k = out["A_rz"].numel()
        f = flat.cpu().numpy().astype(np.uint64)
        tallies = [f[:k].reshape(tuple(out["A_rz"].shape)), f[k:].reshape(tuple(out["A0_z"].shape))]
    rows = per_sds if replay else None
    weights = [r[:, 0].copy() for r in per_sds]
    return Shard(int(counts[:, S].sum()), weights, rows, tallies[0], tallies[1],
                 int(counts[:, S + 1].sum()))


def write_outputs(sim: Sim, run: Shard, directory: str, output_txt: str, flags: int,
                  sim_s: float = 0.0, replay_s: float = 0.0, gpu_name: str = "",
                  grid: Optional[tuple] = None) -> None:
    """The reference's files for a combined run (mcml_write_host_outputs)."""
    lib = load_library()
    S = int(sim.num_sds)
    L = int(sim.num_layers)
    det = np.array([len(w) for w in run.weights], np.uint64)
    if run.rows is not None:
        # FP64 sums over the rows in photon order, as a single run sums them
        wsum = np.array([_ordered_sum(r[:, 0]) for r in run.rows])
        rows = [np.ascontiguousarray(r, np.float32).reshape(-1, L + 2) for r in run.rows]
        ptrs = (C.c_void_p * S)(*[r.ctypes.data for r in rows])
    else:
        wsum = np.array([_ordered_sum(w) for w in run.weights])
        rows, ptrs = None, None
    d = HostData()
    d.photons = run.photons
    d.detected = det.ctypes.data
    d.weight_sum = wsum.ctypes.data
    d.rows = C.cast(ptrs, C.c_void_p) if ptrs is not None else None
    if run.A_rz is not None:
        arz = np.ascontiguousarray(run.A_rz, np.uint64)
        a0z = np.ascontiguousarray(run.A0_z, np.uint64)
        d.A_rz, d.A0_z = arz.ctypes.data, a0z.ctypes.data
    if grid is not None:
        d.grid_nr, d.grid_nz, d.grid_dr, d.grid_dz = grid
    d.gpu_name = gpu_name.encode()
    _check(lib.mcml_write_host_outputs(C.byref(sim), C.byref(d), os.fsencode(directory),
                                       os.fsencode(output_txt), flags, sim_s, replay_s),
           "mcml_write_host_outputs")


def _ordered_sum(w: np.ndarray) -> float:
    """Left-to-right FP64 sum, the order the library's writer adds in
    (a cumulative sum accumulates sequentially; np.sum is pairwise)."""
    w = np.asarray(w, np.float64).reshape(-1)
    return float(np.cumsum(w)[-1]) if w.size else 0.0
