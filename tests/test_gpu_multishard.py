"""Shards of one run walked one after another on one GPU (slot ranges as
a multi-GPU run splits them), combined, and written with the host writer:
every output file equals, byte for byte, what one run over all slots
writes with the same seed.  Covers the combination step of the
multi-GPU path without several GPUs."""
import os
import tempfile
from pathlib import Path

import pytest

from conftest import load_case

import mcml_gpu_b200 as m
from mcml_gpu_b200.distributed import combine, run_shard, write_outputs

SEED = 777


@pytest.mark.gpu
@pytest.mark.parametrize("case,photons,slots,world,binary", [
    ("ring5", 1_200_000, 150_000, 3, True),
    ("fiber3", 2_000_003, 250_000, 4, False),   # remainder slots straddle a shard
])
def test_combined_shards_write_the_single_run_files(case, photons, slots, world, binary,
                                                    gpu_available):
    sim = load_case(case)
    sim.number_photons = photons
    flags = m.OUT_REPLAY | m.OUT_ABSORBANCE | m.OUT_PATHLENGTH | m.OUT_AVERAGE_PL
    if binary:
        flags |= m.OUT_BINARY
    name = m.device_info(0).name.decode()
    with tempfile.TemporaryDirectory() as one, tempfile.TemporaryDirectory() as many:
        with m.Simulation(sim, seed=SEED, slots=slots) as run:
            first = run.run()
            run.replay()
            run.write_outputs(one, os.path.join(one, "output.txt"), flags)
        shards = [run_shard(sim, rank=r, world=world, seed=SEED, slots=slots)
                  for r in range(world)]
        whole = combine(shards)
        assert whole.photons == photons and whole.steps == first.steps
        write_outputs(sim, whole, many, os.path.join(many, "output.txt"), flags, gpu_name=name)
        files = sorted(p.name for p in Path(one).iterdir())
        assert files == sorted(p.name for p in Path(many).iterdir())
        for f in files:
            assert (Path(one) / f).read_bytes() == (Path(many) / f).read_bytes(), f
