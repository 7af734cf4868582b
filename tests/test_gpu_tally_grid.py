"""Absorbance tallies on a grid other than the reference's fixed 1000 x 500
cells of 0.01 cm (mcml_opts.grid_*, CLI `-grid`).

The grid only decides where a replayed drop is binned: the first drop of a
detected photon goes to A0_z, every later one to A_rz, and a drop beyond the
grid's last cell lands in that cell.  So, per SDS, the u64 totals of A0_z
and of A_rz are the same sums of the same integer drops on every grid and
must equal the reference grid's exactly, while the walk, the detections and
the pathlength rows do not depend on the grid at all."""
import numpy as np
import pytest

import mcml_gpu_b200 as m
from conftest import load_case


def _run(sim, grid):
    with m.Simulation(sim, seed=4321, grid=grid) as run:
        res = run.run()
        run.replay()
        rows = [run.rows(s)[0].copy() for s in range(1, int(sim.num_sds) + 1)]
        a_rz, a0_z = run.tallies()
        return res, rows, a_rz, a0_z, run.grid


@pytest.mark.gpu
@pytest.mark.parametrize("grid", [(200, 200, 0.005, 0.005), (37, 11, 0.013, 0.029)])
def test_tally_totals_do_not_depend_on_the_grid(gpu_available, grid):
    sim = load_case("ring5")
    sim.number_photons = 1_000_000
    ref, ref_rows, ref_arz, ref_a0z, ref_grid = _run(sim, None)
    got, rows, arz, a0z, got_grid = _run(sim, grid)
    S = int(sim.num_sds)
    assert ref_grid == (1000, 500, 0.01, 0.01)
    assert got_grid[:2] == grid[:2]
    assert arz.shape == (S, grid[1], grid[0]) and a0z.shape == (S, grid[1])
    assert list(got.detected[:S]) == list(ref.detected[:S])
    assert sum(got.detected[:S]) > 100
    for s in range(S):
        assert rows[s].tobytes() == ref_rows[s].tobytes()
        assert int(a0z[s].sum()) == int(ref_a0z[s].sum())
        assert int(arz[s].sum()) == int(ref_arz[s].sum())
        if got.detected[s]:
            assert int(arz[s].sum()) > 0
    # the coarse grid clamps: its last row and column hold what lies beyond
    if grid[0] * grid[2] < 1.0:
        assert int(arz[:, :, -1].sum()) > 0
