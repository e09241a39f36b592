"""Autotuning of the multigrid schedule: the tail threshold changes which kernels run (one-block
shared-memory tail or strip kernels), not the method, so every threshold must give the same
projection to rounding."""
import numpy as np
import pytest

from fluidsim_b200 import FluidGrid, ProjectionBatch, scenes

pytestmark = pytest.mark.gpu


def _grid(scene, precision):
    g = FluidGrid(scene.width, scene.height, scene.cell_size, precision=precision)
    scenes.upload_scene(g, scene)
    return g


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_tail_threshold_does_not_change_the_solution(precision):
    s = scenes.random_pool(300, 220, seed=12, fill=0.6, obstacles=4, cell_size=1.0 / 300)
    outs = {}
    for cells in (256, 1024, 4096):
        g = _grid(s, precision)
        g.setTailCells(cells)
        r = g.project(s.dt, 400, 1e-8 if precision == "fp64" else 1e-6, relative_tolerance=1e-8 if precision == "fp64" else 1e-6)
        assert r.solve_status == "converged"
        outs[cells] = (r, g.download())
    scale = max(np.abs(outs[1024][1].u).max(), np.abs(outs[1024][1].v).max())
    bar = 1e-9 if precision == "fp64" else 2e-5
    for cells in (256, 4096):
        assert abs(outs[cells][0].iterations - outs[1024][0].iterations) <= 2
        assert np.abs(outs[cells][1].u - outs[1024][1].u).max() <= bar * scale
        assert np.abs(outs[cells][1].v - outs[1024][1].v).max() <= bar * scale


def test_autotune_picks_a_candidate_and_keeps_the_state():
    s = scenes.dam_break(512, 384, seed=3, obstacles=4, velocity=1.0)
    g = _grid(s, "fp32")
    before = g.download()
    cells, ms = g.autotune(3)
    assert cells in (256, 1024, 4096) and ms > 0.0
    after = g.download()
    for name in ("u", "v", "pressure", "liquid_fraction"):
        assert np.array_equal(getattr(before, name), getattr(after, name))
    r = g.project(s.dt, 300, 1e-6, relative_tolerance=1e-6)
    assert r.solve_status == "converged"


def test_batch_autotune_then_batch_equals_single():
    batch_scenes = scenes.uneven_batch(5, seed=31, min_side=64, max_side=400)
    grids = [_grid(s, "fp32") for s in batch_scenes]
    b = ProjectionBatch(grids)
    cells, _ = b.autotune(3)
    assert cells in (256, 1024, 4096)
    results = b.project([s.dt for s in batch_scenes], 300, 1e-6, relative_tolerance=1e-6)
    for s, g, r in zip(batch_scenes, grids, results):
        single = _grid(s, "fp32")
        single.setTailCells(cells)
        rs = single.project(s.dt, 300, 1e-6, relative_tolerance=1e-6)
        assert rs.iterations == r.iterations
        a, c = single.download(), g.download()
        assert np.array_equal(a.u, c.u) and np.array_equal(a.pressure, c.pressure)
    b.destroy()
