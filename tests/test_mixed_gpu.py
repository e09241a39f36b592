"""Mixed precision: the smoothing kernels of the coarse multigrid levels read FP16 copies of the
face weights (scaled per level), while the fine level, every vector, the PCG operator and the
smoothing arithmetic stay FP32 and the reductions FP64. The preconditioner is approximate, so
the bar is the FP32 path's own: the same error against the FP64 restatement solved to 1e-12,
and convergence in about as many iterations."""
import numpy as np
import pytest

from fluidsim_b200 import FluidGrid, ProjectionBatch, scenes

pytestmark = pytest.mark.gpu


def _grid(scene, precision):
    g = FluidGrid(scene.width, scene.height, scene.cell_size, precision=precision)
    scenes.upload_scene(g, scene)
    return g


def _oracle_solution(oracle, s):
    o = oracle.OracleGrid(s.width, s.height, s.cell_size)
    o.upload(s.density(), s.u, s.v, None, s.solid)
    o.project(s.dt, 1000, 1e-12, relative_tolerance=1e-12)
    return o.download()


CASES = [
    ("pool64", lambda: scenes.random_pool(64, 64, seed=3, fill=0.55, cell_size=1.0 / 64)),
    ("pool257x193", lambda: scenes.random_pool(257, 193, seed=5, fill=0.6, cell_size=1.0 / 257)),
    ("pool333x251_obstacles", lambda: scenes.random_pool(333, 251, seed=8, fill=0.5, obstacles=6,
                                                         cell_size=1.0 / 333)),
    ("dam512", lambda: scenes.dam_break(512, 512, seed=2, obstacles=8, velocity=1.0)),
]


@pytest.mark.parametrize("name,make", CASES)
def test_mixed_error_matches_fp32(oracle, name, make):
    s = make()
    uo, vo, po = _oracle_solution(oracle, s)
    scale = max(np.abs(uo).max(), np.abs(vo).max())
    errors, iterations = {}, {}
    for precision in ("fp32", "mixed"):
        g = _grid(s, precision)
        r = g.project(s.dt, 500, 1e-6, relative_tolerance=1e-6)
        out = g.download()
        assert r.solve_status == "converged", (precision, r)
        assert r.residual_l2 <= 1.0001e-6 * r.rhs_l2
        errors[precision] = max(np.abs(out.u - uo).max(), np.abs(out.v - vo).max()) / scale
        iterations[precision] = r.iterations
    # FP32 at a 1e-6 relative residual against the FP64 solution at 1e-12: 1e-4 of the scale.
    assert errors["mixed"] <= 1e-4 and errors["fp32"] <= 1e-4
    assert iterations["mixed"] <= iterations["fp32"] + 2


def test_mixed_batch_equals_single():
    batch_scenes = scenes.uneven_batch(6, seed=21, min_side=64, max_side=300)
    singles = []
    for s in batch_scenes:
        g = _grid(s, "mixed")
        singles.append((g.project(s.dt, 300, 1e-6, relative_tolerance=1e-6), g.download()))
    grids = [_grid(s, "mixed") for s in batch_scenes]
    b = ProjectionBatch(grids)
    results = b.project([s.dt for s in batch_scenes], 300, 1e-6, relative_tolerance=1e-6)
    for (r1, o1), r2, g in zip(singles, results, grids):
        o2 = g.download()
        assert r1.iterations == r2.iterations
        assert np.array_equal(o1.u, o2.u) and np.array_equal(o1.v, o2.v) and np.array_equal(o1.pressure, o2.pressure)
    b.destroy()


def test_mixed_weight_scale_covers_extreme_densities(oracle):
    """Densities far from 1 (1e-4 and 10 here) still map every weight into FP16's range."""
    s = scenes.random_pool(96, 80, seed=4, fill=0.5, liquid_density=10.0, gas_density=1e-4, cell_size=1.0 / 96)
    uo, vo, _ = _oracle_solution(oracle, s)
    g = _grid(s, "mixed")
    r = g.project(s.dt, 500, 1e-6, relative_tolerance=1e-6)
    out = g.download()
    assert r.solve_status == "converged"
    scale = max(np.abs(uo).max(), np.abs(vo).max())
    assert max(np.abs(out.u - uo).max(), np.abs(out.v - vo).max()) <= 1e-4 * scale


def _viscous_restatement(oracle, s):
    """The variable-viscosity step in the FP64 restatement: viscosity to the reference's 1e-4
    relative residual, then the projection to 1e-12."""
    material = oracle.viscosity_material(s.liquid_mass + s.gas_mass, [s.liquid_density] * len(s.liquid_mass)
                                         + [s.gas_density] * len(s.gas_mass),
                                         s.liquid_viscosity + s.gas_viscosity, s.cell_size)
    it, u, v, _ = oracle.Viscosity(s.width, s.height).solve(s.u, s.v, material, s.dt, s.cell_size, 1e-4)
    o = oracle.OracleGrid(s.width, s.height, s.cell_size)
    o.upload(s.density(), u, v, None, s.solid)
    o.project(s.dt, 2000, 1e-12, relative_tolerance=1e-12)
    return it, (u, v), o.download()


@pytest.mark.parametrize("size", [(96, 80), (128, 128)], ids=lambda s: f"{s[0]}x{s[1]}")
def test_viscous_blob_against_restatement(oracle, size):
    """The variable-viscosity workload (fractal liquid blob, 1000:1 densities, viscosity
    log-uniform in [1e-3, 10] from two liquid components) at small sizes. FP64 on the device
    follows the restatement step by step; the viscosity solve is the same FP32 code in plain FP32
    and in mixed precision, and both end close to the FP64 step."""
    w, h = size
    s = scenes.viscous_blob(w, h, seed=9)
    it_o, (uv_o, vv_o), (uo, vo, _) = _viscous_restatement(oracle, s)
    scale = max(np.abs(uo).max(), np.abs(vo).max())

    g = _grid(s, "fp64")
    it, _ = g.applyViscosity(s.dt, 1e-4, 4000)
    mid = g.download()
    assert it == it_o
    assert max(np.abs(mid.u - uv_o).max(), np.abs(mid.v - vv_o).max()) <= 1e-10 * scale
    r = g.project(s.dt, 2000, 1e-12, relative_tolerance=1e-12)
    out = g.download()
    assert r.solve_status == "converged"
    assert max(np.abs(out.u - uo).max(), np.abs(out.v - vo).max()) <= 1e-8 * scale

    runs = {}
    for precision in ("fp32", "mixed"):
        g = _grid(s, precision)
        it, _ = g.applyViscosity(s.dt, 1e-4, 4000)
        mid = g.download()
        r = g.project(s.dt, 500, 1e-6, relative_tolerance=1e-6)
        out = g.download()
        assert r.solve_status == "converged" and r.residual_l2 <= 1.0001e-6 * r.rhs_l2, (precision, r)
        runs[precision] = (it, mid, max(np.abs(out.u - uo).max(), np.abs(out.v - vo).max()) / scale)
    (it32, mid32, err32), (itm, midm, errm) = runs["fp32"], runs["mixed"]
    assert it32 == itm == it_o
    assert np.array_equal(mid32.u, midm.u) and np.array_equal(mid32.v, midm.v)
    # FP32 viscosity and a 1e-6 projection against the FP64 step: 1e-4 of the scale.
    assert err32 <= 1e-4 and errm <= 1e-4
