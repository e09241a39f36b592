"""Dirichlet air on the device (fc_set_air_model, FC_AIR_DIRICHLET) against the FP64
restatement (oracle/fluid_oracle.c, pinned by the hydrostatic free-surface known answer in
tests/test_dirichlet.py). The reference has no such model, so parity is with the restatement.

Tolerances: FP64 device vs FP64 restatement: iterations within three (reduction order can move
a restart near the max-norm threshold), velocities within 1e-8 of their scale, pressure within
1e-7 relative. FP32 at a 1e-6 relative residual vs the restatement at 1e-12: 1e-4 of scale.
"""
import dataclasses

import numpy as np
import pytest

from fluidsim_b200 import FluidGrid, ProjectionBatch, scenes

pytestmark = pytest.mark.gpu


def _dirichlet(scene):
    return dataclasses.replace(scene, air_model="dirichlet")


def _device(scene, precision):
    g = FluidGrid(scene.width, scene.height, scene.cell_size, precision)
    scenes.upload_scene(g, scene)
    return g


def _restatement(oracle, scene, tolerance=1e-6, relative=0.0, gravity=False):
    o = oracle.OracleGrid(scene.width, scene.height, scene.cell_size)
    o.upload(scene.density(), scene.u, scene.v, solid=scene.solid, air=oracle.air_mask(scene.fraction, scene.solid))
    if gravity:
        o.apply_gravity(scene.gravity, scene.dt)
    r = o.project(scene.dt, 2000, tolerance, relative_tolerance=relative)
    return (r,) + tuple(o.download())


def _scale(u, v):
    return max(1.0, float(np.abs(u).max()), float(np.abs(v).max()))


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


CASES = [((13, 9), 0), ((64, 64), 0), ((65, 37), 2), ((129, 65), 0), ((257, 193), 4), ((333, 251), 0), ((2, 67), 0)]


@pytest.mark.parametrize("size,obstacles", CASES)
def test_fp64_matches_the_restatement(oracle, size, obstacles):
    w, h = size
    s = _dirichlet(scenes.random_pool(w, h, seed=3 * w + h, fill=0.55, obstacles=obstacles))
    ro, uo, vo, po = _restatement(oracle, s)
    g = _device(s, "fp64")
    assert g.getAirModel() == "dirichlet"
    r = g.project(s.dt, 2000, 1e-6)
    out = g.download()
    assert r.converged == ro.converged and ro.converged
    assert abs(r.iterations - ro.iterations) <= 3, (r.iterations, ro.iterations)
    scale = _scale(uo, vo)
    assert np.abs(out.u - uo).max() <= 1e-8 * scale
    assert np.abs(out.v - vo).max() <= 1e-8 * scale
    assert _rel(out.pressure, po) <= 1e-7
    # Air holds zero pressure, and the reported divergence is the liquid's, bit for bit.
    air = oracle.air_mask(s.fraction, s.solid) != 0
    assert np.all(out.pressure[air] == 0.0)
    div = ((out.u[:, 1:] - out.u[:, :-1]) + (out.v[1:, :] - out.v[:-1, :])) / s.cell_size
    liquid = ~air if s.solid is None else (~air) & (s.solid == 0)
    assert r.max_divergence == float(np.abs(div[liquid]).max())


@pytest.mark.parametrize("size,obstacles", [((64, 64), 0), ((257, 193), 4), ((333, 251), 0)])
@pytest.mark.parametrize("precision", ["fp32", "mixed"])
def test_fp32_and_mixed_match_the_restatement(oracle, size, obstacles, precision):
    w, h = size
    s = _dirichlet(scenes.random_pool(w, h, seed=5 * w + h, fill=0.6, obstacles=obstacles))
    _, uo, vo, po = _restatement(oracle, s, 1e-12, relative=1e-12)
    g = _device(s, precision)
    r = g.project(s.dt, 2000, 1e-6, relative_tolerance=1e-6)
    out = g.download()
    assert r.solve_status == "converged" and r.residual_l2 <= 1.0001e-6 * r.rhs_l2
    scale = _scale(uo, vo)
    assert np.abs(out.u - uo).max() <= 1e-4 * scale
    assert np.abs(out.v - vo).max() <= 1e-4 * scale
    assert _rel(out.pressure, po) <= 1e-4


@pytest.mark.parametrize("precision,bar", [("fp64", 1e-10), ("fp32", 1e-5)])
def test_hydrostatic_free_surface_known_answer(precision, bar):
    """A liquid layer at rest with air above: rest is kept, air holds p = 0, and the liquid
    pressure is hydrostatic from the free surface, p_top = -g dx (rho_l + rho_a) / 2 and
    -rho_l g dx per row below (FP64 to 1e-10 relative; FP32 storage to 1e-5)."""
    w, h, top, dx, dt, gy, rl, ra = 40, 48, 19, 0.05, 0.01, -9.8, 1000.0, 1.0
    f = np.zeros((h, w))
    f[: top + 1] = 1.0
    s = scenes.Scene(w, h, dx, dt, rl, ra, f, np.zeros((h, w + 1)), np.zeros((h + 1, w)), gravity=gy,
                     air_model="dirichlet")
    g = _device(s, precision)
    g.applyGravity(dt)
    r = g.project(dt, 400, 1e-9)
    out = g.download()
    assert r.solve_status in ("converged", "no_work")
    p_top = -gy * dx * (rl + ra) / 2.0
    expected = np.array([p_top - (top - y) * rl * gy * dx for y in range(top + 1)])
    assert np.abs(out.pressure[: top + 1] - expected[:, None]).max() <= bar * np.abs(expected).max()
    assert np.all(out.pressure[top + 1:] == 0.0)
    assert np.abs(out.v[1: top + 1]).max() <= bar * abs(gy * dt) * 10
    assert np.abs(out.u).max() <= bar * abs(gy * dt) * 10


def test_dam_break_with_obstacles_fp64_matches_the_restatement(oracle):
    """The 1024 x 1024 dam break with 16 obstacles and Dirichlet air, the boundary its workload
    states, after gravity."""
    s = _dirichlet(scenes.dam_break(1024, 1024, seed=11, obstacles=16, velocity=1.0))
    ro, uo, vo, po = _restatement(oracle, s, gravity=True)
    g = _device(s, "fp64")
    g.applyGravity(s.dt)
    r = g.project(s.dt, 400, 1e-6)
    out = g.download()
    assert r.converged and ro.converged
    assert abs(r.iterations - ro.iterations) <= 3, (r.iterations, ro.iterations)
    scale = _scale(uo, vo)
    assert np.abs(out.u - uo).max() <= 1e-8 * scale
    assert np.abs(out.v - vo).max() <= 1e-8 * scale
    assert _rel(out.pressure, po) <= 1e-7


def test_batch_of_both_air_models_equals_single_grids():
    """A batch may hold gas and Dirichlet grids: each grid's result is its single-grid result,
    bit for bit (the air model travels in the grid's own descriptor)."""
    raw = [scenes.random_pool(96, 80, seed=1, fill=0.5, obstacles=2), scenes.random_pool(130, 70, seed=2, fill=0.6),
           scenes.random_pool(200, 150, seed=3, fill=0.4)]
    sample = [_dirichlet(raw[0]), raw[1], _dirichlet(raw[2])]
    singles = []
    for s in sample:
        g = _device(s, "fp32")
        r = g.project(s.dt, 400, 1e-6)
        singles.append((r, g.download()))
    grids = [_device(s, "fp32") for s in sample]
    batch = ProjectionBatch(grids)
    results = batch.project([s.dt for s in sample], 400, 1e-6)
    for (r1, o1), r2, g in zip(singles, results, grids):
        o2 = g.download()
        assert r1.iterations == r2.iterations
        assert np.array_equal(o1.u, o2.u) and np.array_equal(o1.v, o2.v) and np.array_equal(o1.pressure, o2.pressure)
    batch.destroy()


def test_checkpoint_keeps_the_air_model_and_continues_exactly():
    s = _dirichlet(scenes.random_pool(80, 64, seed=9, fill=0.5, obstacles=1))
    a = _device(s, "fp32")
    a.setGravityY(-9.8)
    a.step(s.dt, 200, 1e-6)
    meta, payload = a.saveCheckpoint()
    assert meta["air_model"] == 1
    b = FluidGrid(s.width, s.height, s.cell_size, "fp32")
    b.loadCheckpoint(meta, payload)
    assert b.getAirModel() == "dirichlet"
    for _ in range(2):
        ra, rb = a.step(s.dt, 200, 1e-6), b.step(s.dt, 200, 1e-6)
        assert ra.iterations == rb.iterations
    sa, sb = a.download(), b.download()
    assert np.array_equal(sa.u, sb.u) and np.array_equal(sa.pressure, sb.pressure)


def test_switching_back_to_gas_gives_the_gas_projection():
    s = scenes.random_pool(100, 90, seed=4, fill=0.5)
    ref = _device(s, "fp64")
    r0 = ref.project(s.dt, 300, 1e-6)
    g = _device(_dirichlet(s), "fp64")
    g.project(s.dt, 300, 1e-6)
    g.setAirModel("gas")
    scenes.upload_scene(g, s)
    r1 = g.project(s.dt, 300, 1e-6)
    assert r0.iterations == r1.iterations
    a, b = ref.download(), g.download()
    assert np.array_equal(a.u, b.u) and np.array_equal(a.pressure, b.pressure)


@pytest.mark.parametrize("transport", ["semi_lagrangian", "plic"])
def test_dam_break_steps_with_dirichlet_air(transport):
    """Forty whole steps of a 256 x 256 dam break with obstacles and Dirichlet air: every
    projection meets the reference's stop rule (accepted, none at the iteration cap)."""
    s = _dirichlet(scenes.dam_break(256, 256, seed=5, obstacles=4, velocity=0.0))
    g = _device(s, "fp32")
    g.setTransport(transport)
    for _ in range(40):
        r = g.step(s.dt, 200, 1e-6)
        assert r.accepted() and r.solve_status == "converged", r
        assert r.iterations < 200


def _extend_restatement(u, v, fraction, solid, layers=4):
    """The velocity extension restated in numpy (FP64): layer 0 are the walls, the faces of
    solid cells and of liquid cells (f > 0.5); each layer gives every unknown face beside known
    faces of earlier layers their mean; faces still unknown after the last layer are zero."""
    h, w = fraction.shape
    solid = np.zeros((h, w), bool) if solid is None else solid != 0
    liquid = (fraction > 0.5) & ~solid
    u, v = u.copy(), v.copy()
    ku = np.full(u.shape, 255, dtype=int)
    kv = np.full(v.shape, 255, dtype=int)
    for y in range(h):
        for x in range(w + 1):
            cells = [c for c in (x - 1, x) if 0 <= c < w]
            if x in (0, w) or any(solid[y, c] or liquid[y, c] for c in cells):
                ku[y, x] = 0
    for y in range(h + 1):
        for x in range(w):
            cells = [c for c in (y - 1, y) if 0 <= c < h]
            if y in (0, h) or any(solid[c, x] or liquid[c, x] for c in cells):
                kv[y, x] = 0
    for layer in range(1, layers + 1):
        for val, known in ((u, ku), (v, kv)):
            ny, nx = val.shape
            before = known.copy()
            for y in range(ny):
                for x in range(nx):
                    if before[y, x] != 255:
                        continue
                    vals = [val[qy, qx] for qx, qy in ((x - 1, y), (x + 1, y), (x, y - 1), (x, y + 1))
                            if 0 <= qx < nx and 0 <= qy < ny and before[qy, qx] < layer]
                    if vals:
                        val[y, x] = sum(vals) / len(vals)
                        known[y, x] = layer
                    elif layer == layers:
                        val[y, x] = 0.0
    return u, v


def test_air_velocity_extension_matches_its_restatement():
    """fc_extend_air_velocity against the numpy restatement, bit for bit in FP64 (the same sums
    in the same neighbour order), on a pool with obstacles and a wavy surface."""
    s = _dirichlet(scenes.random_pool(37, 29, seed=8, fill=0.4, obstacles=2))
    s.fraction[12, ::3] = 1.0  # liquid drops above the surface
    g = _device(s, "fp64")
    g.extendAirVelocity()
    out = g.download()
    u, v = _extend_restatement(s.u, s.v, s.fraction, s.solid)
    assert np.array_equal(out.u, u)
    assert np.array_equal(out.v, v)
