"""Parity at the sizes the bench measures, against the reference engine itself.

The reference's own UniformCPU engine (FluidSim/UniformCPU/FluidGridCPU.cpp and
PressureMultigrid.cpp, compiled from its sources into oracle/_ref) projects the same seeded
scenes as the device: the 1024 x 1024 dam break, the 2048 x 2048 headline scene, and grids of
the uneven batch. Scenes with obstacles (an extension the reference has no counterpart for) are
checked against the FP64 restatement instead. The device's own face weights, inverse diagonal
and divergence are checked against the fixtures the reference wrote.

Tolerances, stated per test:
  * FP64 device vs FP64 reference at the reference's rule: iterations within one, velocities
    within 1e-8 of their scale, pressure within 1e-7 relative (only reduction order differs);
  * FP32 device vs the FP64 reference solved to max |div| <= 1e-7: velocities within 1e-4 of
    their scale, pressure within 1e-4 relative.
"""
import dataclasses
import glob
import os

import numpy as np
import pytest

from conftest import GOLDEN, golden
from fluidsim_b200 import FluidGrid, ProjectionBatch, scenes

pytestmark = pytest.mark.gpu


def _threads():
    try:
        return min(8, len(os.sched_getaffinity(0)))
    except Exception:
        return min(8, os.cpu_count() or 1)


@pytest.fixture(scope="module")
def ref(oracle):
    assert oracle.reference_available(), "the reference engine (oracle/_ref) must be built"
    oracle.set_reference_threads(_threads())
    return oracle


def _reference_solution(oracle, scene, tolerance, max_iterations=400, gravity=True):
    g = oracle.ReferenceGrid(scene.width, scene.height, scene.cell_size, scene.liquid_density, scene.gas_density)
    g.set_gravity(scene.gravity)
    g.upload(scene.fraction, scene.u, scene.v, None, scene.liquid_mass[0], scene.gas_mass[0])
    if gravity:
        g.apply_gravity(scene.dt)
    r = g.project(scene.dt, max_iterations, tolerance)
    _, u, v, p = g.download()
    return r, u, v, p


def _device(scene, precision, obstacles=True):
    if not obstacles:
        scene = dataclasses.replace(scene, solid=None)
    g = FluidGrid(scene.width, scene.height, scene.cell_size, precision)
    scenes.upload_scene(g, scene)
    return g


def _scale(u, v):
    return max(1.0, float(np.abs(u).max()), float(np.abs(v).max()))


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _check_fp64(r, out, expected, u, v, p):
    # Same algorithm in FP64, different reduction order: iterations within one, velocities 1e-8
    # of their scale, pressure 1e-7 relative.
    assert r.converged and expected.converged
    assert abs(r.iterations - expected.iterations) <= 1, (r.iterations, expected.iterations)
    scale = _scale(u, v)
    assert np.abs(out.u - u).max() <= 1e-8 * scale
    assert np.abs(out.v - v).max() <= 1e-8 * scale
    assert _rel(out.pressure, p) <= 1e-7


def _check_fp32(out, u, v, p):
    # FP32 against the FP64 reference at max |div| <= 1e-7: 1e-4 of the velocity scale (the
    # reference's own FP32-vs-FP64 precedent is 5e-3 absolute, FluidGridWebGPUTests.cpp:270-305).
    scale = _scale(u, v)
    assert np.abs(out.u - u).max() <= 1e-4 * scale
    assert np.abs(out.v - v).max() <= 1e-4 * scale
    assert _rel(out.pressure, p) <= 1e-4


# ---------------------------------------------------------------------------------------------
# The 1024 x 1024 dam break (config 2's scene) and the 2048 x 2048 headline scene
# ---------------------------------------------------------------------------------------------

@pytest.mark.parametrize("size", [1024, 2048])
def test_dam_break_fp64_equals_the_reference_engine(ref, size):
    """Device FP64 against FluidGridCPU::project under the reference's own rule
    (max |div u| <= 1e-6, FluidGridCPU.cpp:1093) on the dam break with U[-1, 1] velocities."""
    s = scenes.dam_break(size, size, seed=1234, obstacles=0, velocity=1.0)
    expected, u, v, p = _reference_solution(ref, s, 1e-6)
    g = _device(s, "fp64")
    g.applyGravity(s.dt)
    r = g.project(s.dt, 400, 1e-6)
    _check_fp64(r, g.download(), expected, u, v, p)


@pytest.mark.parametrize("size", [1024, 2048])
def test_dam_break_fp32_against_the_reference_engine(ref, size):
    """The FP32 drop-in under both stop rules against the reference's FP64 solve at 1e-7:
    the reference's own rule (the bench's headline setting) and the 1e-6 relative residual."""
    s = scenes.dam_break(size, size, seed=1234, obstacles=0, velocity=1.0)
    expected, u, v, p = _reference_solution(ref, s, 1e-7)
    assert expected.converged
    for relative in (False, True):
        g = _device(s, "fp32")
        g.applyGravity(s.dt)
        if relative:
            r = g.project(s.dt, 400, 1e-6, relative_tolerance=1e-6)
            assert r.solve_status == "converged" and r.residual_l2 <= 1.0001e-6 * r.rhs_l2
        else:
            r = g.project(s.dt, 400, 1e-6)
            # The solver meets the reference's rule on its FP64 residual; the FP32 face
            # velocities can only hold the divergence to their own rounding.
            assert r.solve_status == "converged" and r.accepted()
        _check_fp32(g.download(), u, v, p)


def test_dam_break_with_obstacles_fp64_equals_the_restatement(oracle):
    """Config 2's scene with its 16 circular obstacles (no reference counterpart): device FP64
    against the FP64 restatement at the reference's rule; iterations within three (a restart
    near the max-norm threshold can move by two), velocities 1e-8 of scale."""
    s = scenes.dam_break(1024, 1024, seed=11, obstacles=16, velocity=1.0)
    o = oracle.OracleGrid(s.width, s.height, s.cell_size)
    o.upload(s.density(), s.u, s.v, None, solid=s.solid)
    o.apply_gravity(s.gravity, s.dt)
    ro = o.project(s.dt, 400, 1e-6)
    uo, vo, po = o.download()
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


# ---------------------------------------------------------------------------------------------
# The uneven batch (config 4), grid by grid
# ---------------------------------------------------------------------------------------------

def _batch_sample(count=16):
    """16 grids of the 256-grid uneven batch: the smallest, the largest, the most elongated,
    and 13 more spread over the batch by size."""
    all_scenes = scenes.uneven_batch(256, seed=7)
    order = sorted(range(len(all_scenes)), key=lambda i: all_scenes[i].cells)
    aspect = max(range(len(all_scenes)),
                 key=lambda i: max(all_scenes[i].width, all_scenes[i].height) / min(all_scenes[i].width, all_scenes[i].height))
    picks = {order[0], order[-1], aspect}
    for k in np.linspace(0, len(order) - 1, count + 2)[1:-1]:
        if len(picks) >= count:
            break
        picks.add(order[int(k)])
    return [all_scenes[i] for i in sorted(picks)]


def test_uneven_batch_grids_equal_the_reference_engine(ref):
    """One batched FP64 projection of 16 grids of the uneven batch with their obstacles taken
    out, each grid against FluidGridCPU::project of the same grid."""
    sample = _batch_sample()
    grids = [_device(s, "fp64", obstacles=False) for s in sample]
    batch = ProjectionBatch(grids)
    results = batch.project([s.dt for s in sample], 400, 1e-6)
    for s, g, r in zip(sample, grids, results):
        expected, u, v, p = _reference_solution(ref, dataclasses.replace(s, solid=None), 1e-6, gravity=False)
        _check_fp64(r, g.download(), expected, u, v, p)
    batch.destroy()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_uneven_batch_grids_with_obstacles_equal_the_restatement(oracle, precision):
    """The same 16 grids with their obstacles, batched, against the FP64 restatement: FP64 at
    the reference's rule (iterations within three, 1e-8 of scale), FP32 at a 1e-6 relative
    residual against the restatement solved to 1e-12 relative (1e-4 of scale)."""
    sample = _batch_sample()
    grids = [_device(s, precision) for s in sample]
    batch = ProjectionBatch(grids)
    if precision == "fp64":
        results = batch.project([s.dt for s in sample], 400, 1e-6)
    else:
        results = batch.project([s.dt for s in sample], 400, 1e-6, relative_tolerance=1e-6)
    for s, g, r in zip(sample, grids, results):
        o = oracle.OracleGrid(s.width, s.height, s.cell_size)
        o.upload(s.density(), s.u, s.v, None, solid=s.solid)
        if precision == "fp64":
            ro = o.project(s.dt, 400, 1e-6)
        else:
            ro = o.project(s.dt, 2000, 1e-12, relative_tolerance=1e-12)
        uo, vo, po = o.download()
        out = g.download()
        scale = _scale(uo, vo)
        if precision == "fp64":
            assert r.converged == ro.converged
            assert abs(r.iterations - ro.iterations) <= 3, (s.width, s.height, r.iterations, ro.iterations)
            assert np.abs(out.u - uo).max() <= 1e-8 * scale
            assert np.abs(out.v - vo).max() <= 1e-8 * scale
        else:
            assert r.solve_status in ("converged", "no_work")
            assert np.abs(out.u - uo).max() <= 1e-4 * scale
            assert np.abs(out.v - vo).max() <= 1e-4 * scale
    batch.destroy()


# ---------------------------------------------------------------------------------------------
# The device's own coefficients and divergence against the reference's fixtures
# ---------------------------------------------------------------------------------------------

FIXTURES = sorted(glob.glob(os.path.join(GOLDEN, "project_*.npz")))


def _fixture_grid(d, precision):
    w, h = int(d["width"]), int(d["height"])
    s = scenes.Scene(w, h, float(d["cell_size"]), float(d["dt"]), float(d["liquid_density"]),
                     float(d["gas_density"]), d["fraction"], d["u_in"].astype(np.float64), d["v_in"].astype(np.float64))
    g = FluidGrid(w, h, s.cell_size, precision)
    g.setPreconditioner(str(d["preconditioner"]))
    scenes.upload_scene(g, s)
    return s, g


@pytest.mark.parametrize("path", FIXTURES, ids=os.path.basename)
def test_device_coefficients_are_the_references_bit_for_bit(path):
    """inv_u, inv_v and the inverse diagonal read back from the device (a1, a2): FP64 equal to
    the reference's arrays bit for bit; FP32 equal to the reference's weights rounded to float,
    and to the float inverse diagonal ((wl + wr) + wu) + wd, 1 / sum, in the reference's order."""
    d = golden(os.path.basename(path))
    _, g = _fixture_grid(d, "fp64")
    inv_u, inv_v, inv_d = g.downloadCoefficients()
    assert np.array_equal(inv_u, d["inv_u"])
    assert np.array_equal(inv_v, d["inv_v"])
    assert np.array_equal(inv_d, d["inv_diagonal"])

    _, g32 = _fixture_grid(d, "fp32")
    inv_u, inv_v, inv_d = g32.downloadCoefficients()
    fu, fv = d["inv_u"].astype(np.float32), d["inv_v"].astype(np.float32)
    assert np.array_equal(inv_u, fu.astype(np.float64))
    assert np.array_equal(inv_v, fv.astype(np.float64))
    total = ((fu[:, :-1] + fu[:, 1:]) + fv[:-1, :]) + fv[1:, :]
    with np.errstate(divide="ignore"):
        expected = np.where(total > 0, np.float32(1) / total, np.float32(0))
    assert np.array_equal(inv_d, expected.astype(np.float64))


@pytest.mark.parametrize("path", FIXTURES, ids=os.path.basename)
def test_max_divergence_is_the_references_quantity(path):
    """a12: the divergence the device reports is max |(du + dv) / dx| of its own final
    velocities (FluidGridCPU.cpp:1126-1152, recomputed on the host: bit for bit), meets the
    fixture's convergence flag, and lies within 10 % of the fixture's value. The value after
    the solve is the stopping residual itself, which reduction order moves by a few percent
    (the FP64 restatement differs from the fixtures by up to 7.5 %)."""
    d = golden(os.path.basename(path))
    s, g = _fixture_grid(d, "fp64")
    r = g.project(s.dt, int(d["max_iterations"]), float(d["tolerance"]))
    out = g.download()
    # The reference's association: ((u_right - u_left) + (v_down - v_up)) / dx.
    div = ((out.u[:, 1:] - out.u[:, :-1]) + (out.v[1:, :] - out.v[:-1, :])) / s.cell_size
    host = float(np.abs(div).max())
    assert r.max_divergence == host
    assert r.converged == bool(d["converged"])
    ref = float(d["max_divergence"])
    assert abs(r.max_divergence - ref) <= 0.1 * ref
    assert g.maxDivergence() == r.max_divergence
