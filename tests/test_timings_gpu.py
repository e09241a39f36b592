"""Per-stage step timings, restating the part of the reference's API test that applies to one
backend (tests/FluidGridAPITests.cpp:83-133): asking for timings changes neither the results nor
the state, the stages that ran report time, and a zero-time step clears every stage, even in a
caller's struct that still holds an earlier step's values."""
import ctypes as C

import numpy as np
import pytest

from fluidsim_b200 import FluidGrid, scenes
from fluidsim_b200 import _native as N

pytestmark = pytest.mark.gpu


def _grid(scene, precision):
    g = FluidGrid(scene.width, scene.height, scene.cell_size, precision)
    scenes.upload_scene(g, scene)
    return g


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_timed_steps_match_untimed_steps(precision):
    s = scenes.dam_break(32, 32, seed=3, obstacles=2, velocity=0.5)
    plain, measured = _grid(s, precision), _grid(s, precision)
    for tick in range(8):
        timings = {}
        a = plain.step(0.01, 2000, 1e-3)
        b = measured.step(0.01, 2000, 1e-3, timings)
        assert a.accepted() and b.accepted(), tick
        assert (a.iterations, a.solve_status, a.converged, a.restarts) == (b.iterations, b.solve_status, b.converged,
                                                                          b.restarts)
        sa, sb = plain.download(), measured.download()
        for x, y in ((sa.u, sb.u), (sa.v, sb.v), (sa.pressure, sb.pressure), (sa.liquid_fraction, sb.liquid_fraction)):
            assert np.array_equal(x, y)
        assert timings["transport_ms"] > 0.0 and timings["forces_ms"] > 0.0 and timings["pressure_ms"] > 0.0
        assert timings["selection_ms"] == 0.0 and timings["regrid_ms"] == 0.0


def test_zero_time_step_clears_a_callers_timings():
    s = scenes.dam_break(32, 32, seed=3, obstacles=0, velocity=0.5)
    g = _grid(s, "fp32")
    r, t = N.FcResult(), N.FcTimings()
    N.check(N.lib().fc_step(g.handle, 0.01, 2000, 1e-3, C.byref(r), C.byref(t)))
    assert t.transport_ms > 0.0 and t.pressure_ms > 0.0
    before = g.download()
    N.check(N.lib().fc_step(g.handle, 0.0, 2000, 1e-3, C.byref(r), C.byref(t)))
    assert all(getattr(t, name) == 0.0 for name, _ in N.FcTimings._fields_)
    assert not r.converged and r.physical_steps == 0
    after = g.download()
    assert np.array_equal(before.u, after.u) and np.array_equal(before.liquid_fraction, after.liquid_fraction)


@pytest.mark.parametrize("case", ["gas", "dirichlet", "tension", "viscous", "plic"])
def test_enqueued_substeps_match_waiting_stages(case):
    """Untimed steps enqueue each substep's stages without waiting between them
    (fc_advance_substep); timed steps wait for every stage. Both give the same state bit for bit,
    with Dirichlet air, surface tension (capillary substeps), viscosity and PLIC transport, and
    fc_advance_substep followed by fc_project is the same step again."""
    import dataclasses

    s = scenes.dam_break(48, 40, seed=7, obstacles=2, velocity=0.5, cell_size=1.0 / 128.0,
                         surface_tension=0.07 if case == "tension" else 0.0)
    if case == "dirichlet":
        s = dataclasses.replace(s, air_model="dirichlet")
    if case == "viscous":
        s = dataclasses.replace(s, liquid_viscosity=[0.5], gas_viscosity=[1e-3])
    grids = [_grid(s, "fp32") for _ in range(3)]
    if case == "plic":
        for g in grids:
            g.setTransport("plic")
    untimed, timed, manual = grids
    for tick in range(6):
        a = untimed.step(s.dt, 200, 1e-6)
        b = timed.step(s.dt, 200, 1e-6, {})
        assert (a.iterations, a.viscosity_iterations, a.physical_steps) == (b.iterations, b.viscosity_iterations,
                                                                           b.physical_steps), tick
        if a.physical_steps == 1:
            visc = manual.advanceSubstep(s.dt)
            c = manual.project(s.dt, 200, 1e-6)
            assert (c.iterations, visc) == (a.iterations, a.viscosity_iterations), tick
        else:
            manual.step(s.dt, 200, 1e-6)
        sa, sb, sc = untimed.download(), timed.download(), manual.download()
        for name in ("u", "v", "pressure", "liquid_fraction"):
            assert np.array_equal(getattr(sa, name), getattr(sb, name)), (tick, name)
            assert np.array_equal(getattr(sa, name), getattr(sc, name)), (tick, name)


def test_stream_priority_changes_no_result():
    """A grid moved to the highest stream priority after some steps continues exactly like one
    left at the default; priorities outside the device's range are rejected."""
    from fluidsim_b200 import FluidInvalidArgument

    s = scenes.dam_break(40, 36, seed=9, obstacles=2, velocity=0.5)
    a, b = _grid(s, "fp32"), _grid(s, "fp32")
    for tick in range(6):
        if tick == 2:
            b.setStreamPriority(-1)  # the default is 0, the least priority CUDA offers
        ra, rb = a.step(0.01, 200, 1e-6), b.step(0.01, 200, 1e-6)
        assert ra.iterations == rb.iterations
        sa, sb = a.download(), b.download()
        assert np.array_equal(sa.u, sb.u) and np.array_equal(sa.pressure, sb.pressure)
    with pytest.raises(FluidInvalidArgument):
        b.setStreamPriority(1)
    with pytest.raises(FluidInvalidArgument):
        b.setStreamPriority(-1000)
