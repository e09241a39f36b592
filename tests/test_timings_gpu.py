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
