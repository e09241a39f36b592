"""State transfer and cache invalidation on the device, restating the reference's own tests
(tests/FluidGridTests.cpp:95-139 and :162-226) through this backend's public API. The reference
edits its CPU fields in place and calls invalidateCaches(); here every edit is an upload, which
must rebuild the density, face weights and multigrid hierarchy and restart the warm-start
history, so that a grid that has run for a while behaves exactly like a fresh one."""
import numpy as np
import pytest

from fluidsim_b200 import FluidGrid, FluidGridState, scenes

pytestmark = pytest.mark.gpu


def _grid(scene, precision, transport="semi_lagrangian", preconditioner="multigrid"):
    g = FluidGrid(scene.width, scene.height, scene.cell_size, precision)
    scenes.upload_scene(g, scene)
    g.setTransport(transport)
    g.setPreconditioner(preconditioner)
    return g


def _same(a, b):
    assert np.array_equal(a.u, b.u) and np.array_equal(a.v, b.v)
    assert np.array_equal(a.pressure, b.pressure) and np.array_equal(a.liquid_fraction, b.liquid_fraction)
    for x, y in zip(a.liquid_mass + a.gas_mass, b.liquid_mass + b.gas_mass):
        assert np.array_equal(x, y)


def _tilted_tank():
    """32 x 24 cells of size 4 with a tilted interface, the reference test's materials."""
    y, x = np.mgrid[0:24, 0:32]
    f = np.clip(y + 1.0 - (x + 12.0), 0.0, 1.0)
    zero_u, zero_v = np.zeros((24, 33)), np.zeros((25, 32))
    return scenes.Scene(32, 24, 4.0, 1.0 / 120.0, 100.0, 0.1, f, zero_u, zero_v, gravity=-9.8, name="tilted32x24")


@pytest.mark.parametrize("transport", ["semi_lagrangian", "plic"])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_state_transfer_reproduces_the_trajectory_and_resets_history(precision, transport):
    """:95-139. Two grids given the same state step identically; a download returns the state;
    re-uploading the initial state after 120 steps leaves no pressure history or cached
    coefficients behind, so the next step equals a fresh grid's bit for bit."""
    s = _tilted_tank()
    a, b = _grid(s, precision, transport), _grid(s, precision, transport)
    initial = a.download()
    for tick in range(120):
        ra, rb = a.step(s.dt, 2000, 1e-8), b.step(s.dt, 2000, 1e-8)
        assert ra.solve_status == "converged", (tick, ra)
        assert ra.iterations == rb.iterations, tick
        _same(a.download(), b.download())
    b.upload(initial)
    fresh = _grid(s, precision, transport)
    fresh.upload(initial)
    rb, rf = b.step(s.dt, 2000, 1e-8), fresh.step(s.dt, 2000, 1e-8)
    assert rb.iterations == rf.iterations
    _same(b.download(), fresh.download())


@pytest.mark.parametrize("preconditioner", ["multigrid", "diagonal"])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_new_densities_after_a_projection_match_a_fresh_grid(precision, preconditioner):
    """:162-226. After a projection has built the weights and the multigrid hierarchy, the
    densities change (a sloped interface, masses 400 f and 0.4 (1 - f) on cells of area 4) and
    a swirl is added to the velocities. The next projection must use the new coefficients:
    its result equals that of a fresh grid given the same state, within the reference's 2e-7."""
    w, h, dx = 33, 25, 2.0
    empty = np.zeros((h, w))
    s = scenes.Scene(w, h, dx, 0.01, 100.0, 0.1, empty, np.zeros((h, w + 1)), np.zeros((h + 1, w)),
                     gravity=-9.8, name="cache33x25")
    edited = _grid(s, precision, preconditioner=preconditioner)
    edited.applyGravity(0.01)
    assert edited.project(0.01, 2000, 1e-8).solve_status == "converged"

    state = edited.download()
    y, x = np.mgrid[0:h, 0:w]
    f = np.clip(y + 1.0 - (0.3 * x + 6.0), 0.0, 1.0)
    # A swirl around (30, 24) in world units (cells of size 2) with radius 12, strength 0.1.
    yu, xu = np.mgrid[0:h, 0:w + 1]
    yv, xv = np.mgrid[0:h + 1, 0:w]
    ru = np.hypot(xu * dx - 30.0, (yu + 0.5) * dx - 24.0)
    rv = np.hypot((xv + 0.5) * dx - 30.0, yv * dx - 24.0)
    u = state.u - 0.1 * ((yu + 0.5) * dx - 24.0) * np.clip(1.0 - ru / 12.0, 0.0, 1.0)
    v = state.v + 0.1 * ((xv + 0.5) * dx - 30.0) * np.clip(1.0 - rv / 12.0, 0.0, 1.0)
    u[:, [0, -1]] = 0.0
    v[[0, -1], :] = 0.0
    new = FluidGridState(f, u, v, state.pressure, [400.0 * f], [0.4 * (1.0 - f)])
    edited.upload(new)
    fresh = _grid(s, precision, preconditioner=preconditioner)
    fresh.upload(new)
    re, rf = edited.project(0.01, 2000, 1e-8), fresh.project(0.01, 2000, 1e-8)
    assert re.solve_status == rf.solve_status == "converged"
    a, b = edited.download(), fresh.download()
    assert np.abs(a.u - b.u).max() < 2e-7 and np.abs(a.v - b.v).max() < 2e-7
