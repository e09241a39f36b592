"""Degenerate steps and miscible components on the device, restating the reference's own tests
(tests/FluidGridTests.cpp:421-442 and :444-537) through this backend's public API."""
import numpy as np
import pytest

from fluidsim_b200 import FluidGrid, FluidGridState

pytestmark = pytest.mark.gpu


def _fields(s):
    return [s.u, s.v, s.liquid_fraction] + list(s.liquid_mass) + list(s.gas_mass)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_zero_time_and_failed_projection_are_handled(precision):
    """:421-442. A zero time step reports no convergence and leaves every field untouched; a
    projection allowed no iterations, with gravity having disturbed the state, does not claim
    convergence."""
    g = FluidGrid(8, 8, 1.0, precision)
    g.configureMaterials([100.0], [0.1])
    g.setGravityY(1.0)
    f = np.zeros((8, 8))
    f[3, 3] = 1.0
    g.upload(FluidGridState(f, np.zeros((8, 9)), np.zeros((9, 8)), None, [100.0 * f], [0.1 * (1.0 - f)]))
    before = g.download()
    assert not g.step(0.0).converged
    after = g.download()
    for a, b in zip(_fields(before), _fields(after)):
        assert np.array_equal(a, b)
    assert not g.step(0.01, 0, 1e-8).converged


def test_miscible_components_conserve_mass_and_volume():
    """:444-537. A 32 x 32 tank of cells of size 2 with a cosine surface; four liquid components
    (densities 100, 100, 200 and an unused 1000) and two gas components (0.1, 0.2) whose shares
    partition each phase's volume. 2400 steps of 1/120 (20 s of sloshing) with the reference's
    conservative transport and gravity 100: every projection converges to divergence 1e-8, each
    component's mass drifts by less than 1e-8 of itself, masses stay non-negative, the components'
    volumes add up to their phase's volume within 1e-9, and the unused component stays empty."""
    w = h = 32
    dx = 2.0
    area = dx * dx
    liquid_density = [100.0, 100.0, 200.0, 1000.0]
    gas_density = [0.1, 0.2]
    y, x = np.mgrid[0:h, 0:w].astype(float)
    surface = h * (0.5 + 0.04 * np.cos(np.pi * (x + 0.5) / w))
    f = np.clip(y + 1.0 - surface, 0.0, 1.0)
    heavy = np.where(x >= w // 2, 0.25, 0.0)
    water = (1.0 - heavy) * (y + 0.5) / h
    air = (x + 0.5) / w
    liquid = [100.0 * area * f * water, 100.0 * area * f * (1.0 - water - heavy), 200.0 * area * f * heavy,
              np.zeros((h, w))]
    gas = [0.1 * area * (1.0 - f) * air, 0.2 * area * (1.0 - f) * (1.0 - air)]

    g = FluidGrid(w, h, dx, "fp64")
    g.configureMaterials(liquid_density, gas_density)
    g.setGravityY(100.0)
    g.setTransport("plic")
    g.upload(FluidGridState(f, np.zeros((h, w + 1)), np.zeros((h + 1, w)), None, liquid, gas))
    start = g.download()
    initial_volume = start.liquid_fraction.sum()
    initial_mass = [m.sum() for m in start.liquid_mass + start.gas_mass]
    densities = liquid_density + gas_density

    for tick in range(2400):
        r = g.step(1.0 / 120.0, 2000, 1e-8)
        assert r.converged and r.max_divergence <= 1e-8, (tick, r)
        s = g.download()
        assert np.isfinite(s.u).all() and np.isfinite(s.v).all()
        assert (s.liquid_fraction >= -1e-6).all() and (s.liquid_fraction <= 1.0 + 1e-6).all()
        assert abs(s.liquid_fraction.sum() - initial_volume) <= initial_volume * 1e-10
        assert not s.u[:, [0, -1]].any() and not s.v[[0, -1], :].any()
        masses = s.liquid_mass + s.gas_mass
        for m, m0, rho in zip(masses, initial_mass, densities):
            assert abs(m.sum() - m0) / max(1.0, m0) < 1e-8, tick
            assert np.isfinite(m).all() and (m >= -1e-10 * rho * area).all()
        occupied_liquid = sum(m / (rho * area) for m, rho in zip(s.liquid_mass, liquid_density))
        occupied_gas = sum(m / (rho * area) for m, rho in zip(s.gas_mass, gas_density))
        assert np.abs(occupied_liquid - s.liquid_fraction).max() < 1e-9
        assert np.abs(occupied_gas - (1.0 - s.liquid_fraction)).max() < 1e-9
        assert not s.liquid_mass[3].any()
