"""Properties of the conservative (PLIC) transport on the device, restating the reference's own
transport tests (tests/FluidGridTests.cpp:227-420) through this backend's public API: FP64
grids with the reference's transport selected, materials as the reference tests set them."""
import numpy as np
import pytest

from fluidsim_b200 import FluidGrid, FluidGridState

pytestmark = pytest.mark.gpu


def _grid(w, h, dx, f, u, v, liquid=100.0, gas=0.1, gravity=0.0):
    g = FluidGrid(w, h, dx, "fp64")
    g.configureMaterials([liquid], [gas])
    g.setGravityY(gravity)
    g.setTransport("plic")
    area = dx * dx
    g.upload(FluidGridState(f, u, v, None, [liquid * area * f], [gas * area * (1.0 - f)]))
    return g


def test_transport_conserves_liquid_and_moves_its_centroid():
    """:227-262. A 8 x 12 block carried by u = 1 for 8 time units (through the transport's own
    CFL substeps) keeps its volume and moves its centroid by exactly 8 cells along x."""
    w, h = 64, 32
    f = np.zeros((h, w))
    f[6:18, 8:16] = 1.0
    g = _grid(w, h, 1.0, f, np.ones((h, w + 1)), np.zeros((h + 1, w)))
    g.advect(8.0)
    out = g.download().liquid_fraction
    assert (out >= -1e-14).all() and (out <= 1.0 + 1e-14).all()
    y, x = np.mgrid[0:h, 0:w]
    mass = out.sum()
    assert abs(mass - 96.0) < 1e-10
    assert abs(((x + 0.5) * out).sum() / mass - 20.0) < 1e-10
    assert abs(((y + 0.5) * out).sum() / mass - 12.0) < 1e-10


def test_transport_keeps_straight_interfaces_sharp():
    """:264-289. Uniform motion by eight whole cells moves a full-height slab without blurring
    either interface."""
    w, h = 40, 8
    f = np.zeros((h, w))
    f[:, 8:16] = 1.0
    g = _grid(w, h, 1.0, f, np.ones((h, w + 1)), np.zeros((h + 1, w)))
    g.advect(8.0)
    expected = np.zeros((h, w))
    expected[:, 16:24] = 1.0
    assert np.abs(g.download().liquid_fraction - expected).max() < 1e-12


def _shallow(along, depth, slope, reverse):
    """The exact cell fraction under the line depth = 48.25 + slope (along - 48) (:300-313)."""
    def integral(t):
        return np.where(t <= 0.0, 0.0, np.where(t >= 1.0, t - 0.5, 0.5 * t * t))

    a = depth + 1.0 - (48.25 + slope * (along - 48.0))
    b = a - slope
    fraction = np.clip(a, 0.0, 1.0) if slope == 0.0 else (integral(a) - integral(b)) / slope
    return 1.0 - fraction if reverse else fraction


def test_transport_keeps_shallow_interfaces_straight():
    """:291-355. Straight interfaces of slope 0, +-0.05, +-0.1, either phase below, carried
    either way along x or y by 20 steps of 0.25: in the interior the fraction stays the exact
    integral under the translated line within 1e-6."""
    n = 96
    y, x = np.mgrid[0:n, 0:n].astype(float)
    largest = 0.0
    for vertical in (False, True):
        for reverse in (False, True):
            for slope in (0.0, -0.1, -0.05, 0.05, 0.1):
                for speed in (-1.0, 1.0):
                    along, depth = (y, x) if vertical else (x, y)
                    f = _shallow(along, depth, slope, reverse)
                    u = np.zeros((n, n + 1)) if vertical else np.full((n, n + 1), speed)
                    v = np.full((n + 1, n), speed) if vertical else np.zeros((n + 1, n))
                    g = _grid(n, n, 1.0, f, u, v)
                    for _ in range(20):
                        g.advect(0.25)
                    out = g.download().liquid_fraction
                    expected = _shallow(along - 5.0 * speed, depth, slope, reverse)
                    largest = max(largest, np.abs(out - expected)[24:72, 24:72].max())
                    g.destroy()
    assert largest < 1e-6


def test_closed_pool_remains_valid_over_repeated_motion():
    """:357-382. A 32 x 32 pool (cells of size 4, densities 1000 and 1, gravity 100) with a
    cosine surface sloshes for 2400 steps of 1/120: every projection converges to divergence
    1e-8, fractions stay in [0, 1], liquid volume is kept to 1e-10 and no flow crosses a wall."""
    n = 32
    y, x = np.mgrid[0:n, 0:n].astype(float)
    surface = n * (0.5 + 0.04 * np.cos(np.pi * (x + 0.5) / n))
    f = np.clip(y + 1.0 - surface, 0.0, 1.0)
    g = _grid(n, n, 4.0, f, np.zeros((n, n + 1)), np.zeros((n + 1, n)), 1000.0, 1.0, gravity=100.0)
    volume = f.sum()
    for tick in range(2400):
        r = g.step(1.0 / 120.0, 2000, 1e-8)
        assert r.converged and r.max_divergence <= 1e-8, (tick, r)
        s = g.download()
        assert np.isfinite(s.u).all() and np.isfinite(s.v).all()
        assert (s.liquid_fraction >= -1e-6).all() and (s.liquid_fraction <= 1.0 + 1e-6).all()
        assert abs(s.liquid_fraction.sum() - volume) <= volume * 1e-10
        assert not s.u[:, [0, -1]].any() and not s.v[[0, -1], :].any()


@pytest.mark.parametrize("velocity", [(1.0, 0.75), (-1.0, 0.75), (1.0, -0.75), (-1.0, -0.75)])
def test_transport_preserves_uniform_motion_across_density_changes(velocity):
    """:384-419. A round 1000:1 drop in uniform diagonal motion, transported for one time unit:
    the liquid volume is kept to 1e-10 and, away from the walls, momentum transport across the
    density jump leaves the velocity exactly uniform (1e-10)."""
    n = 48
    y, x = np.mgrid[0:n, 0:n].astype(float)
    f = np.zeros((n, n))
    inner = (slice(18, 30), slice(18, 30))
    f[inner] = np.clip(6.0 - np.hypot(x[inner] - 23.5, y[inner] - 23.5), 0.0, 1.0)
    vx, vy = velocity
    g = _grid(n, n, 1.0, f, np.full((n, n + 1), vx), np.full((n + 1, n), vy), 1000.0, 1.0)
    g.advect(1.0)
    s = g.download()
    assert abs(s.liquid_fraction.sum() - f.sum()) < 1e-10
    assert np.abs(s.u[8:n - 8, 8:n - 8] - vx).max() < 1e-10
    assert np.abs(s.v[8:n - 8, 8:n - 8] - vy).max() < 1e-10
