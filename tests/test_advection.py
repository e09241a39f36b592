"""Semi-Lagrangian transport and the staggered velocity sampler.

The sampler is the reference's own (FluidSim/UniformCPU/FluidGridCPU.cpp:67-90, 465-471): the
restatement and the CUDA kernel must equal it bit for bit. The transport step has no reference
counterpart (the reference transports with PLIC); its restatement is pinned by known answers
(identity at rest, exact translation of affine fields) and the CUDA path must equal the
restatement bit for bit in FP64 and in FP32 storage.
"""
import numpy as np
import pytest

from conftest import golden


def affine_velocity(w, h, dx, origin, horizontal, vertical):
    """Face velocities sampled from two affine functions of world position
    (tests/FluidGridTests.cpp:53-93 builds its fields this way)."""
    u = np.zeros((h, w + 1))
    v = np.zeros((h + 1, w))
    for y in range(h):
        for x in range(w + 1):
            u[y, x] = horizontal(origin[0] + x * dx, origin[1] + (y + 0.5) * dx)
    for y in range(h + 1):
        for x in range(w):
            v[y, x] = vertical(origin[0] + (x + 0.5) * dx, origin[1] + y * dx)
    return u, v


def horizontal(x, y):
    return 0.3 * x + 0.7 * y - 2.0


def vertical(x, y):
    return -0.4 * x + 0.2 * y + 1.0


# ----------------------------------------------------------------------------------------------
# CPU: the restatement
# ----------------------------------------------------------------------------------------------


def test_sampler_reproduces_affine_field(oracle):
    """tests/FluidGridTests.cpp:53-93: bilinear sampling is exact for affine fields."""
    w, h, dx, origin = 9, 7, 2.5, (-7.0, 11.0)
    u, v = affine_velocity(w, h, dx, origin, horizontal, vertical)
    pos = np.array([[-2.3, 16.7], [8.1, 24.2]])
    out = oracle.sample_velocity(u, v, dx, pos, origin=origin)
    for (px, py), (vx, vy) in zip(pos, out):
        assert abs(vx - horizontal(px, py)) < 1e-12
        assert abs(vy - vertical(px, py)) < 1e-12


def test_sampler_matches_reference_golden(oracle):
    g = golden("sampler_9x7.npz")
    out = oracle.sample_velocity(g["u"], g["v"], float(g["cell_size"]), g["positions"], origin=tuple(g["origin"]))
    assert np.array_equal(out, g["velocities"])


def test_sampler_matches_live_reference(oracle):
    if not oracle.reference_available():
        pytest.skip("reference engine not built")
    rng = np.random.default_rng(7)
    w, h, dx, origin = 31, 17, 0.37, (1.5, -2.25)
    u = rng.standard_normal((h, w + 1))
    v = rng.standard_normal((h + 1, w))
    # Sign changes inside a cell exercise both branches of the blend.
    u[::3] *= -1.0
    g = oracle.ReferenceGrid(w, h, dx)
    g.set_origin(*origin)
    g.upload(np.zeros((h, w)), u, v)
    pos = np.column_stack([rng.uniform(0.0, 14.0, 4000), rng.uniform(-5.0, 6.0, 4000)])
    assert np.array_equal(g.sample_velocity(pos), oracle.sample_velocity(u, v, dx, pos, origin=origin))


def test_advect_at_rest_is_identity(oracle):
    rng = np.random.default_rng(3)
    w, h = 23, 11
    f = rng.uniform(0.0, 1.0, (h, w))
    m = rng.uniform(0.0, 5.0, (h, w))
    u_out, v_out, (f_out, m_out) = oracle.advect(np.zeros((h, w + 1)), np.zeros((h + 1, w)), [f, m], 0.1, 0.5)
    assert np.array_equal(f_out, f) and np.array_equal(m_out, m)
    assert not u_out.any() and not v_out.any()


def test_advect_translates_affine_fields(oracle):
    """A uniform velocity (U, V) moves an affine field a + b x + c y to a + b (x - sU) + c (y - sV)
    wherever the back-trace stays inside the sample domain; interior faces keep (U, V)."""
    w, h, dx, dt = 40, 30, 0.25, 0.05
    U, V = 1.7, -0.9
    s = dt / dx
    u = np.full((h, w + 1), U)
    v = np.full((h + 1, w), V)
    y, x = np.mgrid[0:h, 0:w] + 0.5
    field = 0.25 + 0.01 * x - 0.02 * y
    u_out, v_out, (f_out,) = oracle.advect(u, v, [field], dt, dx)
    expect = 0.25 + 0.01 * (x - s * U) - 0.02 * (y - s * V)
    inner = (slice(3, h - 3), slice(3, w - 3))
    assert np.abs(f_out[inner] - expect[inner]).max() < 1e-13
    assert np.array_equal(u_out[:, 1:w], np.full((h, w - 1), U))
    assert np.array_equal(v_out[1:h, :], np.full((h - 1, w), V))
    assert not u_out[:, [0, w]].any() and not v_out[[0, h], :].any()


def test_advect_keeps_fraction_bounded(oracle):
    rng = np.random.default_rng(11)
    w, h = 33, 21
    f = (rng.uniform(size=(h, w)) > 0.5).astype(float)
    u = 3.0 * rng.standard_normal((h, w + 1))
    v = 3.0 * rng.standard_normal((h + 1, w))
    _, _, (f_out,) = oracle.advect(u, v, [f], 0.2, 0.1)
    assert f_out.min() >= 0.0 and f_out.max() <= 1.0


# ----------------------------------------------------------------------------------------------
# GPU: the CUDA path through the C ABI
# ----------------------------------------------------------------------------------------------


def _grid(w, h, dx, precision):
    from fluidsim_b200 import FluidGrid

    return FluidGrid(w, h, dx, precision=precision)


def _upload(grid, f, u, v, liquid_mass=None, gas_mass=None):
    from fluidsim_b200.grid import FluidGridState

    grid.upload(FluidGridState(f, u, v, None, liquid_mass or [], gas_mass or []))


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_gpu_sampler_matches_reference_golden(precision):
    g = golden("sampler_9x7.npz")
    w, h, dx = int(g["width"]), int(g["height"]), float(g["cell_size"])
    grid = _grid(w, h, dx, precision)
    grid.configureMaterials([100.0], [0.1])
    grid.setOrigin(tuple(g["origin"]))
    u, v = g["u"], g["v"]
    if precision == "fp32":
        # FP32 storage rounds the velocities; the sampler itself is the same FP64 arithmetic.
        from oracle import oracle as O

        u32, v32 = (a.astype(np.float32).astype(np.float64) for a in (u, v))
        _upload(grid, np.zeros((h, w)), u32, v32)
        expect = O.sample_velocity(u32, v32, dx, g["positions"], origin=tuple(g["origin"]))
    else:
        _upload(grid, np.zeros((h, w)), u, v)
        expect = g["velocities"]
    assert np.array_equal(grid.sampleVelocity(g["positions"]), expect)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("shape", [(1, 1), (1, 40), (37, 1), (65, 37), (200, 130)])
def test_gpu_advect_matches_restatement(precision, shape, oracle):
    w, h = shape
    dx, dt = 1.0 / max(w, h), 0.01
    rng = np.random.default_rng(w * 1000 + h)
    grid = _grid(w, h, dx, precision)
    grid.configureMaterials([100.0], [0.1])
    f = rng.uniform(0.0, 1.0, (h, w))
    u = 2.0 * rng.standard_normal((h, w + 1))
    v = 2.0 * rng.standard_normal((h + 1, w))
    lm = 100.0 * f * dx * dx
    gm = 0.1 * (1.0 - f) * dx * dx
    _upload(grid, f, u, v, [lm], [gm])
    grid.advect(dt)
    s = grid.download()
    storage = np.float32 if precision == "fp32" else np.float64
    u_e, v_e, (f_e, lm_e, gm_e) = oracle.advect(u, v, [f, lm, gm], dt, dx, storage=storage)
    assert np.array_equal(s.u, u_e)
    assert np.array_equal(s.v, v_e)
    assert np.array_equal(s.liquid_fraction, f_e)
    assert np.array_equal(s.liquid_mass[0], lm_e)
    assert np.array_equal(s.gas_mass[0], gm_e)


@pytest.mark.gpu
def test_gpu_step_transports_then_projects(oracle):
    """step = advect + gravity + projection, in that order (FluidGridCPU.cpp:300-360)."""
    from fluidsim_b200 import scenes

    sc = scenes.dam_break(96, 64, velocity=0.5)
    a = _grid(sc.width, sc.height, sc.cell_size, "fp64")
    b = _grid(sc.width, sc.height, sc.cell_size, "fp64")
    for g in (a, b):
        scenes.upload_scene(g, sc)
    r = a.step(sc.dt, 400, 1e-6)
    b.advect(sc.dt)
    b.applyGravity(sc.dt)
    q = b.project(sc.dt, 400, 1e-6)
    assert r.iterations == q.iterations and r.converged == q.converged
    sa, sb = a.download(), b.download()
    for x, y in ((sa.u, sb.u), (sa.v, sb.v), (sa.pressure, sb.pressure), (sa.liquid_fraction, sb.liquid_fraction)):
        assert np.array_equal(x, y)


@pytest.mark.gpu
def test_gpu_steps_of_a_dam_break_are_all_accepted():
    """Sixty whole FP32 steps of a 256x256 dam break with obstacles, with the reference's step
    defaults (200 iterations, divergence 1e-6): every projection is accepted under the
    reference's result contract, and none runs to its iteration cap."""
    from fluidsim_b200 import scenes

    sc = scenes.dam_break(256, 256, seed=11, obstacles=8, velocity=0.0)
    g = _grid(sc.width, sc.height, sc.cell_size, "fp32")
    scenes.upload_scene(g, sc)
    for step in range(60):
        r = g.step(sc.dt, 200, 1e-6)
        assert r.solve_status == "converged" and r.accepted(), (step, r)
        assert r.iterations < 200
    s = g.download()
    assert np.isfinite(s.u).all() and np.isfinite(s.v).all()
