"""Implicit viscosity: backward Euler m (v - v0) / dt = div(mu (grad v + grad v^T)) on the MAC faces.

The reference solves it only on the GPU (FluidSim/UniformWebGPU/ViscositySolverGPU.cpp, WGSL in
FP32), so the oracle is the FP64 restatement in oracle/fluid_oracle.c. It is pinned the way the
reference's own tests pin the GPU solver (tests/FluidViscosityTests.cpp): an independent FP64
residual assembled from cell and vertex strain energies (:84-138, restated below), analytic
decay of a Fourier mode (:177-220), zero viscosity and rigid rotation (:222-270), variable
viscosity (:272-300) and the iteration cap (:302-340). The CUDA path must pass the same checks
and agree with the restatement.
"""
import numpy as np
import pytest

# Acceptance bounds of tests/FluidViscosityTests.cpp.
DECAY_ERROR = 3e-4
RESIDUAL = 1.5e-4
VARIABLE_RESIDUAL = 1.8e-4
ROTATION_ERROR = 3e-5


class Case:
    """tests/FluidViscosityTests.cpp:21-81: a grid with per-cell density and viscosity."""

    def __init__(self, w, h, rho, mu, dx=1.0):
        self.w, self.h, self.dx = w, h, dx
        self.material = np.zeros((h, w, 2))
        self.material[..., 0] = rho
        self.material[..., 1] = mu
        self.u = np.zeros((h, w + 1))
        self.v = np.zeros((h + 1, w))

    def copy(self):
        c = Case(self.w, self.h, 0.0, 0.0, self.dx)
        c.material, c.u, c.v = self.material.copy(), self.u.copy(), self.v.copy()
        return c

    def um(self):
        rho = self.material[..., 0]
        return 0.5 * (rho[:, :-1] + rho[:, 1:]) * self.dx * self.dx   # interior u faces x = 1..w-1

    def vm(self):
        rho = self.material[..., 0]
        return 0.5 * (rho[:-1, :] + rho[1:, :]) * self.dx * self.dx   # interior v faces y = 1..h-1

    def energy(self):
        return 0.5 * ((self.um() * self.u[:, 1:-1] ** 2).sum() + (self.vm() * self.v[1:-1, :] ** 2).sum())

    def walls_closed(self):
        return (not self.u[:, [0, -1]].any() and not self.v[[0, -1], :].any()
                and np.isfinite(self.u).all() and np.isfinite(self.v).all())


def residual(old, new, dt):
    """tests/FluidViscosityTests.cpp:84-138: forces from independent cell (normal) and vertex
    (shear) strain energies, then the mass-weighted norm of m (v - v0) + dt K v relative to the
    initial kinetic energy."""
    mu = new.material[..., 1]
    ku = np.zeros_like(new.u)
    kv = np.zeros_like(new.v)
    tx = 2 * mu * (new.u[:, 1:] - new.u[:, :-1])
    ty = 2 * mu * (new.v[1:, :] - new.v[:-1, :])
    ku[:, :-1] -= tx
    ku[:, 1:] += tx
    kv[:-1, :] -= ty
    kv[1:, :] += ty
    if new.w > 1 and new.h > 1:
        mv = 0.25 * (mu[:-1, :-1] + mu[:-1, 1:] + mu[1:, :-1] + mu[1:, 1:])          # vertices 1..w-1, 1..h-1
        t = mv * (new.u[1:, 1:-1] - new.u[:-1, 1:-1] + new.v[1:-1, 1:] - new.v[1:-1, :-1])
        ku[1:, 1:-1] += t
        ku[:-1, 1:-1] -= t
        kv[1:-1, 1:] += t
        kv[1:-1, :-1] -= t
    ru = new.um() * (new.u[:, 1:-1] - old.u[:, 1:-1]) + dt * ku[:, 1:-1]
    rv = new.vm() * (new.v[1:-1, :] - old.v[1:-1, :]) + dt * kv[1:-1, :]
    error = (ru * ru / new.um()).sum() + (rv * rv / new.vm()).sum()
    return np.sqrt(error / max(2 * old.energy(), 1e-30))


def decay_case(w, h, mu, transverse):
    """tests/FluidViscosityTests.cpp:177-200: one Fourier mode on closed walls."""
    value = Case(w, h, 2.0, mu, dx=0.7)
    kx = np.pi / w
    ky = np.pi / h if h > 1 else 0.0
    sx = 2 * np.sin(0.5 * kx)
    sy = 2 * np.sin(0.5 * ky)
    x = np.arange(1, w)
    y = np.arange(h) + 0.5
    value.u[:, 1:w] = np.sin(kx * x)[None, :] * (np.cos(ky * y)[:, None] if transverse else 1.0)
    if transverse:
        xv = np.arange(w) + 0.5
        yv = np.arange(1, h)
        value.v[1:h, :] = -sx / sy * np.cos(kx * xv)[None, :] * np.sin(ky * yv)[:, None]
    value.u = value.u.astype(np.float32).astype(np.float64)
    value.v = value.v.astype(np.float32).astype(np.float64)
    return value, sx, sy


DECAYS = [(24, 16, 100.0, 0.02, False), (31, 23, 1000.0, 0.02, True), (65, 49, 100000.0, 0.1, True),
          (47, 1, 1000.0, 0.02, False), (2, 33, 1000.0, 0.02, False)]


def check_decay(old, new, sx, sy, mu, dt, transverse):
    factor = 1.0 / (1.0 + dt * mu * ((sx * sx + sy * sy) if transverse else 2 * sx * sx) / (2 * old.dx * old.dx))
    error = max(np.abs(new.u - factor * old.u).max(), np.abs(new.v - factor * old.v).max())
    assert error < DECAY_ERROR
    assert residual(old, new, dt) < RESIDUAL
    assert new.energy() <= old.energy() * (1 + 1e-6)
    assert new.walls_closed()


def oracle_step(oracle, value, dt, tolerance=1e-4, max_iterations=-1):
    solver = oracle.Viscosity(value.w, value.h)
    it, u, v, rel = solver.solve(value.u, value.v, value.material, dt, value.dx, tolerance, max_iterations)
    out = value.copy()
    if it >= 0:
        out.u, out.v = u, v
    return it, out


# ----------------------------------------------------------------------------------------------
# CPU: the restatement against the reference tests' own checks
# ----------------------------------------------------------------------------------------------


def test_operator_is_symmetric_positive(oracle):
    """The operator is the Hessian of mass and strain energies: x.Ay = y.Ax, x.Ax > 0."""
    rng = np.random.default_rng(0)
    w, h = 13, 9
    value = Case(w, h, 1.0, 0.0)
    value.material[..., 0] = rng.uniform(0.1, 10.0, (h, w))
    value.material[..., 1] = rng.uniform(0.0, 50.0, (h, w))
    solver = oracle.Viscosity(w, h)
    solver.setup(value.material, 0.02, 0.5)
    a, b = rng.standard_normal((2, h + 1, w + 1, 2))
    a[:, 0, 0] = a[:, w, 0] = a[h, :, 0] = 0.0
    a[0, :, 1] = a[h, :, 1] = a[:, w, 1] = 0.0
    b[:, 0, 0] = b[:, w, 0] = b[h, :, 0] = 0.0
    b[0, :, 1] = b[h, :, 1] = b[:, w, 1] = 0.0
    ab, ba = (a * solver.apply(b, 0.02)).sum(), (b * solver.apply(a, 0.02)).sum()
    assert abs(ab - ba) < 1e-12 * abs(ab)
    assert (a * solver.apply(a, 0.02)).sum() > 0.0


@pytest.mark.parametrize("w,h,mu,dt,transverse", DECAYS)
def test_decay_matches_analytic_backward_euler(oracle, w, h, mu, dt, transverse):
    value, sx, sy = decay_case(w, h, mu, transverse)
    it, new = oracle_step(oracle, value, dt)
    assert it > 0 and it % 4 == 0
    check_decay(value, new, sx, sy, mu, dt, transverse)


def test_zero_viscosity_and_rigid_rotation(oracle):
    """tests/FluidViscosityTests.cpp:222-270."""
    value = Case(25, 19, 2.0, 0.0)
    value.u[:, 1:25] = (0.3 * (np.arange(19) - 8))[:, None]
    value.v[1:19, :] = (-0.3 * (np.arange(25) - 10))[None, :]
    it, new = oracle_step(oracle, value, 0.01)
    assert it == 0 and np.array_equal(new.u, value.u) and np.array_equal(new.v, value.v)
    value.material[4:15, 4:21, 1] = 500.0
    it, new = oracle_step(oracle, value, 0.01)
    assert max(np.abs(new.u - value.u).max(), np.abs(new.v - value.v).max()) < ROTATION_ERROR
    rest = Case(25, 19, 2.0, 500.0)
    it, new = oracle_step(oracle, rest, 0.01)
    assert it == 0 and new.energy() == 0.0


@pytest.mark.parametrize("w,h", [(33, 25), (64, 48)])
def test_variable_viscosity(oracle, w, h):
    """tests/FluidViscosityTests.cpp:272-300 (10 of its 40 steps)."""
    value = Case(w, h, 1.0, 0.0)
    dense = np.arange(w)[None, :] < w // 2
    value.material[..., 0] = np.where(dense, 10.0, 0.1)
    value.material[..., 1] = np.where(dense, 10000.0, 0.0)
    x, y = np.meshgrid(np.arange(1, w), np.arange(h))
    value.u[:, 1:w] = np.sin(0.7 * x + 0.3 * y)
    x, y = np.meshgrid(np.arange(w), np.arange(1, h))
    value.v[1:h, :] = np.cos(0.2 * x + 0.8 * y)
    for _ in range(10):
        old = value
        it, value = oracle_step(oracle, old, 0.02)
        assert it > 0
        assert value.energy() <= old.energy() * (1 + 2e-6)
        assert residual(old, value, 0.02) < VARIABLE_RESIDUAL


def test_iteration_cap_and_nonfinite(oracle):
    """tests/FluidViscosityTests.cpp:302-340: a cap that is too small fails without committing,
    the default continues to full accuracy, non-finite input fails."""
    value = Case(33, 25, 1.0, 10000.0)
    x, y = np.meshgrid(np.arange(1, 33), np.arange(25))
    value.u[:, 1:33] = np.sin(0.7 * x + 0.3 * y)
    assert oracle_step(oracle, value, 0.0)[0] == 0
    it, new = oracle_step(oracle, value, 0.02, max_iterations=1)
    assert it == -2
    it, new = oracle_step(oracle, value, 0.02)
    assert it > 1 and residual(value, new, 0.02) < VARIABLE_RESIDUAL
    bad = value.copy()
    bad.u[5, 5] = np.nan
    assert oracle_step(oracle, bad, 0.02)[0] == -1


def test_material_blend(oracle):
    """Volume-weighted viscosity of two components (FluidGridGPU.cpp:172-217, 987-1037)."""
    dx = 0.5
    f = np.array([[0.0, 0.25, 1.0]])
    lm, gm = 1000.0 * f * dx * dx, 1.0 * (1 - f) * dx * dx
    m = oracle.viscosity_material([lm, gm], [1000.0, 1.0], [2.0, 0.01], dx)
    assert np.allclose(m[..., 0], 1000.0 * f + (1 - f))
    assert np.allclose(m[..., 1], 2.0 * f + 0.01 * (1 - f))


# ----------------------------------------------------------------------------------------------
# GPU: the CUDA path through the C ABI
# ----------------------------------------------------------------------------------------------


def _device_case(value, precision, liquid=None, gas=None):
    """A FluidGrid holding a Case: liquid cells are those with value.material's liquid pair."""
    from fluidsim_b200 import FluidGrid
    from fluidsim_b200.grid import FluidGridState

    rho, mu = value.material[..., 0], value.material[..., 1]
    liquid = liquid or (float(rho.max()), float(mu.max()))
    gas = gas or (float(rho.min()), float(mu.min()))
    is_liquid = (rho == liquid[0]) & (mu == liquid[1])
    area = value.dx * value.dx
    f = is_liquid.astype(float)
    lm, gm = liquid[0] * f * area, gas[0] * (1.0 - f) * area
    g = FluidGrid(value.w, value.h, value.dx, precision=precision)
    g.configureMaterials([liquid[0]], [gas[0]], [liquid[1]], [gas[1]])
    g.upload(FluidGridState(f, value.u, value.v, None, [lm], [gm]))
    return g, lm, gm, liquid, gas


def device_step(value, dt, precision, tolerance=1e-4, max_iterations=-1, **kw):
    g, *_ = _device_case(value, precision, **kw)
    it, rel = g.applyViscosity(dt, tolerance, max_iterations)
    s = g.download()
    out = value.copy()
    out.u, out.v = s.u, s.v
    return it, out


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp32", "fp64"])
@pytest.mark.parametrize("w,h,mu,dt,transverse", DECAYS)
def test_gpu_decay_matches_analytic_backward_euler(precision, w, h, mu, dt, transverse):
    value, sx, sy = decay_case(w, h, mu, transverse)
    it, new = device_step(value, dt, precision, gas=(2.0, 0.0))
    assert it > 0 and it % 4 == 0
    check_decay(value, new, sx, sy, mu, dt, transverse)


@pytest.mark.gpu
@pytest.mark.parametrize("w,h,mu,dt,transverse", DECAYS)
def test_gpu_fp64_matches_restatement(oracle, w, h, mu, dt, transverse):
    """FP64 on the device against the FP64 restatement: the same iteration count and velocities
    equal to rounding (the two sum their reductions in different orders)."""
    value, _, _ = decay_case(w, h, mu, transverse)
    g, lm, gm, liquid, gas = _device_case(value, "fp64", gas=(2.0, 0.0))
    material = oracle.viscosity_material([lm, gm], [liquid[0], gas[0]], [liquid[1], gas[1]], value.dx)
    it_o, u_o, v_o, _ = oracle.Viscosity(w, h).solve(value.u, value.v, material, dt, value.dx, 1e-4)
    it, _ = g.applyViscosity(dt, 1e-4)
    s = g.download()
    assert it == it_o
    scale = max(np.abs(u_o).max(), np.abs(v_o).max())
    assert np.abs(s.u - u_o).max() <= 1e-10 * scale and np.abs(s.v - v_o).max() <= 1e-10 * scale


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_gpu_rigid_rotation_and_rest(precision):
    value = Case(25, 19, 2.0, 0.0)
    # FP32 values, as the reference test stores them, so FP32 storage holds them exactly.
    value.u[:, 1:25] = np.float32(0.3) * (np.arange(19, dtype=np.float32) - 8)[:, None]
    value.v[1:19, :] = np.float32(-0.3) * (np.arange(25, dtype=np.float32) - 10)[None, :]
    it, new = device_step(value, 0.01, precision, liquid=(2.0, 500.0), gas=(2.0, 0.0))
    assert it == 0 and np.array_equal(new.u, value.u) and np.array_equal(new.v, value.v)
    # A rigid rotation has no strain: a viscous region leaves it (nearly) unchanged.
    value.material[4:15, 4:21, 1] = 500.0
    it, new = device_step(value, 0.01, precision, liquid=(2.0, 500.0), gas=(2.0, 0.0))
    assert max(np.abs(new.u - value.u).max(), np.abs(new.v - value.v).max()) < ROTATION_ERROR
    rest = Case(25, 19, 2.0, 500.0)
    it, new = device_step(rest, 0.01, precision, gas=(2.0, 0.0))
    assert it == 0 and new.energy() == 0.0


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp32", "fp64"])
@pytest.mark.parametrize("w,h", [(33, 25), (64, 48)])
def test_gpu_variable_viscosity(precision, w, h):
    from fluidsim_b200.grid import FluidGridState

    value = Case(w, h, 1.0, 0.0)
    dense = np.arange(w)[None, :] < w // 2
    value.material[..., 0] = np.where(dense, 10.0, 0.1)
    value.material[..., 1] = np.where(dense, 10000.0, 0.0)
    x, y = np.meshgrid(np.arange(1, w), np.arange(h))
    value.u[:, 1:w] = np.sin(0.7 * x + 0.3 * y)
    x, y = np.meshgrid(np.arange(w), np.arange(1, h))
    value.v[1:h, :] = np.cos(0.2 * x + 0.8 * y)
    g, *_ = _device_case(value, precision)
    # 40 steps on the device-resident state (tests/FluidViscosityTests.cpp:272-300).
    for step in range(40):
        old = value
        it, _ = g.applyViscosity(0.02)
        s = g.download()
        value = old.copy()
        value.u, value.v = s.u, s.v
        # Later steps may start below the target once the viscous region has decayed.
        assert it > 0 or step > 0
        assert value.energy() <= old.energy() * (1 + 2e-6)
        assert residual(old, value, 0.02) < VARIABLE_RESIDUAL
        assert value.walls_closed()


@pytest.mark.gpu
def test_gpu_iteration_cap_and_nonfinite():
    from fluidsim_b200 import FluidCudaError
    from fluidsim_b200.grid import FluidGridState

    value = Case(33, 25, 1.0, 10000.0)
    x, y = np.meshgrid(np.arange(1, 33), np.arange(25))
    value.u[:, 1:33] = np.sin(0.7 * x + 0.3 * y)
    g, lm, gm, *_ = _device_case(value, "fp32", gas=(1.0, 0.0))
    assert g.applyViscosity(0.0) == (0, 0.0)
    before = g.download()
    with pytest.raises(FluidCudaError):
        g.applyViscosity(0.02, 1e-4, 1)
    after = g.download()
    assert np.array_equal(before.u, after.u) and np.array_equal(before.v, after.v)
    it, _ = g.applyViscosity(0.02)
    new = value.copy()
    new.u, new.v = g.download().u, g.download().v
    assert it > 1 and residual(value, new, 0.02) < VARIABLE_RESIDUAL
    bad = value.u.copy()
    bad[5, 5] = np.nan
    g.upload(FluidGridState(np.ones((25, 33)), bad, value.v, None, [lm], [gm]))
    with pytest.raises(FluidCudaError):
        g.applyViscosity(0.02)
    assert np.array_equal(g.download().v, value.v)


@pytest.mark.gpu
def test_gpu_step_counts_viscosity_iterations():
    from fluidsim_b200 import FluidGrid, scenes

    sc = scenes.dam_break(64, 48, obstacles=2, velocity=0.5)
    # FP64: the max-norm rule at 1e-6 asks for more than FP32 velocities can resolve here.
    g = FluidGrid(sc.width, sc.height, sc.cell_size, "fp64")
    scenes.upload_scene(g, sc)
    r0 = g.step(sc.dt, 200, 1e-6)
    assert r0.viscosity_iterations == 0
    g.setComponentViscosity("liquid", 0, 1.0)
    r = g.step(sc.dt, 200, 1e-6)
    assert r.viscosity_iterations > 0 and r.converged
    s = g.download()
    # Faces of obstacle cells stay closed after the viscous solve and the projection.
    solid = sc.solid.astype(bool)
    assert not s.u[:, 1:-1][solid[:, :-1] | solid[:, 1:]].any()
    assert not s.v[1:-1, :][solid[:-1, :] | solid[1:, :]].any()
