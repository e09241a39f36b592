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
