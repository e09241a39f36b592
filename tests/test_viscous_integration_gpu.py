"""Implicit viscosity inside whole grids, restating the reference's integration tests
(tests/FluidViscosityIntegrationTests.cpp:25-83 set-up, :85-162 blending, :164-207 checkpoint
continuation) through this backend's public API. The reference runs them on its WebGPU engine;
the solver it compares against is restated in the oracle."""
import json

import numpy as np
import pytest

from fluidsim_b200 import FluidGrid, FluidGridState, FluidInvalidArgument

pytestmark = pytest.mark.gpu


def _f32(a):
    return np.asarray(a, dtype=np.float32).astype(np.float64)


def _initialize(g, liquids, gases):
    """:25-83: liquid k has density 10 + k and viscosity 20 + 100 k, gas k density 0.1 + 0.01 k
    and no viscosity; fraction (y + 1) / (h + 1) shared equally by each phase's components; a
    closed sine stream function for the velocities; FP32 values as the reference's state holds."""
    w, h, dx = g.getWidth(), g.getHeight(), g.getCellSize()
    ld = [10.0 + k for k in range(liquids)]
    lmu = [20.0 + 100.0 * k for k in range(liquids)]
    gd = [0.1 + 0.01 * k for k in range(gases)]
    g.configureMaterials(ld, gd, lmu, [0.0] * gases)
    g.setGravityY(0.0)
    area = np.float32(dx * dx)
    y = np.arange(h, dtype=np.float32)[:, None] * np.ones((1, w), dtype=np.float32)
    f = (y + np.float32(1)) / np.float32(h + 1)
    lm = [_f32(area * f * np.float32(d) / np.float32(liquids)) for d in ld]
    gm = [_f32(area * (np.float32(1) - f) * np.float32(d) / np.float32(gases)) for d in gd]

    def psi(x, yy):
        inner = (x > 0) & (x < w) & (yy > 0) & (yy < h)
        return np.where(inner, 2.0 * np.sin(np.pi * x / w) * np.sin(np.pi * yy / h), 0.0)

    yu, xu = np.mgrid[0:h, 0:w + 1].astype(float)
    yv, xv = np.mgrid[0:h + 1, 0:w].astype(float)
    u = _f32(psi(xu, yu + 1) - psi(xu, yu))
    v = _f32(psi(xv, yv) - psi(xv + 1, yv))
    g.upload(FluidGridState(_f32(f), u, v, None, lm, gm))
    return ld + gd, lmu + [0.0] * gases


def _same(a, b):
    return (np.array_equal(a.u, b.u) and np.array_equal(a.v, b.v) and np.array_equal(a.pressure, b.pressure)
            and np.array_equal(a.liquid_fraction, b.liquid_fraction)
            and all(np.array_equal(x, y) for x, y in zip(a.liquid_mass + a.gas_mass, b.liquid_mass + b.gas_mass)))


@pytest.mark.parametrize("liquids,gases", [(2, 2), (17, 3)])
def test_blended_viscosity_matches_independent_coefficients(oracle, liquids, gases):
    """:85-162. With the last gas component made viscous, the grid's solve equals the solver run
    on independently computed cell densities and volume-weighted viscosities: FP64 equals the
    oracle's solver (the same iterations, 1e-10 of scale); FP32, solved in its own arithmetic,
    stays within 1e-4 of scale of it. Composition and geometry are
    untouched; a zero step and all-zero viscosities do nothing; gas viscosity alone activates
    the solver."""
    for precision in ("fp64", "fp32"):
        g = FluidGrid(24, 18, 0.7, precision)
        densities, viscosities = _initialize(g, liquids, gases)
        g.setComponentViscosity("gas", gases - 1, 5.0)
        viscosities[-1] = 5.0
        initial = g.download()

        masses = initial.liquid_mass + initial.gas_mass
        volume = sum(m / d for m, d in zip(masses, densities))
        material = np.stack([sum(masses) / (0.7 * 0.7),
                             sum(m / d * mu for m, d, mu in zip(masses, densities, viscosities)) / volume], axis=-1)
        it_o, u_o, v_o, _ = oracle.Viscosity(24, 18).solve(initial.u, initial.v, material, 0.01, 0.7, 1e-4)

        it, _ = g.applyViscosity(0.01)
        assert it > 0
        result = g.download()
        scale = max(np.abs(u_o).max(), np.abs(v_o).max())
        bound = (1e-10 if precision == "fp64" else 1e-4) * scale
        assert np.abs(result.u - u_o).max() < bound and np.abs(result.v - v_o).max() < bound
        if precision == "fp64":
            assert it == it_o
        assert np.array_equal(result.liquid_fraction, initial.liquid_fraction)
        assert all(np.array_equal(a, b) for a, b in zip(result.liquid_mass + result.gas_mass, masses))

        assert g.applyViscosity(0.0)[0] == 0 and _same(result, g.download())
        for k in range(liquids):
            g.setComponentViscosity("liquid", k, 0.0)
        for k in range(gases):
            g.setComponentViscosity("gas", k, 0.0)
        assert g.applyViscosity(0.01)[0] == 0 and _same(result, g.download())
        g.setComponentViscosity("gas", gases - 1, 5.0)
        assert g.applyViscosity(0.01)[0] > 0
        gas_only = g.download()
        assert np.array_equal(gas_only.liquid_fraction, result.liquid_fraction)
        assert all(np.array_equal(a, b) for a, b in zip(gas_only.liquid_mass + gas_only.gas_mass, masses))


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_viscous_checkpoint_continues_and_rejects_invalid_viscosity(precision):
    """:164-207 (without the WebGPU engine's pressure recovery). Twelve viscous steps, a save,
    a load into a fresh grid, then twelve more steps on both: every step accepted, the same
    viscosity iterations, identical states; a saved negative viscosity is rejected and leaves
    the live state as it was."""
    g = FluidGrid(24, 18, 1.0, precision)
    _initialize(g, 2, 2)
    for _ in range(12):
        assert g.step(0.004, 2000, 0.001).accepted()
    meta, payload = g.saveCheckpoint()
    assert meta["liquid_mixture"][1]["dynamic_viscosity"] == 120.0

    restored = FluidGrid(24, 18, 1.0, precision)
    restored.loadCheckpoint(meta, payload)
    for _ in range(12):
        a, b = g.step(0.004, 2000, 0.001), restored.step(0.004, 2000, 0.001)
        assert a.accepted() and b.accepted()
        assert a.viscosity_iterations == b.viscosity_iterations
    assert _same(g.download(), restored.download())

    before = restored.download()
    bad = json.loads(json.dumps(meta))
    bad["liquid_mixture"][0]["dynamic_viscosity"] = -1.0
    with pytest.raises(FluidInvalidArgument):
        restored.loadCheckpoint(bad, payload)
    assert _same(before, restored.download())
