"""Conservative PLIC transport: the reference's own FluidGridCPU::advect
(FluidSim/UniformCPU/FluidGridCPU.cpp:362-463) against the CUDA path with the PLIC scheme.

The device evaluates every operation in the reference's order without fused multiply-adds, and
the reference here is built without contraction, so FP64 results must agree bit for bit. In FP32
storage the transport still runs in FP64 on the FP32-rounded velocities, so fraction and masses
match the reference run on the same rounded velocities exactly, and the velocities match its
result rounded to FP32.
"""
import numpy as np
import pytest

from fluidsim_b200 import scenes


def _reference(oracle):
    if not oracle.reference_available():
        pytest.skip("reference engine not built")


def _blobs(w, h, seed):
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:h, 0:w].astype(float)
    f = np.zeros((h, w))
    for _ in range(6):
        cx, cy, r = rng.uniform(0, w), rng.uniform(0, h), rng.uniform(2.0, 9.0)
        d = np.sqrt((x + 0.5 - cx) ** 2 + (y + 0.5 - cy) ** 2)
        f = np.maximum(f, np.clip(r - d + 0.5, 0.0, 1.0))
    u = rng.uniform(-1.0, 1.0, (h, w + 1))
    v = rng.uniform(-1.0, 1.0, (h + 1, w))
    u[:, [0, w]] = 0.0
    v[[0, h], :] = 0.0
    return scenes.Scene(w, h, 1.0 / max(w, h), 1.0 / 60.0, 1000.0, 1.0, f, u, v, name=f"blobs{w}x{h}")


CASES = {
    "sloped40x30": lambda: scenes.sloped_pool(40, 30),
    "dam64x48": lambda: scenes.dam_break(64, 48, seed=4, obstacles=0, velocity=1.0),
    "blobs57x41": lambda: _blobs(57, 41, seed=9),
}


def _reference_advect(oracle, s, u, v, dt):
    g = oracle.ReferenceGrid(s.width, s.height, s.cell_size, s.liquid_density, s.gas_density)
    g.upload(s.fraction, u, v, None, s.liquid_mass[0], s.gas_mass[0])
    g.advect(dt)
    f, uo, vo, _ = g.download()
    lm, gm = g.masses()
    return f, uo, vo, lm, gm


def test_reference_transport_conserves_mass_in_solenoidal_flow(oracle):
    """With a discretely divergence-free velocity (from a node stream function that vanishes on
    the walls) the corrections vanish and every component's total mass is kept to rounding."""
    _reference(oracle)
    s = CASES["blobs57x41"]()
    w, h = s.width, s.height
    y, x = np.mgrid[0:h + 1, 0:w + 1].astype(float)
    psi = np.sin(np.pi * x / w) * np.sin(np.pi * y / h) * 3.0
    u = psi[1:, :] - psi[:-1, :]          # (h, w + 1)
    v = -(psi[:, 1:] - psi[:, :-1])       # (h + 1, w)
    div = (u[:, 1:] - u[:, :-1]) + (v[1:, :] - v[:-1, :])
    assert np.abs(div).max() < 1e-12
    f, _, _, lm, gm = _reference_advect(oracle, s, u, v, s.dt)
    assert abs(lm.sum() - s.liquid_mass[0].sum()) <= 1e-9 * s.liquid_mass[0].sum()
    assert abs(gm.sum() - s.gas_mass[0].sum()) <= 1e-9 * s.gas_mass[0].sum()
    assert abs(f.sum() - s.fraction.sum()) <= 1e-9 * s.fraction.sum()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("case", sorted(CASES))
def test_gpu_plic_matches_reference(case, precision, oracle):
    from fluidsim_b200 import FluidGrid

    _reference(oracle)
    s = CASES[case]()
    u, v = s.u, s.v
    if precision == "fp32":
        u, v = (a.astype(np.float32).astype(np.float64) for a in (u, v))
    f, uo, vo, lm, gm = _reference_advect(oracle, s, u, v, s.dt)
    g = FluidGrid(s.width, s.height, s.cell_size, precision=precision)
    scenes.upload_scene(g, scenes.Scene(s.width, s.height, s.cell_size, s.dt, s.liquid_density, s.gas_density,
                                        s.fraction, u, v))
    g.setTransport("plic")
    assert g.getTransport() == "plic"
    g.advect(s.dt)
    out = g.download()
    if precision == "fp32":
        uo, vo = (a.astype(np.float32).astype(np.float64) for a in (uo, vo))
    for name, mine, ref in (("fraction", out.liquid_fraction, f), ("u", out.u, uo), ("v", out.v, vo),
                            ("liquid mass", out.liquid_mass[0], lm), ("gas mass", out.gas_mass[0], gm)):
        assert np.array_equal(mine, ref), (name, np.abs(mine - ref).max())


@pytest.mark.gpu
def test_gpu_plic_step_tracks_reference_step(oracle):
    """Whole steps (transport, gravity, projection) with the reference's own step: the FP64
    projections agree to their solver tolerance, so the states stay within 1e-7 of scale."""
    from fluidsim_b200 import FluidGrid

    _reference(oracle)
    s = scenes.dam_break(48, 40, seed=2, obstacles=0, velocity=0.5, gravity=-9.8)
    ref = oracle.ReferenceGrid(s.width, s.height, s.cell_size, s.liquid_density, s.gas_density)
    ref.set_gravity(s.gravity)
    ref.upload(s.fraction, s.u, s.v, None, s.liquid_mass[0], s.gas_mass[0])
    g = FluidGrid(s.width, s.height, s.cell_size, precision="fp64")
    scenes.upload_scene(g, s)
    g.setTransport("plic")
    for _ in range(3):
        rr = ref.step(s.dt, 2000, 1e-10)
        rg = g.step(s.dt, 2000, 1e-10)
        assert rr.converged and rg.converged
    f, u, v, p = ref.download()
    out = g.download()
    scale = max(np.abs(u).max(), np.abs(v).max())
    assert np.abs(out.liquid_fraction - f).max() <= 1e-7
    assert np.abs(out.u - u).max() <= 1e-7 * scale and np.abs(out.v - v).max() <= 1e-7 * scale
