"""The CPU oracle pinned against the reference: golden fixtures made by the reference engine,
the live reference engine (when built here), and the reference tests' known answers."""
import glob
import os

import numpy as np
import pytest

from conftest import GOLDEN, golden
from fluidsim_b200 import scenes


def _density(d):
    f = d["fraction"]
    area = float(d["cell_size"]) ** 2
    lm = float(d["liquid_density"]) * f * area
    gm = float(d["gas_density"]) * (1.0 - f) * area
    return (lm + gm) * (1.0 / area)


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "project_*.npz"))), ids=os.path.basename)
def test_restatement_matches_reference_fixture(oracle, path):
    d = golden(os.path.basename(path))
    w, h = int(d["width"]), int(d["height"])
    g = oracle.OracleGrid(w, h, float(d["cell_size"]))
    g.set_preconditioner(str(d["preconditioner"]) == "multigrid")
    density = _density(d)
    g.upload(density, d["u_in"].astype(np.float64), d["v_in"].astype(np.float64))
    r = g.project(float(d["dt"]), int(d["max_iterations"]), float(d["tolerance"]))
    u, v, p = g.download()
    # Coefficients: same formula, same order -> bit-exact.
    inv_u, inv_v, inv_d = oracle.coefficients(density)
    assert np.array_equal(inv_u, d["inv_u"]) and np.array_equal(inv_v, d["inv_v"])
    assert np.array_equal(inv_d, d["inv_diagonal"])
    assert r.iterations == int(d["iterations"])
    assert bool(r.converged) == bool(d["converged"])
    scale = max(1.0, np.abs(d["u"]).max(), np.abs(d["v"]).max())
    assert np.abs(u - d["u"]).max() <= 1e-9 * scale
    assert np.abs(v - d["v"]).max() <= 1e-9 * scale
    pscale = max(1e-300, np.abs(d["p"]).max())
    assert np.abs(p - d["p"]).max() <= 1e-9 * pscale


@pytest.mark.parametrize("name", ["1x1", "13x9", "65x37"])
def test_multigrid_matches_reference_fixture(oracle, name):
    d = golden(f"multigrid_{name}.npz")
    w, h = int(d["width"]), int(d["height"])
    inv_u, inv_v, _ = oracle.coefficients(d["density"])
    mg = oracle.Multigrid(w, h)
    assert mg.rebuild(inv_u, inv_v)
    z = mg.apply(d["residual"])
    assert np.abs(z - d["correction"]).max() <= 1e-12 * max(1.0, np.abs(d["correction"]).max())


@pytest.mark.parametrize("size", [(1, 1), (1, 129), (131, 1), (2, 67), (13, 9), (64, 64), (65, 37), (256, 256)])
def test_multigrid_contract(oracle, size):
    """Linear, symmetric, positive, history-free, constant-annihilating (FluidGridTests.cpp:538-625)."""
    w, h = size
    y, x = np.mgrid[0:h, 0:w]
    density = np.where(((x // 3 + y // 4) % 2) == 0, 0.1, 100.0)
    inv_u, inv_v, _ = oracle.coefficients(density)
    mg = oracle.Multigrid(w, h)
    assert mg.rebuild(inv_u, inv_v)
    i = np.arange(w * h)
    a = (np.sin(i * 0.31) + np.cos(i * 0.073)).reshape(h, w)
    b = (np.cos(i * 0.17) - np.sin(i * 0.019)).reshape(h, w)
    a -= a.mean()
    b -= b.mean()
    ma, mb, mc = mg.apply(a), mg.apply(b), mg.apply(1.3 * a - 0.7 * b)
    assert np.array_equal(ma, mg.apply(a))
    ma, mb, mc = ma - ma.mean(), mb - mb.mean(), mc - mc.mean()
    assert np.abs(mc - (1.3 * ma - 0.7 * mb)).max() <= 1e-10 * max(1.0, np.abs(mc).max())
    ea, eb = float((a * ma).sum()), float((b * mb).sum())
    assert abs(float((a * mb).sum()) - float((b * ma).sum())) <= 1e-10 * max(1.0, np.sqrt(abs(ea * eb)))
    if w * h == 1:
        assert ea == 0.0
    else:
        assert ea > 0.0 and eb > 0.0
    assert np.all(mg.apply(np.full((h, w), 7.0), 7.0) == 0.0)


def test_hydrostatic_known_answer(oracle):
    """Full tank: gravity cancelled, pressure rises by rho g dx (H-1) (FluidGridTests.cpp:140-160)."""
    d = golden("hydrostatic_12x10.npz")
    w, h, dx = int(d["width"]), int(d["height"]), float(d["cell_size"])
    g = oracle.OracleGrid(w, h, dx)
    g.upload(np.full((h, w), 100.0), None, None)
    g.apply_gravity(100.0, float(d["dt"]))
    r = g.project(float(d["dt"]), 2000, 1e-8)
    u, v, p = g.download()
    assert r.converged
    assert np.abs(v).max() < 1e-7
    expected = 100.0 * 100.0 * dx * (h - 1)
    rise = p[h - 1, 0] - p[0, 0]
    assert abs(rise - expected) < expected * 1e-8
    # and the reference's own step gives the same fields
    assert np.abs(p - d["p"]).max() <= 1e-9 * np.abs(d["p"]).max()
    assert np.abs(v - d["v"]).max() <= 1e-12


def test_classification_thresholds(oracle):
    f = np.array([[0.0, 1e-300, 0.5, np.nextafter(0.5, 1.0)], [1.0, np.nextafter(1.0, 0.0), 0.7, 0.2]])
    solid = np.array([[0, 0, 0, 0], [0, 0, 1, 0]], dtype=np.uint8)
    m = oracle.classify(f, solid)
    assert m.tolist() == [[0, 2, 2, 3], [1, 3, 4, 2]]


def test_obstacles_project_to_divergence_free(oracle):
    s = scenes.random_pool(80, 56, seed=5, fill=0.6, obstacles=5, cell_size=1.0 / 80)
    g = oracle.OracleGrid(s.width, s.height, s.cell_size)
    g.upload(s.density(), s.u, s.v, None, solid=s.solid)
    r = g.project(s.dt, 500, 1e-7)
    u, v, p = g.download()
    assert r.converged and r.max_divergence <= 1e-7
    assert np.all(p[s.solid != 0] == 0.0)
    # closed faces carry no flow
    ys, xs = np.nonzero(s.solid)
    assert np.all(u[ys, xs] == 0.0) and np.all(u[ys, xs + 1] == 0.0)
    assert np.all(v[ys, xs] == 0.0) and np.all(v[ys + 1, xs] == 0.0)


def test_relative_rule(oracle):
    s = scenes.liquid_box(96, 64, seed=2)
    g = oracle.OracleGrid(s.width, s.height, s.cell_size)
    g.upload(s.density(), s.u, s.v)
    r = g.project(s.dt, 200, 1e-6, relative_tolerance=1e-6)
    assert r.residual_l2 <= 1e-6 * r.rhs_l2


needs_reference = pytest.mark.skipif(
    not os.path.exists(os.path.join(os.path.dirname(GOLDEN), "..", "oracle", "_ref", "libfluidref.so")),
    reason="reference engine not built here")


@needs_reference
@pytest.mark.parametrize("size", [(13, 9), (65, 37), (2, 67), (100, 70), (129, 65)])
def test_restatement_matches_live_reference(oracle, size):
    w, h = size
    s = scenes.random_pool(w, h, seed=w * 7 + h, fill=0.55, cell_size=1.0 / w)
    ref = oracle.ReferenceGrid(w, h, s.cell_size, s.liquid_density, s.gas_density)
    ref.upload(s.fraction, s.u, s.v, None, s.liquid_mass[0], s.gas_mass[0])
    rr = ref.project(s.dt, 300, 1e-6)
    _, ur, vr, pr = ref.download()
    g = oracle.OracleGrid(w, h, s.cell_size)
    g.upload(s.density(), s.u, s.v)
    gr = g.project(s.dt, 300, 1e-6)
    ug, vg, pg = g.download()
    assert gr.iterations == rr.iterations and gr.converged == rr.converged
    assert np.abs(ug - ur).max() <= 1e-8 * max(1.0, np.abs(ur).max())
    assert np.abs(pg - pr).max() <= 1e-8 * np.abs(pr).max()


@pytest.mark.parametrize("size", [(1, 129), (131, 1), (2, 67), (65, 47), (128, 128)], ids=lambda s: f"{s[0]}x{s[1]}")
def test_restatement_multigrid_matches_diagonal(oracle, size):
    """FluidGridTests.cpp:627-660: both preconditioners give the same velocities within 2e-6."""
    s = scenes.sloped_pool(*size)
    out = []
    for multigrid in (True, False):
        g = oracle.OracleGrid(s.width, s.height, s.cell_size)
        g.set_preconditioner(multigrid)
        g.upload(s.density(), s.u, s.v)
        assert g.project(1.0 / 120.0, 4000, 1e-8).converged
        out.append(g.download())
    assert np.abs(out[0][0] - out[1][0]).max() < 2e-6 and np.abs(out[0][1] - out[1][1]).max() < 2e-6


def test_restatement_large_mixed_pressure_within_default_budget(oracle):
    """FluidGridTests.cpp:662-681: the 512x512 sloped pool converges within 200 iterations."""
    s = scenes.sloped_pool(512, 512)
    g = oracle.OracleGrid(512, 512, s.cell_size)
    g.upload(s.density(), s.u, s.v)
    r = g.project(1.0 / 120.0)
    assert r.converged and r.max_divergence <= 1e-6


def test_restatement_matches_live_reference_on_odd_grid(oracle):
    """FluidGridTests.cpp:683-708's 513x257 grid: the restatement and the reference engine itself
    agree within the reference test's 2e-7."""
    w, h = 513, 257
    y, x = np.mgrid[0:h, 0:w]
    f = np.clip(y + 1.0 - (0.3 * x + 30.0), 0.0, 1.0)
    u = np.sin(np.arange((w + 1) * h) * 0.03).reshape(h, w + 1)
    v = np.cos(np.arange(w * (h + 1)) * 0.017).reshape(h + 1, w)
    ref = oracle.ReferenceGrid(w, h, 1.0, 100.0, 0.1)
    ref.upload(f, u, v, None, 100.0 * f, 0.1 * (1.0 - f))
    rr = ref.project(0.004, 2000, 1e-8)
    _, ur, vr, _ = ref.download()
    g = oracle.OracleGrid(w, h, 1.0)
    g.upload(100.0 * f + 0.1 * (1.0 - f), u, v)
    gr = g.project(0.004, 2000, 1e-8)
    ug, vg, _ = g.download()
    assert rr.converged and gr.converged
    assert np.abs(ug - ur).max() < 2e-7 and np.abs(vg - vr).max() < 2e-7
