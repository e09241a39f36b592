"""Dirichlet air (p = 0 in the air, the free-surface boundary of the dam-break workload) in the
FP64 restatement: the known answer it must meet, and how it leaves the reference's gas model
untouched. The reference has no such model (its air is a light gas component of a closed,
mean-free system, FluidGridCPU.cpp:1063-1090), so this restatement is pinned by the known
answer and by the equations it must satisfy, not by reference outputs."""
import numpy as np
import pytest

from fluidsim_b200 import scenes


def _hydrostatic(oracle, w=12, h=20, liquid_rows=8, dx=0.1, dt=0.01, g=-9.8, rl=1000.0, ra=1.0, obstacle=False):
    f = np.zeros((h, w))
    f[:liquid_rows, :] = 1.0
    solid = None
    if obstacle:
        solid = np.zeros((h, w), dtype=np.uint8)
        solid[2:4, 3:6] = 1  # a block inside the liquid
        f[solid != 0] = 0.0
    density = rl * f + ra * (1.0 - f)
    o = oracle.OracleGrid(w, h, dx)
    o.upload(density, np.zeros((h, w + 1)), np.zeros((h + 1, w)), solid=solid, air=oracle.air_mask(f, solid))
    o.apply_gravity(g, dt)
    r = o.project(dt, 400, 1e-10)
    u, v, p = o.download()
    return r, u, v, p, f, solid


def test_hydrostatic_free_surface_known_answer(oracle):
    """A liquid layer at rest under gravity with air above: the liquid stays at rest, the air
    holds p = 0 and the liquid pressure is hydrostatic from the free surface. The top liquid
    cell's face to the air has weight 2 / (rho_l + rho_a), so p_top = -g dx (rho_l + rho_a) / 2,
    and every row below adds -rho_l g dx. Exact in FP64 to 1e-10 relative."""
    rl, ra, g, dx = 1000.0, 1.0, -9.8, 0.1
    r, u, v, p, f, _ = _hydrostatic(oracle, rl=rl, ra=ra, g=g, dx=dx)
    assert r.converged
    top = 7
    p_top = -g * dx * (rl + ra) / 2.0
    expected = np.array([p_top - (top - y) * rl * g * dx for y in range(top + 1)])
    for x in range(p.shape[1]):
        assert np.abs(p[: top + 1, x] - expected).max() <= 1e-10 * np.abs(expected).max()
    assert np.all(p[top + 1:] == 0.0)
    assert np.abs(v[1: top + 1]).max() <= 1e-10  # liquid faces, interface included
    assert np.abs(u).max() <= 1e-10


def test_hydrostatic_with_an_obstacle_in_the_liquid(oracle):
    """An obstacle inside the liquid changes nothing for the cells beside it: the liquid is still
    at rest (its faces hold no velocity) and the air still holds zero."""
    r, u, v, p, f, solid = _hydrostatic(oracle, obstacle=True)
    assert r.converged
    assert np.abs(v[1:8]).max() <= 1e-9 and np.abs(u).max() <= 1e-9
    assert np.all(p[8:] == 0.0) and np.all(p[solid != 0] == 0.0)


def test_air_mask_is_the_complement_of_liquid_and_solid(oracle):
    f = np.array([[0.0, 0.5, 0.5000001, 1.0], [0.2, 0.7, 0.0, 1.0]])
    solid = np.array([[0, 0, 0, 1], [1, 0, 0, 0]], dtype=np.uint8)
    air = oracle.air_mask(f, solid)
    assert air.tolist() == [[1, 1, 0, 0], [0, 0, 1, 0]]
    assert oracle.air_mask(f).tolist() == [[1, 1, 0, 0], [1, 0, 1, 0]]


@pytest.mark.parametrize("size,obstacles", [((33, 25), 0), ((64, 48), 3), ((65, 37), 0)])
def test_projection_makes_the_liquid_divergence_free(oracle, size, obstacles):
    """Random pools: after the projection the liquid cells meet the stop rule on the velocity
    divergence; the air cells are not constrained, and their pressure is zero."""
    w, h = size
    s = scenes.random_pool(w, h, seed=w + h, fill=0.55, obstacles=obstacles)
    air = oracle.air_mask(s.fraction, s.solid)
    o = oracle.OracleGrid(w, h, s.cell_size)
    o.upload(s.density(), s.u, s.v, solid=s.solid, air=air)
    r = o.project(s.dt, 400, 1e-8)
    u, v, p = o.download()
    assert r.converged and r.max_divergence <= 1e-8
    div = ((u[:, 1:] - u[:, :-1]) + (v[1:, :] - v[:-1, :])) / s.cell_size
    liquid = (air == 0) & (s.solid == 0 if s.solid is not None else True)
    assert np.abs(div[liquid]).max() <= 1e-8
    assert np.all(p[air != 0] == 0.0)
    # The air moves freely: its divergence is not driven to zero.
    assert np.abs(div[air != 0]).max() > 1.0


def test_gas_model_is_unchanged_by_the_air_switch(oracle):
    """Setting and clearing the Dirichlet mask gives the gas model's projection bit for bit."""
    s = scenes.random_pool(40, 30, seed=3, fill=0.6)
    a = oracle.OracleGrid(40, 30, s.cell_size)
    a.upload(s.density(), s.u, s.v)
    ra = a.project(s.dt, 200, 1e-6)
    b = oracle.OracleGrid(40, 30, s.cell_size)
    b.upload(s.density(), s.u, s.v, air=oracle.air_mask(s.fraction))
    b.upload(s.density(), s.u, s.v, air=None)
    rb = b.project(s.dt, 200, 1e-6)
    assert ra.iterations == rb.iterations
    for x, y in zip(a.download(), b.download()):
        assert np.array_equal(x, y)
