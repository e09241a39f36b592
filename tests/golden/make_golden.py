"""Generates the golden fixtures of the projection from the reference engine itself.

Runs FluidSim's own UniformCPU code (FluidSim/UniformCPU/FluidGridCPU.cpp and
PressureMultigrid.cpp, compiled from the reference sources into oracle/_ref/libfluidref.so by
oracle/Makefile) on seeded inputs and stores inputs and outputs as .npz files next to this
script. Needs the reference checkout, so it runs only where that exists:

    make -C oracle && python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from fluidsim_b200 import scenes  # noqa: E402


def projection_case(name, scene, max_iterations, tolerance, preconditioner="multigrid"):
    g = O.ReferenceGrid(scene.width, scene.height, scene.cell_size, scene.liquid_density, scene.gas_density)
    g.set_preconditioner(preconditioner == "multigrid")
    g.upload(scene.fraction, scene.u, scene.v, None, scene.liquid_mass[0], scene.gas_mass[0])
    # Inputs that are exact in FP32 (the seeded scenes) are stored in FP32.
    exact32 = all(np.array_equal(a.astype(np.float32).astype(np.float64), a) for a in (scene.u, scene.v))
    store = (lambda a: a.astype(np.float32)) if exact32 else (lambda a: a)
    r = g.project(scene.dt, max_iterations, tolerance)
    _, u, v, p = g.download()
    inv_u, inv_v, inv_d = g.coefficients()
    np.savez_compressed(
        os.path.join(HERE, f"project_{name}.npz"),
        width=scene.width, height=scene.height, cell_size=scene.cell_size, dt=scene.dt,
        liquid_density=scene.liquid_density, gas_density=scene.gas_density,
        fraction=scene.fraction, u_in=store(scene.u), v_in=store(scene.v),
        max_iterations=max_iterations, tolerance=tolerance, preconditioner=preconditioner,
        iterations=r.iterations, converged=r.converged, max_divergence=r.max_divergence,
        u=u, v=v, p=p, inv_u=inv_u, inv_v=inv_v, inv_diagonal=inv_d)
    print(name, scene.width, scene.height, "iterations", r.iterations, "maxdiv", r.max_divergence)


def multigrid_case(name, w, h):
    """The reference test's checkerboard densities (tests/FluidGridTests.cpp:538-625)."""
    y, x = np.mgrid[0:h, 0:w]
    density = np.where(((x // 3 + y // 4) % 2) == 0, 0.1, 100.0)
    inv_u, inv_v, _ = O.coefficients(density)
    i = np.arange(w * h)
    a = (np.sin(i * 0.31) + np.cos(i * 0.073)).reshape(h, w)
    a -= a.mean()
    z = O.reference_mg_apply(inv_u, inv_v, a, 0.0)
    np.savez_compressed(os.path.join(HERE, f"multigrid_{name}.npz"), width=w, height=h, density=density,
                        residual=a, correction=z)
    print(name, w, h, "levels", O.Multigrid(w, h).levels)


def hydrostatic_case():
    """A full tank after one step with gravity (tests/FluidGridTests.cpp:140-160)."""
    w, h, dx = 12, 10, 2.0
    g = O.ReferenceGrid(w, h, dx, 100.0, 0.1)
    f = np.ones((h, w))
    g.upload(f, None, None, None, 100.0 * f * dx * dx, 0.1 * (1 - f) * dx * dx)
    r = g.step(1.0 / 120.0, 2000, 1e-8)
    _, u, v, p = g.download()
    np.savez_compressed(os.path.join(HERE, "hydrostatic_12x10.npz"), width=w, height=h, cell_size=dx,
                        dt=1.0 / 120.0, gravity=100.0, liquid_density=100.0, gas_density=0.1,
                        iterations=r.iterations, converged=r.converged, u=u, v=v, p=p)
    print("hydrostatic", r.iterations, "rise", p[h - 1, 0] - p[0, 0])


def sampler_case():
    """FluidGridCPU::sampleVelocity on a 9 x 7 grid with origin (-7, 11) and cell size 2.5 (the
    geometry of tests/FluidGridTests.cpp:53-93), seeded velocities, positions inside and outside
    the sample domain."""
    w, h, dx, origin = 9, 7, 2.5, (-7.0, 11.0)
    rng = np.random.default_rng(53)
    u = rng.standard_normal((h, w + 1))
    v = rng.standard_normal((h + 1, w))
    g = O.ReferenceGrid(w, h, dx)
    g.set_origin(*origin)
    g.upload(np.zeros((h, w)), u, v)
    positions = np.column_stack([rng.uniform(-12.0, 20.0, 512), rng.uniform(5.0, 35.0, 512)])
    velocities = g.sample_velocity(positions)
    np.savez_compressed(os.path.join(HERE, "sampler_9x7.npz"), width=w, height=h, cell_size=dx,
                        origin=np.array(origin), u=u, v=v, positions=positions, velocities=velocities)
    print("sampler", positions.shape[0], "positions")


def antialiased(w, h, inside, sub=8):
    """Liquid fraction of each cell from sub x sub point samples of an inside(x, y) test."""
    y, x = np.mgrid[0:h, 0:w].astype(float)
    f = np.zeros((h, w))
    for sy in range(sub):
        for sx in range(sub):
            f += inside(x + (sx + 0.5) / sub, y + (sy + 0.5) / sub)
    return f / (sub * sub)


def tension_case(name, fraction, cell_size, sigma=0.07, dt=1.0 / 120.0, seed=0):
    """FluidGridCPU::applySurfaceTension and FluidSurfaceTensionCPU's curvature, run by the
    reference itself on one liquid (1000) and one gas (1) component."""
    h, w = fraction.shape
    rng = np.random.default_rng(seed)
    u = rng.uniform(-1.0, 1.0, (h, w + 1))
    v = rng.uniform(-1.0, 1.0, (h + 1, w))
    area = cell_size * cell_size
    g = O.ReferenceGrid(w, h, cell_size, 1000.0, 1.0)
    g.set_surface_tension(sigma)
    g.upload(fraction, u, v, None, 1000.0 * fraction * area, 1.0 * (1.0 - fraction) * area)
    limit = g.capillary_step_limit()
    g.apply_surface_tension(dt)
    _, u_out, v_out, _ = g.download()
    kappa, valid = O.reference_surface_curvature(fraction, cell_size)
    np.savez_compressed(os.path.join(HERE, f"tension_{name}.npz"), width=w, height=h, cell_size=cell_size,
                        sigma=sigma, dt=dt, fraction=fraction, u_in=u, v_in=v, u=u_out, v=v_out,
                        curvature=kappa, valid=valid, capillary_step_limit=limit)
    print("tension", name, "valid", int(valid.sum()), "max |du|", np.abs(u_out - u).max())


def tension_cases():
    drop = antialiased(48, 40, lambda x, y: (x - 24.0) ** 2 + (y - 20.0) ** 2 < 12.0 ** 2)
    tension_case("drop48x40", drop, 1.0 / 48.0)
    wave = antialiased(64, 48, lambda x, y: y > 24.0 + 4.0 * np.sin(2.0 * np.pi * x / 32.0))
    tension_case("wave64x48", wave, 1.0 / 64.0, seed=1)
    # Seeded blobs, thin filaments and near-pure cells a few ulps from 0 and 1.
    rng = np.random.default_rng(17)
    blobs = np.zeros((37, 53))
    for _ in range(9):
        cx, cy, r = rng.uniform(0, 53), rng.uniform(0, 37), rng.uniform(1.0, 7.0)
        blobs = np.maximum(blobs, antialiased(53, 37, lambda x, y: (x - cx) ** 2 + (y - cy) ** 2 < r * r))
    blobs[5, 3:40] = np.maximum(blobs[5, 3:40], 0.3)
    blobs[blobs == 1.0] -= 4e-16 * (rng.uniform(size=(blobs == 1.0).sum()) < 0.2)
    blobs[blobs == 0.0] += 3e-17 * (rng.uniform(size=(blobs == 0.0).sum()) < 0.2)
    tension_case("blobs53x37", blobs, 0.02, sigma=0.5, seed=2)


def main():
    O.build(reference=True)
    O.set_reference_threads(1)
    projection_case("box128", scenes.liquid_box(128, 128, seed=0), 200, 1e-6)
    for (w, h) in [(13, 9), (65, 37), (2, 67), (1, 129), (131, 1)]:
        projection_case(f"sloped{w}x{h}", scenes.sloped_pool(w, h), 4000, 1e-8)
    projection_case("sloped65x37_diagonal", scenes.sloped_pool(65, 37), 4000, 1e-8, preconditioner="diagonal")
    projection_case("pool64x48", scenes.random_pool(64, 48, seed=3, fill=0.6, cell_size=1.0 / 64), 200, 1e-6)
    for (w, h) in [(1, 1), (13, 9), (65, 37)]:
        multigrid_case(f"{w}x{h}", w, h)
    hydrostatic_case()
    sampler_case()
    tension_cases()


if __name__ == "__main__":
    main()
