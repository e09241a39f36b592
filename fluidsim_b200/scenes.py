"""Seeded synthetic scenes for the uniform-grid projection workloads.

The reference publishes no dataset for this path; these generators are the full definition of
the inputs (numpy PCG64 streams, so a seed reproduces a scene exactly). Velocities are drawn in
FP64 and rounded to FP32, so the FP32 device path and the FP64 oracle see identical values.

Materials follow the reference's two-phase model (FluidSim/UniformCPU/FluidGridCPU.cpp:1399-1423):
one liquid and one gas component whose masses are density * phase volume, so the cell density
is a volume-weighted mix (the reference test fixture, tests/FluidTestSetup.h:36-61).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np


@dataclass
class Scene:
    width: int
    height: int
    cell_size: float
    dt: float
    liquid_density: float
    gas_density: float
    fraction: np.ndarray          # h x w
    u: np.ndarray                 # h x (w+1)
    v: np.ndarray                 # (h+1) x w
    gravity: float = 0.0
    solid: Optional[np.ndarray] = None  # h x w uint8, or None
    surface_tension: float = 0.0
    name: str = ""
    liquid_mass: List[np.ndarray] = field(default_factory=list)
    gas_mass: List[np.ndarray] = field(default_factory=list)
    # Per-component viscosities (liquid components, then gas); None leaves the grid inviscid.
    liquid_viscosity: Optional[List[float]] = None
    gas_viscosity: Optional[List[float]] = None
    # Air model of the pressure solve: "gas" (the reference's) or "dirichlet" (p = 0 in the air).
    air_model: str = "gas"

    def __post_init__(self):
        area = self.cell_size * self.cell_size
        if not self.liquid_mass:
            self.liquid_mass = [self.liquid_density * self.fraction * area]
        if not self.gas_mass:
            self.gas_mass = [self.gas_density * (1.0 - self.fraction) * area]

    @property
    def cells(self) -> int:
        return self.width * self.height

    def density(self) -> np.ndarray:
        """Sum of component masses over the cell area, in the reference's order."""
        total = np.zeros_like(self.fraction)
        for m in self.liquid_mass + self.gas_mass:
            total = total + m
        return total * (1.0 / (self.cell_size * self.cell_size))


def _f32(a):
    return np.asarray(a, dtype=np.float32).astype(np.float64)


def _random_faces(rng, w, h, amplitude=1.0):
    u = _f32(rng.uniform(-amplitude, amplitude, (h, w + 1)))
    v = _f32(rng.uniform(-amplitude, amplitude, (h + 1, w)))
    return u, v


def _close_walls(u, v):
    u[:, 0] = 0.0
    u[:, -1] = 0.0
    v[0, :] = 0.0
    v[-1, :] = 0.0


def _circles(rng, w, h, count, rmin, rmax):
    solid = np.zeros((h, w), dtype=np.uint8)
    if count == 0:
        return solid
    yy, xx = np.mgrid[0:h, 0:w]
    for _ in range(count):
        r = rng.uniform(rmin, rmax)
        cx = rng.uniform(0, w)
        cy = rng.uniform(0, h)
        solid[(xx + 0.5 - cx) ** 2 + (yy + 0.5 - cy) ** 2 <= r * r] = 1
    return solid


def liquid_box(width=128, height=128, seed=0, dt=1.0 / 60.0) -> Scene:
    """All-liquid closed box, density 1, i.i.d. U[-1, 1] FP32 face velocities, walls zeroed."""
    rng = np.random.default_rng(seed)
    u, v = _random_faces(rng, width, height)
    _close_walls(u, v)
    f = np.ones((height, width))
    return Scene(width, height, 1.0 / width, dt, 1.0, 0.001, f, u, v, name=f"liquid_box_{width}x{height}")


def dam_break(width=1024, height=1024, seed=0, dt=1.0 / 120.0, obstacles=16, block=(200, 300),
              liquid_density=1000.0, gas_density=1.0, gravity=-9.8, velocity=0.0, cell_size=None,
              surface_tension=0.0) -> Scene:
    """Dam break: liquid below half height plus a seeded block, optional circular obstacles.

    Rows are y; gravity acts along y, so the liquid sits in the low rows. Block sizes are in
    cells and shrink with the grid when it is smaller than 1024. The cell size defaults to
    1/width (a unit-wide domain).
    """
    rng = np.random.default_rng(seed)
    f = np.zeros((height, width))
    f[: height // 2, :] = 1.0
    bw = max(1, min(width, block[0] * width // 1024))
    bh = max(1, min(height - height // 2, block[1] * height // 1024))
    x0 = int(rng.integers(0, max(1, width - bw + 1)))
    f[height // 2: height // 2 + bh, x0: x0 + bw] = 1.0
    if velocity:
        u, v = _random_faces(rng, width, height, velocity)
    else:
        u = np.zeros((height, width + 1))
        v = np.zeros((height + 1, width))
    solid = None
    if obstacles:
        scale = width / 1024.0
        solid = _circles(rng, width, height, obstacles, max(1.0, 8 * scale), max(2.0, 40 * scale))
        f[solid != 0] = 0.0
    dx = cell_size if cell_size is not None else 1.0 / width
    return Scene(width, height, dx, dt, liquid_density, gas_density, f, u, v, gravity=gravity,
                 solid=solid, name=f"dam_break_{width}x{height}", surface_tension=surface_tension)


def serving_requests(count, seed=0, min_side=64, max_side=2048, sigma=0.07, cell_size=1.0 / 128.0) -> List[Scene]:
    """Simulation requests of the serving workload: square dam breaks with sides log-uniform in
    [min_side, max_side], surface tension sigma, liquid 1000 and air 1, gravity -9.8, dt 1/120.
    The resolution is fixed (cell_size, default 1/128 m) so the domain grows with the grid; at
    this resolution one capillary substep covers dt = 1/120."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        side = int(round(np.exp(rng.uniform(np.log(min_side), np.log(max_side)))))
        out.append(dam_break(side, side, seed=int(rng.integers(0, 2**31 - 1)), obstacles=0, cell_size=cell_size,
                             surface_tension=sigma))
    return out


def sloped_pool(width, height, cell_size=4.0, dt=1.0 / 120.0, liquid_density=100.0, gas_density=0.1) -> Scene:
    """The reference tests' sloped two-phase pool (tests/FluidGridTests.cpp:627-660) with its
    deterministic sin/cos velocities."""
    y, x = np.mgrid[0:height, 0:width]
    f = np.clip(y + 1.0 - (0.35 * x + 0.2 * height), 0.0, 1.0)
    i_u = np.arange((width + 1) * height)
    i_v = np.arange(width * (height + 1))
    u = (3.0 * np.sin(i_u * 0.07)).reshape(height, width + 1)
    v = (4.0 * np.cos(i_v * 0.11)).reshape(height + 1, width)
    return Scene(width, height, cell_size, dt, liquid_density, gas_density, f, u, v, name=f"sloped_{width}x{height}")


def random_pool(width, height, seed=0, dt=1.0 / 60.0, liquid_density=1000.0, gas_density=1.0, fill=0.5,
                obstacles=0, amplitude=1.0, cell_size=None) -> Scene:
    """Liquid filling the low `fill` fraction of the rows, U[-a, a] FP32 velocities, optional
    circular obstacles (radii up to an eighth of the shorter side)."""
    rng = np.random.default_rng(seed)
    u, v = _random_faces(rng, width, height, amplitude)
    _close_walls(u, v)
    f = np.zeros((height, width))
    level = fill * height
    full = int(np.floor(level))
    f[:full, :] = 1.0
    if full < height:
        f[full, :] = level - full
    solid = None
    if obstacles:
        side = min(width, height)
        solid = _circles(rng, width, height, obstacles, max(1.0, side / 32), max(2.0, side / 8))
        f[solid != 0] = 0.0
    dx = cell_size if cell_size is not None else 1.0 / max(width, height)
    return Scene(width, height, dx, dt, liquid_density, gas_density, f, u, v, solid=solid,
                 name=f"pool_{width}x{height}")


def _fractal_noise(rng, w, h, octaves=7, base=4):
    """Value noise: octave k is a (base * 2^k + 1)^2 lattice of U[0, 1) values, bilinearly
    interpolated to the cell centres (along x on the lattice rows, then along y), with
    amplitude 2^-k."""
    total = np.zeros((h, w))
    for k in range(octaves):
        n = base << k
        lattice = rng.random((n + 1, n + 1))
        xs = (np.arange(w) + 0.5) * (n / w)
        x0 = np.minimum(xs.astype(int), n - 1)
        tx = xs - x0
        rows = lattice[:, x0] * (1 - tx) + lattice[:, x0 + 1] * tx
        ys = (np.arange(h) + 0.5) * (n / h)
        y0 = np.minimum(ys.astype(int), n - 1)
        ty = (ys - y0)[:, None]
        total += (rows[y0] * (1 - ty) + rows[y0 + 1] * ty) * 0.5 ** k
    return total


def _uniform_ranks(a):
    """Maps values to U(0, 1] by rank."""
    ranks = np.empty(a.size)
    ranks[np.argsort(a, axis=None)] = np.arange(1, a.size + 1)
    return ranks / a.size


def viscous_blob(width=4096, height=4096, seed=0, dt=1.0 / 120.0, cover=0.6, mu_range=(1e-3, 10.0),
                 liquid_density=1000.0, gas_density=1.0) -> Scene:
    """Variable-viscosity flow: a fractal-noise liquid blob over `cover` of the domain in air
    (1000:1 density ratio), i.i.d. U[-1, 1] FP32 face velocities with the walls closed, no
    gravity. Inside the liquid the viscosity is log-uniform over `mu_range` along a second
    smooth noise field. The liquid is two components of equal density with the end viscosities;
    the volume-weighted blend of their viscosities (FluidSim/UniformWebGPU/FluidGridGPU.cpp:172-217)
    gives each cell its target. Air has the lower viscosity. The cell size is 1/width."""
    rng = np.random.default_rng(seed)
    blob = _fractal_noise(rng, width, height)
    fraction = (blob >= np.quantile(blob, 1.0 - cover)).astype(float)
    lo, hi = mu_range
    liquid_cells = fraction > 0
    mu = np.full((height, width), lo)
    mu[liquid_cells] = lo * (hi / lo) ** _uniform_ranks(_fractal_noise(rng, width, height)[liquid_cells])
    share = (mu - lo) / (hi - lo)  # volume share of the viscous component in the liquid
    u, v = _random_faces(rng, width, height)
    _close_walls(u, v)
    dx = 1.0 / width
    area = dx * dx
    liquid = [liquid_density * fraction * (1.0 - share) * area, liquid_density * fraction * share * area]
    return Scene(width, height, dx, dt, liquid_density, gas_density, fraction, u, v,
                 name=f"viscous_blob_{width}x{height}", liquid_mass=liquid,
                 gas_mass=[gas_density * (1.0 - fraction) * area], liquid_viscosity=[lo, hi],
                 gas_viscosity=[lo])


def uneven_batch(count=256, seed=0, min_side=64, max_side=1024, max_aspect=2.0, obstacles=True) -> List[Scene]:
    """Independent scenes with log-uniform sides, aspect up to 2:1, fill in [0.3, 0.9],
    0-8 circular obstacles and U[-1, 1] FP32 velocities."""
    rng = np.random.default_rng(seed)
    scenes = []
    for k in range(count):
        while True:
            a = int(round(np.exp(rng.uniform(np.log(min_side), np.log(max_side)))))
            b = int(round(np.exp(rng.uniform(np.log(min_side), np.log(max_side)))))
            if max(a, b) <= max_aspect * min(a, b) and a != b:
                break
        fill = float(rng.uniform(0.3, 0.9))
        n_obstacles = int(rng.integers(0, 9)) if obstacles else 0
        scenes.append(random_pool(a, b, seed=int(rng.integers(0, 2**31 - 1)), fill=fill, obstacles=n_obstacles))
    return scenes


def configure_grid(grid, scene: Scene):
    """Configures a FluidGrid's materials, gravity, surface tension and obstacles from a scene.
    Every component of a phase has the phase's density."""
    grid.configureMaterials([scene.liquid_density] * len(scene.liquid_mass), [scene.gas_density] * len(scene.gas_mass),
                            scene.liquid_viscosity, scene.gas_viscosity)
    grid.setGravityY(scene.gravity)
    grid.setAirModel(scene.air_model)
    if scene.surface_tension:
        grid.setSurfaceTension(scene.surface_tension)
    grid.setObstacles(scene.solid)


def upload_scene(grid, scene: Scene, pressure=None):
    """Configures materials, obstacles and state of a FluidGrid from a scene."""
    from .grid import FluidGridState

    configure_grid(grid, scene)
    grid.upload(FluidGridState(scene.fraction, scene.u, scene.v, pressure, scene.liquid_mass, scene.gas_mass))
