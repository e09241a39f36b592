"""The multigrid tail (the coarse levels one CTA cycles as register strips) against the oracle's
PressureMultigrid restatement, V-cycle by V-cycle (PressureMultigrid.cpp:386-434).

Every tail threshold moves levels between the strip kernels and the tail. The FP64 V-cycle must
match the restatement to rounding at every threshold. This holds for shapes that stress the
tail's strip layout: the widest and tallest levels it takes (64 columns or rows), odd sides
whose coarse cells keep a shorter last cell, and strips one or two cells thin."""
import numpy as np
import pytest

from fluidsim_b200 import FluidGrid, scenes

pytestmark = pytest.mark.gpu

SHAPES = [(64, 64), (63, 64), (64, 45), (127, 2), (2, 130), (190, 130), (257, 129), (1000, 3)]


def _case(w, h):
    y, x = np.mgrid[0:h, 0:w]
    density = np.where(((x // 3 + y // 5) % 2) == 0, 0.1, 100.0) * (1.0 + 0.25 * np.sin(0.37 * x + 0.11 * y))
    i = np.arange(w * h, dtype=float)
    residual = (np.sin(i * 0.29) + np.cos(i * 0.061)).reshape(h, w)
    return density, residual - residual.mean()


@pytest.mark.parametrize("cells", [64, 256, 1024, 4096])
@pytest.mark.parametrize("size", SHAPES, ids=lambda s: f"{s[0]}x{s[1]}")
def test_vcycle_matches_restatement_at_every_tail_threshold(oracle, size, cells):
    w, h = size
    density, residual = _case(w, h)
    inv_u, inv_v, _ = oracle.coefficients(density)
    mg = oracle.Multigrid(w, h)
    assert mg.rebuild(inv_u, inv_v)
    expected = mg.apply(residual)

    s = scenes.Scene(w, h, 1.0, 1.0, 1.0, 1.0, np.ones((h, w)), np.zeros((h, w + 1)), np.zeros((h + 1, w)),
                     liquid_mass=[density], gas_mass=[np.zeros((h, w))])
    g = FluidGrid(w, h, 1.0, "fp64")
    scenes.upload_scene(g, s)
    g.setTailCells(cells)
    z = g.applyPreconditioner(residual)
    scale = max(1.0, np.abs(expected).max())
    assert np.abs(z - expected).max() <= 1e-10 * scale


@pytest.mark.parametrize("size", [(64, 64), (190, 130), (1000, 3)], ids=lambda s: f"{s[0]}x{s[1]}")
def test_fp32_tail_stays_close_to_fp64(size):
    """The FP32 tail differs from the FP64 one only by rounding."""
    w, h = size
    density, residual = _case(w, h)
    s = scenes.Scene(w, h, 1.0, 1.0, 1.0, 1.0, np.ones((h, w)), np.zeros((h, w + 1)), np.zeros((h + 1, w)),
                     liquid_mass=[density], gas_mass=[np.zeros((h, w))])
    out = {}
    for precision in ("fp64", "fp32"):
        g = FluidGrid(w, h, 1.0, precision)
        scenes.upload_scene(g, s)
        g.setTailCells(4096)
        out[precision] = g.applyPreconditioner(residual)
    scale = max(1.0, np.abs(out["fp64"]).max())
    assert np.abs(out["fp32"] - out["fp64"]).max() <= 5e-4 * scale
