"""The no-allocation divergence entry point against the grid's own divergence check.

fc_divergence_noalloc exists for callers that cannot allocate device memory (a host that owns
all device memory through its own allocator, a process held to a fixed device-memory budget,
a real-time loop that must not stall in the driver). It keeps its scratch in a fixed device
array instead, so this test checks that two calls in a row, on different data, each give the
same answer as fc_max_divergence, which uses the grid's allocated scratch.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _host_divergence(state, dx):
    du = state.u[:, 1:] - state.u[:, :-1]
    dv = state.v[1:, :] - state.v[:-1, :]
    return (du + dv) / dx


def test_noalloc_divergence_matches_allocating_entry_point_twice():
    import torch

    from fluidsim_b200 import FluidGrid, scenes
    from fluidsim_b200 import _native as N

    lib = N.lib()
    stats = torch.zeros(3, dtype=torch.float64, device="cuda")
    for seed, (w, h) in ((3, (300, 200)), (4, (129, 257))):
        s = scenes.random_pool(w, h, seed=seed, fill=0.5, amplitude=2.0)
        g = FluidGrid(s.width, s.height, s.cell_size, "fp32")
        scenes.upload_scene(g, s)
        expected = g.maxDivergence()
        u, v = g.velocityPointers()
        stats.fill_(-1.0)
        torch.cuda.synchronize()
        rc = lib.fc_divergence_noalloc(C.c_void_p(u), C.c_void_p(v), s.width, s.height, s.cell_size, 0,
                                       C.c_void_p(stats.data_ptr()), C.c_void_p(g.stream()))
        assert rc == 0, lib.fc_last_error()
        g.synchronize()
        got = stats.cpu().numpy()
        # The maximum does not depend on the folding order; the tests' FP64 tolerance is 1e-12.
        assert abs(got[0] - expected) <= 1e-12 * expected
        div = _host_divergence(g.download(), s.cell_size)
        assert abs(got[2] - float((div * div).sum())) <= 1e-12 * float((div * div).sum())
        assert 0.0 <= got[1] <= got[0]


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
@pytest.mark.parametrize("size", [(300, 200), (1, 257), (256, 1), (64, 64), (2048, 2048)])
def test_noalloc_statistics_equal_the_projections_own(precision, size):
    """The three statistics against the ones the grid's projection reports from its own
    divergence kernel on the same final velocities: the maximum and the rounding excess are
    maxima of the same per-cell values, so they agree exactly; the sum of squares is folded in
    another order (1e-12 relative). 2048 x 2048 is exactly the 4096-tile limit; 1 x 257 and
    256 x 1 are single-column and single-row grids. Two calls in a row give the same answer."""
    import torch

    from fluidsim_b200 import FluidGrid, scenes
    from fluidsim_b200 import _native as N

    w, h = size
    s = scenes.random_pool(w, h, seed=w + 7 * h, fill=0.5, amplitude=2.0)
    g = FluidGrid(s.width, s.height, s.cell_size, precision)
    scenes.upload_scene(g, s)
    r = g.project(s.dt, 3, 1e-6)  # a few iterations: a non-trivial divergence field
    u, v = g.velocityPointers()
    code = N.PRECISION[precision]
    stats = torch.zeros(3, dtype=torch.float64, device="cuda")
    for _ in range(2):
        stats.fill_(-1.0)
        torch.cuda.synchronize()
        rc = N.lib().fc_divergence_noalloc(C.c_void_p(u), C.c_void_p(v), w, h, s.cell_size, code,
                                           C.c_void_p(stats.data_ptr()), C.c_void_p(g.stream()))
        assert rc == 0, N.lib().fc_last_error()
        g.synchronize()
        got = stats.cpu().numpy()
        assert got[0] == r.max_divergence
        assert got[1] == r.divergence_excess
        assert abs(got[2] - r.divergence_l2 ** 2) <= 1e-12 * r.divergence_l2 ** 2


def test_noalloc_rejects_grids_beyond_its_scratch():
    import torch

    from fluidsim_b200 import _native as N

    stats = torch.zeros(3, dtype=torch.float64, device="cuda")
    dummy = C.c_void_p(stats.data_ptr())
    rc = N.lib().fc_divergence_noalloc(dummy, dummy, 4096, 4097, 1.0, 0, dummy, None)
    assert rc == 1
    assert b"4,194,304" in N.lib().fc_last_error()
