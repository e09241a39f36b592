"""The "cuda-uniform" checkpoint: exact continuation after save/load, and validation before any
state changes (the reference's contract, FluidSim/FluidGridBase.h:121-125; its WebGPU test
saves, reloads and compares, tests/FluidWebGPUAPITests.cpp:500-)."""
import json

import numpy as np
import pytest

from fluidsim_b200 import FluidGrid, FluidInvalidArgument, scenes

pytestmark = pytest.mark.gpu


def _grid(scene, precision):
    g = FluidGrid(scene.width, scene.height, scene.cell_size, precision)
    scenes.upload_scene(g, scene)
    return g


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_checkpoint_continues_exactly(precision):
    s = scenes.random_pool(96, 72, seed=12, fill=0.55, obstacles=2, cell_size=1.0 / 96)
    a = _grid(s, precision)
    a.setGravityY(-9.8)
    a.step(s.dt, 200, 1e-6)
    meta, payload = a.saveCheckpoint()
    assert meta["backend"] == "cuda-uniform" and meta["version"] == 1
    assert meta["width"] == 96 and meta["obstacles"] is True
    assert len(payload) == meta["payload_bytes"]

    b = FluidGrid(s.width, s.height, s.cell_size, precision)
    b.loadCheckpoint(meta, payload)
    assert b.getGravityY() == -9.8
    sa, sb = a.download(), b.download()
    for field in ("liquid_fraction", "u", "v", "pressure"):
        assert np.array_equal(getattr(sa, field), getattr(sb, field)), field
    # The next steps (which warm-start from the pressure history) agree bit for bit.
    for _ in range(2):
        ra, rb = a.step(s.dt, 200, 1e-6), b.step(s.dt, 200, 1e-6)
        assert ra.iterations == rb.iterations
    sa, sb = a.download(), b.download()
    assert np.array_equal(sa.u, sb.u) and np.array_equal(sa.v, sb.v) and np.array_equal(sa.pressure, sb.pressure)
    assert np.array_equal(sa.liquid_mass[0], sb.liquid_mass[0]) and np.array_equal(sa.gas_mass[0], sb.gas_mass[0])


def test_checkpoint_rejects_incompatible_input_before_changing_state():
    s = scenes.random_pool(64, 48, seed=13, fill=0.5, cell_size=1.0 / 64)
    a = _grid(s, "fp32")
    meta, payload = a.saveCheckpoint()
    target = _grid(scenes.random_pool(64, 48, seed=14, fill=0.3, cell_size=1.0 / 64), "fp32")
    before = target.download()

    def rejected(m, p):
        with pytest.raises(FluidInvalidArgument):
            target.loadCheckpoint(m, p)
        after = target.download()
        assert np.array_equal(before.u, after.u) and np.array_equal(before.liquid_fraction, after.liquid_fraction)

    rejected(dict(meta, backend="webgpu-uniform"), payload)
    rejected(dict(meta, version=2), payload)
    rejected(dict(meta, width=65), payload)
    rejected(dict(meta, scalar="float64"), payload)
    rejected(meta, payload[:-8])
    rejected("{not json", payload)
    # Numbers are checked before any cast: finite, integral and in range.
    rejected(dict(meta, width=1e300), payload)
    rejected(dict(meta, version=-1), payload)
    rejected(dict(meta, version=1.5), payload)
    rejected(dict(meta, precision=2 ** 40), payload)
    rejected(dict(meta, payload_bytes=-8), payload)
    rejected(dict(meta, preconditioner=1e30), payload)
    text = json.dumps(meta)
    # 1e999 parses as infinity: a non-finite gravity, origin or density is refused.
    rejected(text.replace('"gravity_y": ' + json.dumps(meta["gravity_y"]), '"gravity_y": 1e999'), payload)
    rejected(json.dumps(dict(meta, origin=[0.0, "x"])), payload)
    rejected(text.replace('"origin": ' + json.dumps(meta["origin"]), '"origin": [1e999, 0]'), payload)
    other = FluidGrid(64, 48, 1.0 / 64, "fp64")
    with pytest.raises(FluidInvalidArgument):
        other.loadCheckpoint(meta, payload)
