"""Serving loop: admission by device-memory budget, continuous batching, results that do not
depend on the mix.

The reference drives one scene at a time (FluidSim/FluidScene.inl:328-420). The serving loop
runs many simulations at once; its contract is that each simulation's final state is exactly
the state fc_step produces when the simulation runs alone.
"""
import numpy as np
import pytest


# ----------------------------------------------------------------------------------------------
# CPU: host-side logic (no device call)
# ----------------------------------------------------------------------------------------------


def test_device_bytes_is_host_arithmetic():
    from fluidsim_b200.serving import grid_device_bytes

    small = grid_device_bytes(64, 64)
    big = grid_device_bytes(2048, 2048)
    assert 0 < small < big
    assert grid_device_bytes(512, 512, "fp64") > grid_device_bytes(512, 512, "fp32")
    assert grid_device_bytes(512, 512, surface_tension=True) > grid_device_bytes(512, 512)
    assert grid_device_bytes(512, 512, components=4) == grid_device_bytes(512, 512, components=2) + 2 * 512 * 512 * 8 + 16
    # A 2048^2 FP32 grid with tension stays well under 1 GB: hundreds fit a 150 GB budget.
    assert grid_device_bytes(2048, 2048, surface_tension=True) < 1 << 30


def test_device_bytes_rejects_bad_descriptions():
    from fluidsim_b200 import FluidInvalidArgument
    from fluidsim_b200.serving import grid_device_bytes

    for args in ((0, 10), (10, -1)):
        with pytest.raises(FluidInvalidArgument):
            grid_device_bytes(*args)
    with pytest.raises(KeyError):
        grid_device_bytes(8, 8, "fp16")


def test_poisson_arrivals_rate():
    from fluidsim_b200.serving import poisson_arrivals

    t = poisson_arrivals(200.0, 20000, seed=1)
    assert np.all(np.diff(t) > 0)
    assert abs(t[-1] / len(t) - 1.0 / 200.0) < 0.05 / 200.0


def test_serving_requests_are_seeded_dam_breaks():
    from fluidsim_b200 import scenes

    a = scenes.serving_requests(32, seed=4)
    b = scenes.serving_requests(32, seed=4)
    assert [s.width for s in a] == [s.width for s in b]
    assert all(np.array_equal(x.fraction, y.fraction) for x, y in zip(a, b))
    assert all(64 <= s.width <= 2048 and s.width == s.height for s in a)
    assert all(s.surface_tension == 0.07 and s.cell_size == 1.0 / 128.0 for s in a)
    assert all(s.liquid_density == 1000.0 and s.gas_density == 1.0 for s in a)


def test_size_class_bounds_are_validated_before_any_device_call():
    import ctypes as C

    from fluidsim_b200 import FluidInvalidArgument
    from fluidsim_b200 import _native as N

    handle = C.c_void_p()
    for classes, bounds in ((0, []), (17, [1] * 16), (3, [100, 100]), (3, [200, 100]), (2, [0]), (3, [-5, 10])):
        arr = (C.c_longlong * max(1, len(bounds)))(*bounds)
        with pytest.raises(FluidInvalidArgument):
            N.check(N.lib().fc_server_create_classes(1 << 30, 4, classes, arr, C.byref(handle)))
    with pytest.raises(FluidInvalidArgument):
        N.check(N.lib().fc_server_create_classes(1 << 30, 4, 2, None, C.byref(handle)))


# ----------------------------------------------------------------------------------------------
# GPU: the serving loop through the C ABI
# ----------------------------------------------------------------------------------------------


def _alone(scene, steps, precision):
    from fluidsim_b200 import FluidGrid, scenes

    g = FluidGrid(scene.width, scene.height, scene.cell_size, precision=precision)
    scenes.upload_scene(g, scene)
    iterations, converged = 0, True
    for _ in range(steps):
        r = g.step(scene.dt, 200, 1e-6)
        iterations += r.iterations
        converged &= r.converged
    return g.download(), iterations, converged


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_gpu_each_result_is_the_same_alone_and_in_the_mix(precision):
    from fluidsim_b200 import scenes
    from fluidsim_b200.serving import Server, grid_device_bytes, poisson_arrivals, serve

    reqs = scenes.serving_requests(6, seed=11, min_side=40, max_side=160)
    reqs.append(scenes.dam_break(72, 50, seed=5, obstacles=3, velocity=0.5, cell_size=1.0 / 128.0,
                                 surface_tension=0.07))
    steps = 5
    need = [grid_device_bytes(s.width, s.height, precision, 2, True) for s in reqs]
    # Room for about half of them at a time: admission has to wait for memory.
    budget = max(max(need), sum(need) // 2)
    server = Server(budget, max_active=64)
    out = serve(server, reqs, poisson_arrivals(200.0, len(reqs), seed=2), steps, precision=precision)
    stats = server.stats()
    assert 1 <= stats["peak_active"] < len(reqs) and stats["peak_bytes"] <= budget
    assert stats["steps"] == steps * len(reqs)
    assert stats["cell_steps"] == steps * sum(s.cells for s in reqs)
    assert len(server.step_latencies()) == stats["steps"]
    for scene, sim, st in zip(reqs, out["ids"], out["statuses"]):
        assert st.state == "done" and st.steps_done == steps
        mixed = server.download(sim)
        alone, iterations, converged = _alone(scene, steps, precision)
        assert st.iterations == iterations and st.converged == converged
        for name in ("liquid_fraction", "u", "v", "pressure"):
            assert np.array_equal(getattr(mixed, name), getattr(alone, name)), (scene.name, name)
        for a, b in zip(mixed.liquid_mass + mixed.gas_mass, alone.liquid_mass + alone.gas_mass):
            assert np.array_equal(a, b)
        server.release(sim)
    server.close()


@pytest.mark.gpu
@pytest.mark.parametrize("size_classes", [[48 * 48, 100 * 100], []], ids=["three_classes", "lockstep"])
def test_gpu_size_classes_step_each_simulation_as_alone(size_classes):
    """Grids of three size classes (two bounds) run by three workers side by side, and the same
    mix in one lockstep class: every simulation ends exactly as it ends alone, each class counts
    its own steps, and the classes' statistics add up to the server's."""
    from fluidsim_b200 import scenes
    from fluidsim_b200.serving import Server, poisson_arrivals, serve

    reqs = [scenes.dam_break(n, n, seed=n, obstacles=2, velocity=0.5, cell_size=1.0 / 128.0, surface_tension=0.07)
            for n in (24, 40, 56, 64, 90, 100, 120, 150)]
    steps = 4
    server = Server(1 << 34, max_active=64, size_classes=size_classes)
    out = serve(server, reqs, poisson_arrivals(400.0, len(reqs), seed=3), steps)
    assert all(st.state == "done" for st in out["statuses"]), [(s.name, st) for s, st in zip(reqs, out["statuses"])]
    stats, per_class = server.stats(), server.class_stats()
    assert len(per_class) == len(size_classes) + 1
    bounds = list(size_classes) + [None]
    for k, c in enumerate(per_class):
        expect = [s for s in reqs if (k == 0 or s.cells > bounds[k - 1]) and (bounds[k] is None or s.cells <= bounds[k])]
        assert c["steps"] == steps * len(expect)
        assert c["cell_steps"] == steps * sum(s.cells for s in expect)
        if bounds[k] is not None:
            assert c["max_cells"] == bounds[k]
    assert stats["steps"] == sum(c["steps"] for c in per_class) == steps * len(reqs)
    assert stats["ticks"] == sum(c["ticks"] for c in per_class)
    assert len(server.step_latencies()) == stats["steps"]
    for scene, sim, st in zip(reqs, out["ids"], out["statuses"]):
        assert st.state == "done" and st.steps_done == steps
        mixed = server.download(sim)
        alone, iterations, converged = _alone(scene, steps, "fp32")
        assert st.iterations == iterations and st.converged == converged
        for name in ("liquid_fraction", "u", "v", "pressure"):
            assert np.array_equal(getattr(mixed, name), getattr(alone, name)), (scene.name, name)
        server.release(sim)
    server.close()


@pytest.mark.gpu
def test_gpu_server_rejects_what_can_never_fit():
    from fluidsim_b200 import FluidInvalidArgument, FluidLifecycleError, scenes
    from fluidsim_b200.serving import Server, grid_device_bytes

    scene = scenes.dam_break(128, 128, obstacles=0)
    server = Server(grid_device_bytes(64, 64), max_active=4)
    with pytest.raises(FluidInvalidArgument):
        server.submit(scene, 1)
    small = scenes.dam_break(32, 32, obstacles=0)
    sim = server.submit(small, 2)
    st = server.wait(sim, 120.0)
    assert st.state == "done" and st.steps_done == 2
    with pytest.raises(FluidInvalidArgument):
        server.status(sim + 100)
    assert server.error(sim) == ""
    server.release(sim)
    # A time step that would need more capillary substeps than an int holds fails the
    # simulation at admission (FluidGridCPU.cpp:309-320 throws there); the server keeps why.
    import dataclasses

    doomed = server.submit(dataclasses.replace(small, dt=1e12, surface_tension=0.07), 1)
    st = server.wait(doomed, 120.0)
    assert st.state == "failed" and "substeps" in server.error(doomed)
    server.release(doomed)
    with pytest.raises(FluidInvalidArgument):
        server.release(sim)
    server.close()
