"""Serving: many simulations on one GPU with continuous batching (fc_server_* in fluidcuda.h).

The request loop lives in the native library (fluidsim_b200/csrc/fc_server.cpp): simulations are
sorted by grid size into classes, and each class's worker thread admits simulations by the shared
device-memory budget, keeps their state on the device across steps and projects its running
grids in one batched solve per tick. This module is its Python face, plus the Poisson arrival
driver used by the serving measurement.
"""
from __future__ import annotations

import ctypes as C
import threading
import time
from dataclasses import dataclass
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import _native as N
from .grid import FluidGridState
from .scenes import Scene

SIM_STATES = {0: "queued", 1: "running", 2: "done", 3: "failed"}


@dataclass
class SimStatus:
    state: str
    error: int
    steps_done: int
    physical_steps: int
    iterations: int
    converged: bool
    max_divergence: float
    queued_ms: float
    run_ms: float
    device_bytes: int

    @classmethod
    def of(cls, s: N.FcSimStatus) -> "SimStatus":
        return cls(SIM_STATES.get(s.state, str(s.state)), s.error, s.steps_done, s.physical_steps, s.iterations,
                   bool(s.converged), s.max_divergence, s.queued_ms, s.run_ms, s.device_bytes)


def grid_device_bytes(width: int, height: int, precision: str = "fp32", components: int = 2,
                      surface_tension: bool = False) -> int:
    """Device bytes one grid holds once running: the admission figure of the serving loop."""
    out = C.c_size_t()
    N.check(N.lib().fc_grid_device_bytes(int(width), int(height), N.PRECISION[precision], int(components),
                                         1 if surface_tension else 0, C.byref(out)))
    return out.value


class Server:
    """Continuous-batching request loop over one GPU.

    size_classes: increasing cell-count bounds of the size classes (a class per bound plus one
    for larger grids), each stepped by its own worker; None for the library's default (up to
    128 x 128, 256 x 256, 512 x 512, 1024 x 1024, larger); [] for one class that steps everything
    in lockstep."""

    def __init__(self, device_budget_bytes: int, max_active: int = 256, size_classes: Optional[Sequence[int]] = None):
        handle = C.c_void_p()
        if size_classes is None:
            N.check(N.lib().fc_server_create(int(device_budget_bytes), int(max_active), C.byref(handle)))
        else:
            bounds = (C.c_longlong * max(1, len(size_classes)))(*[int(b) for b in size_classes])
            N.check(N.lib().fc_server_create_classes(int(device_budget_bytes), int(max_active), len(size_classes) + 1,
                                                     bounds, C.byref(handle)))
        self._h = handle
        self._shapes: Dict[int, tuple] = {}

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            N.check(N.lib().fc_server_destroy(self._h))
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, scene: Scene, steps: int, max_iterations: int = 200, divergence_tolerance: float = 1e-6,
               precision: str = "fp32") -> int:
        """Queues a simulation of `scene` for `steps` time steps of scene.dt; returns its id."""
        w, h = scene.width, scene.height
        keep = []

        def arr(a, dtype=np.float64):
            if a is None:
                return None
            b = np.ascontiguousarray(a, dtype=dtype)
            keep.append(b)
            return b.ctypes.data

        def ptrs(arrays):
            if not arrays:
                return None
            table = (C.c_void_p * len(arrays))(*[arr(a) for a in arrays])
            keep.append(table)
            return C.cast(table, C.c_void_p).value

        d = N.FcSimDesc()
        d.width, d.height, d.cell_size = w, h, float(scene.cell_size)
        d.precision = N.PRECISION[precision]
        d.liquid_count, d.liquid_densities = 1, arr([scene.liquid_density])
        d.gas_count, d.gas_densities = 1, arr([scene.gas_density])
        d.gravity_y = float(scene.gravity)
        d.surface_tension = float(scene.surface_tension)
        d.solid = arr(scene.solid, np.uint8) if scene.solid is not None else None
        d.liquid_fraction, d.u, d.v = arr(scene.fraction), arr(scene.u), arr(scene.v)
        d.pressure = None
        d.liquid_mass, d.gas_mass = ptrs(scene.liquid_mass), ptrs(scene.gas_mass)
        d.steps, d.dt = int(steps), float(scene.dt)
        d.max_iterations, d.divergence_tolerance = int(max_iterations), float(divergence_tolerance)
        out = C.c_longlong()
        N.check(N.lib().fc_server_submit(self._h, C.byref(d), C.byref(out)))
        self._shapes[out.value] = (w, h, len(scene.liquid_mass), len(scene.gas_mass))
        return out.value

    def status(self, sim: int) -> SimStatus:
        s = N.FcSimStatus()
        N.check(N.lib().fc_server_status(self._h, sim, C.byref(s)))
        return SimStatus.of(s)

    def wait(self, sim: int, timeout: float = 600.0) -> SimStatus:
        s = N.FcSimStatus()
        N.check(N.lib().fc_server_wait(self._h, sim, float(timeout), C.byref(s)))
        return SimStatus.of(s)

    def download(self, sim: int) -> FluidGridState:
        w, h, nl, ng = self._shapes[sim]
        f, p = np.empty((h, w)), np.empty((h, w))
        u, v = np.empty((h, w + 1)), np.empty((h + 1, w))
        lm = [np.empty((h, w)) for _ in range(nl)]
        gm = [np.empty((h, w)) for _ in range(ng)]
        lt = (C.c_void_p * max(nl, 1))(*[a.ctypes.data for a in lm])
        gt = (C.c_void_p * max(ng, 1))(*[a.ctypes.data for a in gm])
        N.check(N.lib().fc_server_download(self._h, sim, f.ctypes.data, u.ctypes.data, v.ctypes.data, p.ctypes.data,
                                           C.cast(lt, C.c_void_p) if nl else None,
                                           C.cast(gt, C.c_void_p) if ng else None))
        return FluidGridState(f, u, v, p, lm, gm)

    def error(self, sim: int) -> str:
        """Why a simulation failed ('' unless it did)."""
        buf = C.create_string_buffer(1024)
        N.check(N.lib().fc_server_error(self._h, sim, buf, len(buf)))
        return buf.value.decode(errors="replace")

    def release(self, sim: int):
        N.check(N.lib().fc_server_release(self._h, sim))
        self._shapes.pop(sim, None)

    def stats(self) -> dict:
        s = N.FcServerStats()
        N.check(N.lib().fc_server_get_stats(self._h, C.byref(s)))
        return {name: getattr(s, name) for name, _ in N.FcServerStats._fields_}

    def class_stats(self) -> List[dict]:
        """Statistics of each size class, with its cell bound under 'max_cells'."""
        count = C.c_int()
        N.check(N.lib().fc_server_class_count(self._h, C.byref(count)))
        out = []
        for k in range(count.value):
            s, bound = N.FcServerStats(), C.c_longlong()
            N.check(N.lib().fc_server_get_class_stats(self._h, k, C.byref(s), C.byref(bound)))
            d = {name: getattr(s, name) for name, _ in N.FcServerStats._fields_}
            d["max_cells"] = bound.value
            out.append(d)
        return out

    def step_latencies(self) -> np.ndarray:
        count = C.c_size_t()
        N.check(N.lib().fc_server_step_latencies(self._h, None, 0, C.byref(count)))
        out = np.empty(count.value)
        N.check(N.lib().fc_server_step_latencies(self._h, out.ctypes.data, out.size, C.byref(count)))
        return out


def poisson_arrivals(rate: float, count: int, seed: int = 0) -> np.ndarray:
    """Arrival times (seconds from the start) of a Poisson stream with mean `rate` per second."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, count))


def serve(server: Server, scenes: Sequence[Scene], arrivals: Sequence[float], steps: int,
          max_iterations: int = 200, divergence_tolerance: float = 1e-6, precision: str = "fp32",
          timeout: float = 3600.0) -> dict:
    """Submits scenes[i] at arrivals[i] seconds (a submitting thread sleeps between arrivals),
    waits for every simulation and returns ids, statuses and the wall time from the first arrival
    to the last completion."""
    ids: List[Optional[int]] = [None] * len(scenes)
    error: List[BaseException] = []
    start = time.perf_counter()

    def submitter():
        try:
            for i, (scene, at) in enumerate(zip(scenes, arrivals)):
                delay = start + float(at) - time.perf_counter()
                if delay > 0:
                    time.sleep(delay)
                ids[i] = server.submit(scene, steps, max_iterations, divergence_tolerance, precision)
        except BaseException as e:  # surfaced to the caller below
            error.append(e)

    thread = threading.Thread(target=submitter)
    thread.start()
    thread.join()
    if error:
        raise error[0]
    statuses = [server.wait(i, timeout) for i in ids]
    wall = time.perf_counter() - start - float(arrivals[0])
    return {"ids": ids, "statuses": statuses, "wall_s": wall}
