"""Python mirror of FluidSim's FluidGrid engine contract over the UniformCUDA C ABI.

Names, argument meaning and error behaviour follow fluid::FluidGridBase
(FluidSim/FluidGridBase.h:20-147) and fluid::FluidGridState / FluidProjectionResult
(FluidSim/FluidGridTypes.h:10-80): ``upload`` takes the FP64 host state, ``step`` and ``project``
return a ProjectionResult, size mismatches raise ValueError before any state changes (the
reference's std::invalid_argument, FluidGridCPU.cpp:205-218), and use before upload raises the
lifecycle error (std::logic_error).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

from . import _native as N

_dp = C.POINTER(C.c_double)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_dp)


def _as_f64(values, shape, name):
    if values is None:
        return None
    a = np.ascontiguousarray(values, dtype=np.float64)
    if a.size != int(np.prod(shape)):
        raise ValueError(f"{name}: expected {int(np.prod(shape))} values, got {a.size}")
    return a.reshape(shape)


@dataclass
class FluidGridState:
    """fluid::FluidGridState<double>: empty fields mean zero."""
    liquid_fraction: Optional[np.ndarray] = None
    u: Optional[np.ndarray] = None
    v: Optional[np.ndarray] = None
    pressure: Optional[np.ndarray] = None
    liquid_mass: List[np.ndarray] = field(default_factory=list)
    gas_mass: List[np.ndarray] = field(default_factory=list)


@dataclass
class ProjectionResult:
    """fluid::FluidProjectionResult, plus the solver's own measurements."""
    iterations: int = 0
    max_divergence: float = float("inf")
    converged: bool = False
    physical_steps: int = 1
    transport_steps: int = 0
    relaxed: bool = False
    max_volume_error: float = 0.0
    rms_volume_error: float = 0.0
    viscosity_iterations: int = 0
    precision_limited: bool = False
    solve_status: str = "running"
    residual_max: float = float("nan")
    residual_l2: float = float("nan")
    rhs_l2: float = float("nan")
    divergence_excess: float = float("nan")
    divergence_l2: float = float("nan")
    restarts: int = 0
    kernels: int = 0
    refreshes: int = 0

    def accepted(self) -> bool:
        """FluidProjectionResult::accepted (FluidGridTypes.h:76)."""
        return self.converged or self.relaxed or self.precision_limited

    @property
    def relative_residual(self) -> float:
        return self.residual_l2 / self.rhs_l2 if self.rhs_l2 > 0 else 0.0

    @classmethod
    def from_c(cls, r: N.FcResult) -> "ProjectionResult":
        return cls(r.iterations, r.max_divergence, bool(r.converged), r.physical_steps, r.transport_steps,
                   bool(r.relaxed), r.max_volume_error, r.rms_volume_error, r.viscosity_iterations,
                   bool(r.precision_limited), N.SOLVE_STATUS.get(r.solve_status, str(r.solve_status)),
                   r.residual_max, r.residual_l2, r.rhs_l2, r.divergence_excess, r.divergence_l2,
                   r.restarts, r.kernels, r.refreshes)


class FluidGrid:
    """The UniformCUDA engine for one uniform MAC grid (FluidGridCPU's public surface)."""

    def __init__(self, width: int, height: int, cell_size: float, precision: str = "fp32"):
        if precision not in N.PRECISION:
            raise ValueError(f"unknown precision {precision!r}")
        handle = C.c_void_p()
        N.check(N.lib().fc_create(int(width), int(height), float(cell_size), N.PRECISION[precision], C.byref(handle)))
        self._h = handle
        self.width, self.height, self.cell_size = int(width), int(height), float(cell_size)
        self.precision = precision
        self._liquid: List[float] = []
        self._gas: List[float] = []

    # -- lifecycle --------------------------------------------------------------------------
    def destroy(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            N.check(N.lib().fc_destroy(self._h))
        self._h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    @property
    def handle(self):
        if self._h is None:
            raise N.FluidLifecycleError(2, "grid destroyed")
        return self._h

    # -- geometry and settings --------------------------------------------------------------
    def getWidth(self) -> int:
        return self.width

    def getHeight(self) -> int:
        return self.height

    def getCellSize(self) -> float:
        return self.cell_size

    def getOrigin(self):
        x, y = C.c_double(), C.c_double()
        N.check(N.lib().fc_get_origin(self.handle, C.byref(x), C.byref(y)))
        return (x.value, y.value)

    def setOrigin(self, origin):
        N.check(N.lib().fc_set_origin(self.handle, float(origin[0]), float(origin[1])))

    def requiresRenderThread(self) -> bool:
        return False

    def configureMaterials(self, liquid_densities: Sequence[float], gas_densities: Sequence[float],
                           liquid_viscosities: Optional[Sequence[float]] = None,
                           gas_viscosities: Optional[Sequence[float]] = None):
        ld = np.ascontiguousarray(liquid_densities, dtype=np.float64)
        gd = np.ascontiguousarray(gas_densities, dtype=np.float64)
        lv = None if liquid_viscosities is None else np.ascontiguousarray(liquid_viscosities, dtype=np.float64)
        gv = None if gas_viscosities is None else np.ascontiguousarray(gas_viscosities, dtype=np.float64)
        N.check(N.lib().fc_configure_materials(self.handle, len(ld), _ptr(ld), _ptr(lv), len(gd), _ptr(gd), _ptr(gv)))
        self._liquid = list(map(float, ld))
        self._gas = list(map(float, gd))

    def getGravityY(self) -> float:
        g = C.c_double()
        N.check(N.lib().fc_get_gravity(self.handle, C.byref(g)))
        return g.value

    def setGravityY(self, acceleration: float):
        N.check(N.lib().fc_set_gravity(self.handle, float(acceleration)))

    def setPreconditioner(self, which: str):
        N.check(N.lib().fc_set_preconditioner(self.handle, N.PRECONDITIONER[which]))

    def setObstacles(self, solid: Optional[np.ndarray]):
        if solid is None:
            N.check(N.lib().fc_set_obstacles(self.handle, None))
            return
        s = np.ascontiguousarray(solid, dtype=np.uint8)
        if s.size != self.width * self.height:
            raise ValueError("obstacle mask must have width*height cells")
        N.check(N.lib().fc_set_obstacles(self.handle, s.ctypes.data_as(C.POINTER(C.c_uint8))))

    # -- state ------------------------------------------------------------------------------
    def upload(self, state: FluidGridState):
        w, h = self.width, self.height
        f = _as_f64(state.liquid_fraction, (h, w), "liquid_fraction")
        u = _as_f64(state.u, (h, w + 1), "u")
        v = _as_f64(state.v, (h + 1, w), "v")
        p = _as_f64(state.pressure, (h, w), "pressure")
        lm = [_as_f64(m, (h, w), "liquid_mass") for m in state.liquid_mass]
        gm = [_as_f64(m, (h, w), "gas_mass") for m in state.gas_mass]
        if lm and len(lm) != len(self._liquid):
            raise ValueError("upload component count does not match the mixture")
        if gm and len(gm) != len(self._gas):
            raise ValueError("upload component count does not match the mixture")
        lp = (_dp * max(1, len(lm)))(*[_ptr(m) for m in lm]) if lm else None
        gp = (_dp * max(1, len(gm)))(*[_ptr(m) for m in gm]) if gm else None
        N.check(N.lib().fc_upload(self.handle, _ptr(f), _ptr(u), _ptr(v), _ptr(p), lp, gp))

    def download(self) -> FluidGridState:
        w, h = self.width, self.height
        f = np.empty((h, w))
        u = np.empty((h, w + 1))
        v = np.empty((h + 1, w))
        p = np.empty((h, w))
        lm = [np.empty((h, w)) for _ in self._liquid]
        gm = [np.empty((h, w)) for _ in self._gas]
        lp = (_dp * max(1, len(lm)))(*[_ptr(m) for m in lm]) if lm else None
        gp = (_dp * max(1, len(gm)))(*[_ptr(m) for m in gm]) if gm else None
        N.check(N.lib().fc_download(self.handle, _ptr(f), _ptr(u), _ptr(v), _ptr(p), lp, gp))
        return FluidGridState(f, u, v, p, lm, gm)

    def saveCheckpoint(self):
        """Returns (metadata dict, payload bytes) of the native "cuda-uniform" checkpoint."""
        import json

        mb, pb = C.c_size_t(), C.c_size_t()
        N.check(N.lib().fc_save_checkpoint(self.handle, None, 0, C.byref(mb), None, 0, C.byref(pb)))
        meta = C.create_string_buffer(mb.value)
        payload = C.create_string_buffer(max(1, pb.value))
        N.check(N.lib().fc_save_checkpoint(self.handle, meta, mb.value, C.byref(mb), payload, pb.value, C.byref(pb)))
        return json.loads(meta.value.decode()), payload.raw[: pb.value]

    def loadCheckpoint(self, metadata, payload: bytes):
        import json

        text = metadata if isinstance(metadata, str) else json.dumps(metadata)
        buf = C.create_string_buffer(payload, len(payload))
        N.check(N.lib().fc_load_checkpoint(self.handle, text.encode(), buf, len(payload)))
        m = json.loads(text)
        self._liquid = [c["density"] for c in m["liquid_mixture"]]
        self._gas = [c["density"] for c in m["gas_mixture"]]

    def copyStateFrom(self, other: "FluidGrid"):
        N.check(N.lib().fc_copy_state(self.handle, other.handle))

    # -- stepping ---------------------------------------------------------------------------
    def step(self, dt: float, max_iterations: int = 200, divergence_tolerance: float = 1e-6,
             timings: Optional[dict] = None) -> ProjectionResult:
        # Without a timings request the step enqueues each substep's stages without waiting
        # between them; with one, every stage waits so that its time is its own.
        r, t = N.FcResult(), N.FcTimings()
        N.check(N.lib().fc_step(self.handle, float(dt), int(max_iterations), float(divergence_tolerance),
                                C.byref(r), C.byref(t) if timings is not None else None))
        if timings is not None:
            timings.update({k: getattr(t, k) for k, _ in N.FcTimings._fields_})
        return ProjectionResult.from_c(r)

    def project(self, dt: float, max_iterations: int = 200, divergence_tolerance: float = 1e-6,
                relative_tolerance: Optional[float] = None) -> ProjectionResult:
        r = N.FcResult()
        if relative_tolerance is None:
            N.check(N.lib().fc_project(self.handle, float(dt), int(max_iterations), float(divergence_tolerance),
                                       C.byref(r)))
        else:
            N.check(N.lib().fc_project_relative(self.handle, float(dt), int(max_iterations),
                                                float(relative_tolerance), float(divergence_tolerance), C.byref(r)))
        return ProjectionResult.from_c(r)

    def setAirModel(self, model: str):
        """'gas' (the reference's two-phase model, default) or 'dirichlet' (air held at p = 0,
        the free-surface boundary; see fc_set_air_model)."""
        if model not in N.AIR_MODEL:
            raise ValueError(f"unknown air model {model!r}")
        N.check(N.lib().fc_set_air_model(self.handle, N.AIR_MODEL[model]))

    def extendAirVelocity(self):
        """The liquid's face velocities extended into Dirichlet air (fc_extend_air_velocity)."""
        N.check(N.lib().fc_extend_air_velocity(self.handle))

    def setStreamPriority(self, priority: int):
        """CUDA stream priority of the grid's work (fc_set_stream_priority; lower runs first)."""
        N.check(N.lib().fc_set_stream_priority(self.handle, int(priority)))

    def advanceSubstep(self, dt: float) -> int:
        """fc_step's substep before the projection, enqueued without waiting (fc_advance_substep);
        returns the viscosity iterations."""
        it = C.c_int()
        N.check(N.lib().fc_advance_substep(self.handle, float(dt), C.byref(it)))
        return it.value

    def getAirModel(self) -> str:
        m = C.c_int()
        N.check(N.lib().fc_get_air_model(self.handle, C.byref(m)))
        return {v: k for k, v in N.AIR_MODEL.items()}[m.value]

    def setTransport(self, scheme: str):
        """'semi_lagrangian' (default) or 'plic' (UniformCPU's conservative transport)."""
        N.check(N.lib().fc_set_transport(self.handle, N.TRANSPORT[scheme]))

    def getTransport(self) -> str:
        out = C.c_int()
        N.check(N.lib().fc_get_transport(self.handle, C.byref(out)))
        return {v: k for k, v in N.TRANSPORT.items()}[out.value]

    def advect(self, dt: float):
        """Semi-Lagrangian transport of velocities, liquid fraction and component masses."""
        N.check(N.lib().fc_advect(self.handle, float(dt)))

    def applyViscosity(self, dt: float, tolerance: float = 1e-4, max_iterations: int = -1):
        """Implicit viscosity step; returns (iterations, relative residual)."""
        it, rel = C.c_int(), C.c_double()
        N.check(N.lib().fc_apply_viscosity(self.handle, float(dt), float(tolerance), int(max_iterations),
                                           C.byref(it), C.byref(rel)))
        return it.value, rel.value

    def setComponentViscosity(self, phase: str, component: int, coefficient: float):
        N.check(N.lib().fc_set_component_viscosity(self.handle, {"liquid": 0, "gas": 1}[phase], int(component),
                                                   float(coefficient)))

    def autotune(self, repeats: int = 10):
        """Picks the fastest multigrid tail threshold for this grid; returns (cells, V-cycle ms)."""
        cells, ms = C.c_int(), C.c_double()
        N.check(N.lib().fc_autotune(self.handle, int(repeats), C.byref(cells), C.byref(ms)))
        return cells.value, ms.value

    def setTailCells(self, cells: int):
        N.check(N.lib().fc_set_tail_cells(self.handle, int(cells)))

    def getSurfaceTension(self) -> float:
        out = C.c_double()
        N.check(N.lib().fc_get_surface_tension(self.handle, C.byref(out)))
        return out.value

    def setSurfaceTension(self, coefficient: float):
        N.check(N.lib().fc_set_surface_tension(self.handle, float(coefficient)))

    def capillaryStepLimit(self) -> float:
        out = C.c_double()
        N.check(N.lib().fc_capillary_step_limit(self.handle, C.byref(out)))
        return out.value

    def applySurfaceTension(self, dt: float):
        N.check(N.lib().fc_apply_surface_tension(self.handle, float(dt)))

    def surfaceCurvature(self):
        """Completed height-function curvature per cell (1/length) and its validity mask."""
        k = np.empty((self.height, self.width))
        ok = np.empty((self.height, self.width), dtype=np.uint8)
        N.check(N.lib().fc_surface_curvature(self.handle, k.ctypes.data, ok.ctypes.data))
        return k, ok.astype(bool)

    def sampleVelocity(self, positions) -> np.ndarray:
        """FluidGridCPU::sampleVelocity at world positions, shape (n, 2) -> (n, 2)."""
        pos = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1, 2)
        out = np.empty_like(pos)
        N.check(N.lib().fc_sample_velocity(self.handle, pos.shape[0], pos.ctypes.data, out.ctypes.data))
        return out

    def applyGravity(self, dt: float):
        N.check(N.lib().fc_apply_gravity(self.handle, float(dt)))

    def maxDivergence(self) -> float:
        out = C.c_double()
        N.check(N.lib().fc_max_divergence(self.handle, C.byref(out)))
        return out.value

    def classify(self) -> np.ndarray:
        mask = np.empty((self.height, self.width), dtype=np.uint8)
        N.check(N.lib().fc_classify(self.handle, mask.ctypes.data_as(C.POINTER(C.c_uint8))))
        return mask

    def downloadCoefficients(self):
        """The fine level's (inv_u, inv_v, inv_diagonal) in the reference's layout
        (FluidGridCPU::rebuildPressureCoefficients, FluidGridCPU.cpp:1154-1205)."""
        w, h = self.width, self.height
        inv_u, inv_v, inv_d = np.zeros((h, w + 1)), np.zeros((h + 1, w)), np.zeros((h, w))
        N.check(N.lib().fc_download_coefficients(self.handle, _ptr(inv_u), _ptr(inv_v), _ptr(inv_d)))
        return inv_u, inv_v, inv_d

    def applyPreconditioner(self, residual: np.ndarray, residual_mean: float = 0.0) -> np.ndarray:
        r = _as_f64(residual, (self.height, self.width), "residual")
        z = np.empty((self.height, self.width))
        N.check(N.lib().fc_apply_preconditioner(self.handle, _ptr(r), float(residual_mean), _ptr(z)))
        return z

    def timeKernel(self, kernel: int, repeats: int = 10) -> float:
        """Mean milliseconds of one projection kernel, timed with CUDA events on the grid's stream."""
        ms = C.c_double()
        N.check(N.lib().fc_time_kernel(self.handle, int(kernel), int(repeats), C.byref(ms)))
        return ms.value

    def synchronize(self):
        N.check(N.lib().fc_synchronize(self.handle))

    def stream(self) -> int:
        s = C.c_void_p()
        N.check(N.lib().fc_get_stream(self.handle, C.byref(s)))
        return s.value or 0

    def velocityPointers(self):
        u, v = C.c_void_p(), C.c_void_p()
        N.check(N.lib().fc_velocity_pointers(self.handle, C.byref(u), C.byref(v)))
        return u.value, v.value


class ProjectionBatch:
    """Many independent grids projected together: one launch per kernel for the whole batch."""

    def __init__(self, grids: Sequence[FluidGrid]):
        arr = (C.c_void_p * len(grids))(*[g.handle.value for g in grids])
        handle = C.c_void_p()
        N.check(N.lib().fc_batch_create(arr, len(grids), C.byref(handle)))
        self._h = handle
        self.grids = list(grids)

    def destroy(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            N.check(N.lib().fc_batch_destroy(self._h))
        self._h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    def project(self, dts, max_iterations: int = 200, divergence_tolerance: float = 1e-6,
                relative_tolerance: float = 0.0) -> List[ProjectionResult]:
        n = len(self.grids)
        d = np.ascontiguousarray(np.broadcast_to(np.asarray(dts, dtype=np.float64), (n,)))
        results = (N.FcResult * n)()
        N.check(N.lib().fc_batch_project(self._h, _ptr(d), int(max_iterations), float(divergence_tolerance),
                                         float(relative_tolerance), results))
        return [ProjectionResult.from_c(results[i]) for i in range(n)]

    def stream(self) -> int:
        s = C.c_void_p()
        N.check(N.lib().fc_batch_get_stream(self._h, C.byref(s)))
        return s.value or 0

    def autotune(self, repeats: int = 10):
        """Picks the fastest multigrid tail threshold for the batch; returns (cells, V-cycle ms).
        The batch's stream changes (its plan is rebuilt)."""
        cells, ms = C.c_int(), C.c_double()
        N.check(N.lib().fc_batch_autotune(self._h, int(repeats), C.byref(cells), C.byref(ms)))
        return cells.value, ms.value
