"""ctypes access to the CPU oracle (test infrastructure only).

Two libraries, both FP64 on the host:

* ``_build/liboracle.so``: the C restatement of the UniformCPU projection (fluid_oracle.c).
* ``_ref/libfluidref.so``: the reference engine itself (FluidSim/UniformCPU/FluidGridCPU.cpp and
  PressureMultigrid.cpp), compiled from the reference sources by oracle/Makefile when the
  reference checkout is present. It travels with the repository snapshot as a built file.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libfluidref.so")

_dp = C.POINTER(C.c_double)
_u8p = C.POINTER(C.c_uint8)


def reference_checkout():
    """Root of the reference checkout whose sources the reference build compiles: the
    FLUIDSIM_REFERENCE environment variable, else the checkout beside this build's working
    tree; None when neither holds FluidSim/UniformCPU/FluidGridCPU.cpp."""
    for root in (os.environ.get("FLUIDSIM_REFERENCE"), "/root/reference"):
        if root and os.path.isfile(os.path.join(root, "FluidSim", "UniformCPU", "FluidGridCPU.cpp")):
            return root
    return None


def json_include_dir():
    """A directory holding nlohmann/json.hpp (the JSON type bitloop's checkpoint metadata
    follows), from the Python environment's site-packages; None when absent."""
    import sysconfig

    for base in {sysconfig.get_paths()["purelib"], sysconfig.get_paths()["platlib"]}:
        d = os.path.join(base, "include", "cudnn_frontend", "thirdparty")
        if os.path.isfile(os.path.join(d, "nlohmann", "json.hpp")):
            return d
    return None


def build(reference: bool = True) -> None:
    """Compile the restatement, and the reference engine when its sources are present."""
    targets = ["all"] if reference else ["oracle"]
    extra = []
    root = reference_checkout() if reference else None
    if root:
        extra.append(f"REFERENCE={root}")
        inc = json_include_dir()
        if inc:
            extra.append(f"JSON_INCLUDE={inc}")
    subprocess.run(["make", "-s", "-f", os.path.join(HERE, "Makefile")] + targets + extra, check=True)


def _ptr(a):
    if a is None:
        return None
    return a.ctypes.data_as(_dp)


def _f64(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


class _OrResult(C.Structure):
    _fields_ = [("iterations", C.c_int), ("converged", C.c_int), ("max_divergence", C.c_double),
                ("residual_max", C.c_double), ("residual_l2", C.c_double), ("rhs_l2", C.c_double)]


class _RefResult(C.Structure):
    _fields_ = [("iterations", C.c_int), ("converged", C.c_int), ("max_divergence", C.c_double),
                ("elapsed_ms", C.c_double)]


@dataclass
class ProjectionResult:
    iterations: int
    converged: bool
    max_divergence: float
    residual_max: float = float("nan")
    residual_l2: float = float("nan")
    rhs_l2: float = float("nan")
    elapsed_ms: float = float("nan")


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build(reference=False)
        L = C.CDLL(ORACLE_SO)
        L.or_grid_create.restype = C.c_void_p
        L.or_grid_create.argtypes = [C.c_int, C.c_int, C.c_double]
        L.or_grid_destroy.argtypes = [C.c_void_p]
        L.or_grid_set_preconditioner.argtypes = [C.c_void_p, C.c_int]
        L.or_grid_set_solid.argtypes = [C.c_void_p, _u8p]
        L.or_grid_set_air.argtypes = [C.c_void_p, _u8p]
        L.or_air_mask.argtypes = [C.c_int, _dp, _u8p, _u8p]
        L.or_grid_upload.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp]
        L.or_grid_download.argtypes = [C.c_void_p, _dp, _dp, _dp]
        L.or_grid_apply_gravity.argtypes = [C.c_void_p, C.c_double, C.c_double]
        L.or_grid_project.restype = _OrResult
        L.or_grid_project.argtypes = [C.c_void_p, C.c_double, C.c_int, C.c_double, C.c_double]
        L.or_grid_max_divergence.restype = C.c_double
        L.or_grid_max_divergence.argtypes = [C.c_void_p]
        L.or_coefficients.argtypes = [C.c_int, C.c_int, _dp, _dp, _dp, _dp]
        L.or_operator.restype = C.c_double
        L.or_operator.argtypes = [C.c_int, C.c_int, _dp, _dp, _dp, _dp]
        L.or_rhs.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, _dp, _dp, _dp]
        L.or_classify.argtypes = [C.c_int, _dp, _u8p, _u8p]
        L.or_face_flags.argtypes = [C.c_int, C.c_int, _u8p, _dp, _dp]
        L.or_mg_create.restype = C.c_void_p
        L.or_mg_create.argtypes = [C.c_int, C.c_int]
        L.or_mg_destroy.argtypes = [C.c_void_p]
        L.or_mg_levels.restype = C.c_int
        L.or_mg_levels.argtypes = [C.c_void_p]
        L.or_mg_rebuild.restype = C.c_int
        L.or_mg_rebuild.argtypes = [C.c_void_p, _dp, _dp]
        L.or_mg_apply.argtypes = [C.c_void_p, _dp, _dp, C.c_double]
        L.or_mg_set_sweeps.argtypes = [C.c_void_p, C.c_int, C.c_int]
        L.or_grid_set_sweeps.argtypes = [C.c_void_p, C.c_int, C.c_int]
        L.or_sample_scalar.restype = C.c_double
        L.or_sample_scalar.argtypes = [_dp, C.c_int, C.c_int, C.c_double, C.c_double]
        L.or_sample_velocity.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, _dp, _dp, C.c_int,
                                         _dp, _dp]
        L.or_visc_create.restype = C.c_void_p
        L.or_visc_create.argtypes = [C.c_int, C.c_int]
        L.or_visc_destroy.argtypes = [C.c_void_p]
        L.or_visc_levels.restype = C.c_int
        L.or_visc_levels.argtypes = [C.c_void_p]
        L.or_visc_setup.argtypes = [C.c_void_p, _dp, C.c_double, C.c_double]
        L.or_visc_apply.argtypes = [C.c_void_p, C.c_int, C.c_double, _dp, _dp]
        L.or_visc_precondition.argtypes = [C.c_void_p, _dp, _dp]
        L.or_visc_solve.restype = C.c_int
        L.or_visc_solve.argtypes = [C.c_void_p, _dp, _dp, _dp, C.c_double, C.c_double, C.c_double, C.c_int, _dp]
        L.or_visc_material.argtypes = [C.c_int, C.c_int, C.POINTER(_dp), _dp, _dp, C.c_double, _dp]
        L.or_advect.argtypes = [C.c_int, C.c_int, C.c_double, _dp, _dp, C.c_int, C.POINTER(_dp), C.POINTER(_dp),
                                _dp, _dp]
        _lib = L
    return _lib


def reference_available() -> bool:
    return os.path.exists(REF_SO)


def ref():
    global _ref
    if _ref is None:
        if not os.path.exists(REF_SO):
            raise FileNotFoundError("reference engine not built: " + REF_SO)
        L = C.CDLL(REF_SO)
        L.ref_create.restype = C.c_void_p
        L.ref_create.argtypes = [C.c_int, C.c_int, C.c_double]
        L.ref_destroy.argtypes = [C.c_void_p]
        L.ref_set_threads.argtypes = [C.c_int]
        L.ref_configure.argtypes = [C.c_void_p, C.c_double, C.c_double]
        L.ref_set_gravity.argtypes = [C.c_void_p, C.c_double]
        L.ref_set_preconditioner.argtypes = [C.c_void_p, C.c_int]
        L.ref_upload.restype = C.c_int
        L.ref_upload.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp, _dp, _dp]
        L.ref_download.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp]
        L.ref_project.restype = _RefResult
        L.ref_project.argtypes = [C.c_void_p, C.c_double, C.c_int, C.c_double]
        L.ref_set_origin.argtypes = [C.c_void_p, C.c_double, C.c_double]
        L.ref_advect.argtypes = [C.c_void_p, C.c_double]
        L.ref_masses.argtypes = [C.c_void_p, _dp, _dp]
        L.ref_set_surface_tension.argtypes = [C.c_void_p, C.c_double]
        L.ref_capillary_step_limit.restype = C.c_double
        L.ref_capillary_step_limit.argtypes = [C.c_void_p]
        L.ref_apply_surface_tension.argtypes = [C.c_void_p, C.c_double]
        L.ref_surface_curvature.argtypes = [C.c_int, C.c_int, C.c_double, _dp, _dp, _u8p]
        L.ref_sample_velocity.argtypes = [C.c_void_p, C.c_int, _dp, _dp]
        L.ref_step.restype = _RefResult
        L.ref_step.argtypes = [C.c_void_p, C.c_double, C.c_int, C.c_double]
        L.ref_apply_gravity.argtypes = [C.c_void_p, C.c_double]
        L.ref_max_divergence.restype = C.c_double
        L.ref_max_divergence.argtypes = [C.c_void_p]
        L.ref_coefficients.argtypes = [C.c_void_p, _dp, _dp, _dp]
        L.ref_mg_apply.restype = C.c_int
        L.ref_mg_apply.argtypes = [C.c_int, C.c_int, _dp, _dp, _dp, C.c_double, _dp]
        _ref = L
    return _ref


# --------------------------------------------------------------------------------------------
# Restatement
# --------------------------------------------------------------------------------------------

def coefficients(density):
    """Face weights (inv_u, inv_v, inv_diagonal) of a h x w density field."""
    density = _f64(density)
    h, w = density.shape
    inv_u = np.zeros((h, w + 1))
    inv_v = np.zeros((h + 1, w))
    inv_d = np.zeros((h, w))
    lib().or_coefficients(w, h, _ptr(density), _ptr(inv_u), _ptr(inv_v), _ptr(inv_d))
    return inv_u, inv_v, inv_d


def apply_operator(inv_u, inv_v, x):
    inv_u, inv_v, x = _f64(inv_u), _f64(inv_v), _f64(x)
    h, w = x.shape
    y = np.zeros_like(x)
    dot = lib().or_operator(w, h, _ptr(inv_u), _ptr(inv_v), _ptr(x), _ptr(y))
    return y, dot


def classify(fraction, solid=None):
    f = _f64(fraction)
    mask = np.zeros(f.shape, dtype=np.uint8)
    s = None if solid is None else np.ascontiguousarray(solid, dtype=np.uint8)
    lib().or_classify(f.size, _ptr(f), None if s is None else s.ctypes.data_as(_u8p), mask.ctypes.data_as(_u8p))
    return mask


def air_mask(fraction, solid=None):
    """Dirichlet air cells: neither solid nor liquid phase (f > 0.5)."""
    f = _f64(fraction)
    air = np.zeros(f.shape, dtype=np.uint8)
    s = None if solid is None else np.ascontiguousarray(solid, dtype=np.uint8)
    lib().or_air_mask(f.size, _ptr(f), None if s is None else s.ctypes.data_as(_u8p), air.ctypes.data_as(_u8p))
    return air


def close_solid_faces(inv_u, inv_v, solid):
    """Zero the face weights around solid cells (in place)."""
    s = np.ascontiguousarray(solid, dtype=np.uint8)
    h, w = s.shape
    lib().or_face_flags(w, h, s.ctypes.data_as(_u8p), _ptr(inv_u), _ptr(inv_v))


class Multigrid:
    """PressureMultigrid restated: rebuild from face weights, apply one V-cycle."""

    def __init__(self, width, height):
        self.w, self.h = width, height
        self.handle = lib().or_mg_create(width, height)

    def __del__(self):
        if getattr(self, "handle", None):
            lib().or_mg_destroy(self.handle)
            self.handle = None

    @property
    def levels(self):
        return lib().or_mg_levels(self.handle)

    def rebuild(self, inv_u, inv_v) -> bool:
        self._u, self._v = _f64(inv_u), _f64(inv_v)
        return bool(lib().or_mg_rebuild(self.handle, _ptr(self._u), _ptr(self._v)))

    def apply(self, residual, residual_mean=0.0):
        r = _f64(residual)
        z = np.zeros((self.h, self.w))
        lib().or_mg_apply(self.handle, _ptr(r), _ptr(z), float(residual_mean))
        return z


class OracleGrid:
    """FP64 restatement of FluidGridCPU's projection for one grid."""

    def __init__(self, width, height, cell_size):
        self.w, self.h, self.dx = width, height, cell_size
        self.handle = lib().or_grid_create(width, height, cell_size)

    def __del__(self):
        if getattr(self, "handle", None):
            lib().or_grid_destroy(self.handle)
            self.handle = None

    def set_preconditioner(self, multigrid: bool):
        lib().or_grid_set_preconditioner(self.handle, 1 if multigrid else 0)

    def set_sweeps(self, pre: int, post: int):
        lib().or_grid_set_sweeps(self.handle, pre, post)

    def upload(self, density, u, v, pressure=None, solid=None, air=None):
        """`air`: a mask of Dirichlet air cells (p = 0), or None for the reference's gas model."""
        lib().or_grid_upload(self.handle, _ptr(_f64(density)), _ptr(_f64(u)), _ptr(_f64(v)), _ptr(_f64(pressure)))
        if solid is not None:
            s = np.ascontiguousarray(solid, dtype=np.uint8)
            lib().or_grid_set_solid(self.handle, s.ctypes.data_as(_u8p))
        self._air = None if air is None else np.ascontiguousarray(air, dtype=np.uint8)
        lib().or_grid_set_air(self.handle, None if self._air is None else self._air.ctypes.data_as(_u8p))

    def download(self):
        u = np.zeros((self.h, self.w + 1))
        v = np.zeros((self.h + 1, self.w))
        p = np.zeros((self.h, self.w))
        lib().or_grid_download(self.handle, _ptr(u), _ptr(v), _ptr(p))
        return u, v, p

    def apply_gravity(self, gravity, dt):
        lib().or_grid_apply_gravity(self.handle, gravity, dt)

    def project(self, dt, max_iterations=200, tolerance=1e-6, relative_tolerance=0.0):
        r = lib().or_grid_project(self.handle, dt, max_iterations, tolerance, relative_tolerance)
        return ProjectionResult(r.iterations, bool(r.converged), r.max_divergence, r.residual_max,
                                r.residual_l2, r.rhs_l2)

    def max_divergence(self):
        return lib().or_grid_max_divergence(self.handle)


# --------------------------------------------------------------------------------------------
# Reference engine
# --------------------------------------------------------------------------------------------

class ReferenceGrid:
    """The reference FluidGridCPU (two components: one liquid, one gas)."""

    def __init__(self, width, height, cell_size, liquid_density=100.0, gas_density=0.1):
        self.w, self.h, self.dx = width, height, cell_size
        self.handle = ref().ref_create(width, height, cell_size)
        ref().ref_configure(self.handle, liquid_density, gas_density)

    def __del__(self):
        if getattr(self, "handle", None):
            ref().ref_destroy(self.handle)
            self.handle = None

    def set_preconditioner(self, multigrid: bool):
        ref().ref_set_preconditioner(self.handle, 1 if multigrid else 0)

    def set_gravity(self, g):
        ref().ref_set_gravity(self.handle, g)

    def upload(self, fraction=None, u=None, v=None, pressure=None, liquid_mass=None, gas_mass=None):
        rc = ref().ref_upload(self.handle, *(_ptr(_f64(a)) for a in (fraction, u, v, pressure, liquid_mass, gas_mass)))
        if rc != 0:
            raise ValueError("reference rejected the upload")

    def download(self):
        f = np.zeros((self.h, self.w))
        u = np.zeros((self.h, self.w + 1))
        v = np.zeros((self.h + 1, self.w))
        p = np.zeros((self.h, self.w))
        ref().ref_download(self.handle, _ptr(f), _ptr(u), _ptr(v), _ptr(p))
        return f, u, v, p

    def coefficients(self):
        inv_u = np.zeros((self.h, self.w + 1))
        inv_v = np.zeros((self.h + 1, self.w))
        inv_d = np.zeros((self.h, self.w))
        ref().ref_coefficients(self.handle, _ptr(inv_u), _ptr(inv_v), _ptr(inv_d))
        return inv_u, inv_v, inv_d

    def project(self, dt, max_iterations=200, tolerance=1e-6):
        r = ref().ref_project(self.handle, dt, max_iterations, tolerance)
        return ProjectionResult(r.iterations, bool(r.converged), r.max_divergence, elapsed_ms=r.elapsed_ms)

    def step(self, dt, max_iterations=200, tolerance=1e-6):
        r = ref().ref_step(self.handle, dt, max_iterations, tolerance)
        return ProjectionResult(r.iterations, bool(r.converged), r.max_divergence, elapsed_ms=r.elapsed_ms)

    def apply_gravity(self, dt):
        ref().ref_apply_gravity(self.handle, dt)

    def max_divergence(self):
        return ref().ref_max_divergence(self.handle)

    def advect(self, dt):
        """FluidGridCPU::advect (the reference's own PLIC transport)."""
        ref().ref_advect(self.handle, float(dt))

    def masses(self):
        lm = np.zeros((self.h, self.w))
        gm = np.zeros((self.h, self.w))
        ref().ref_masses(self.handle, _ptr(lm), _ptr(gm))
        return lm, gm

    def set_surface_tension(self, sigma):
        ref().ref_set_surface_tension(self.handle, float(sigma))

    def capillary_step_limit(self):
        return ref().ref_capillary_step_limit(self.handle)

    def apply_surface_tension(self, dt):
        """FluidGridCPU::applySurfaceTension (the reference's own code)."""
        ref().ref_apply_surface_tension(self.handle, float(dt))

    def set_origin(self, x, y):
        ref().ref_set_origin(self.handle, x, y)

    def sample_velocity(self, positions):
        pos = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1, 2)
        out = np.empty_like(pos)
        ref().ref_sample_velocity(self.handle, pos.shape[0], _ptr(pos), _ptr(out))
        return out


def reference_surface_curvature(fraction, cell_size):
    """FluidSurfaceTensionCPU (the reference's own header) on a fraction field: completed
    curvature per cell and its validity."""
    f = _f64(fraction)
    h, w = f.shape
    k = np.zeros((h, w))
    ok = np.zeros((h, w), dtype=np.uint8)
    ref().ref_surface_curvature(w, h, float(cell_size), _ptr(f), _ptr(k), ok.ctypes.data_as(_u8p))
    return k, ok.astype(bool)


def sample_scalar(data, x, y):
    """FluidGridCPU.cpp:67-90 on a row-major (h, w) array at fractional index (x, y)."""
    d = _f64(data)
    h, w = d.shape
    return lib().or_sample_scalar(_ptr(d), w, h, float(x), float(y))


def sample_velocity(u, v, cell_size, positions, origin=(0.0, 0.0)):
    """FluidGridCPU::sampleVelocity (FluidGridCPU.cpp:465-471) at (n, 2) world positions."""
    u, v = _f64(u), _f64(v)
    h, w1 = u.shape
    pos = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1, 2)
    out = np.empty_like(pos)
    lib().or_sample_velocity(w1 - 1, h, float(cell_size), float(origin[0]), float(origin[1]), _ptr(u), _ptr(v),
                             pos.shape[0], _ptr(pos), _ptr(out))
    return out


def advect(u, v, fields, dt, cell_size, storage=np.float64):
    """Semi-Lagrangian transport of face velocities and cell fields (restatement of the
    UniformCUDA transport). ``storage`` is the device's velocity storage type: velocities are
    rounded to it before tracing and after, as the FP32 engine holds them."""
    u = np.asarray(u, dtype=np.float64).astype(storage).astype(np.float64)
    v = np.asarray(v, dtype=np.float64).astype(storage).astype(np.float64)
    u, v = np.ascontiguousarray(u), np.ascontiguousarray(v)
    h, w1 = u.shape
    w = w1 - 1
    ins = [_f64(f) for f in fields]
    outs = [np.zeros((h, w)) for _ in ins]
    u_out, v_out = np.zeros_like(u), np.zeros_like(v)
    in_ptrs = (_dp * max(1, len(ins)))(*[_ptr(a) for a in ins])
    out_ptrs = (_dp * max(1, len(outs)))(*[_ptr(a) for a in outs])
    lib().or_advect(w, h, float(dt) / float(cell_size), _ptr(u), _ptr(v), len(ins), in_ptrs, out_ptrs, _ptr(u_out),
                    _ptr(v_out))
    return u_out.astype(storage).astype(np.float64), v_out.astype(storage).astype(np.float64), outs


class Viscosity:
    """The FP64 restatement of the reference's implicit viscosity solve
    (UniformWebGPU/ViscositySolverGPU.cpp). Node fields are (h+1, w+1, 2) arrays: [..., 0] is u
    face (x, y), [..., 1] is v face (x, y)."""

    def __init__(self, width, height):
        self.w, self.h = width, height
        self.handle = lib().or_visc_create(width, height)

    def __del__(self):
        if getattr(self, "handle", None):
            lib().or_visc_destroy(self.handle)
            self.handle = None

    @property
    def levels(self):
        return lib().or_visc_levels(self.handle)

    def setup(self, material, dt, cell_size):
        m = _f64(material)
        lib().or_visc_setup(self.handle, _ptr(m), float(dt), float(cell_size))

    def apply(self, field, dt, level=0):
        f = _f64(field)
        out = np.zeros_like(f)
        lib().or_visc_apply(self.handle, level, float(dt), _ptr(f), _ptr(out))
        return out

    def precondition(self, residual):
        r = _f64(residual)
        z = np.zeros_like(r)
        lib().or_visc_precondition(self.handle, _ptr(r), _ptr(z))
        return z

    def solve(self, u, v, material, dt, cell_size, tolerance=1e-4, max_iterations=-1):
        """Returns (iterations, u, v, relative_residual); iterations -1 = breakdown or
        non-finite state, -2 = the iteration cap was reached."""
        u, v, m = _f64(u).copy(), _f64(v).copy(), _f64(material)
        rel = C.c_double()
        it = lib().or_visc_solve(self.handle, _ptr(u), _ptr(v), _ptr(m), float(dt), float(cell_size),
                                 float(tolerance), int(max_iterations), C.byref(rel))
        return it, u, v, rel.value


def viscosity_material(masses, densities, viscosities, cell_size):
    """Cell density and volume-weighted viscosity (FluidGridGPU.cpp:172-217), (h, w, 2)."""
    ms = [_f64(m) for m in masses]
    h, w = ms[0].shape
    out = np.zeros((h, w, 2))
    table = (_dp * len(ms))(*[_ptr(m) for m in ms])
    d, mu = _f64(np.asarray(densities, dtype=float)), _f64(np.asarray(viscosities, dtype=float))
    lib().or_visc_material(w * h, len(ms), table, _ptr(d), _ptr(mu), float(cell_size), _ptr(out))
    return out


def reference_mg_apply(inv_u, inv_v, residual, residual_mean=0.0):
    inv_u, inv_v, r = _f64(inv_u), _f64(inv_v), _f64(residual)
    h, w = r.shape
    z = np.zeros((h, w))
    rc = ref().ref_mg_apply(w, h, _ptr(inv_u), _ptr(inv_v), _ptr(r), float(residual_mean), _ptr(z))
    if rc != 0:
        raise RuntimeError("reference multigrid breakdown")
    return z


def set_reference_threads(n: int):
    ref().ref_set_threads(int(n))
