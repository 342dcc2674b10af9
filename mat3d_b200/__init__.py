"""mat3d_b200 -- B200-native FFT homogenization (Lippmann-Schwinger) solver.

Python host layer over the C ABI of ``libmat3d_b200.so`` (include/mat3d_b200.h).
It mirrors the reference's two solver classes (FayyazNo/MAT3d
include/FFT_analysis3D.hpp:36-215 and include/FFT_thermal3D.hpp:37-154):
same class names, method names, argument meaning and public result fields,
with numpy arrays in place of Eigen matrices (``epsilon``/``sigma`` are
``(6, N^3)`` arrays laid out like the reference's column-major 6 x N^3
matrices, i.e. voxel-major in memory).

There is no CPU fallback: the solve always runs on the GPU, and importing the
library raises if the compiled extension is missing.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

__all__ = [
    "Solver", "FFT_Analysis3D", "FFT_analysis3d_thermal", "load_library", "M3DError",
    "KIND_MECH", "KIND_THERMAL", "ELASTIC", "J2", "DAMAGE", "FP64", "FP32", "FP32_REFINE",
    "CRIT_REFERENCE", "CRIT_RESIDUAL",
]

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmat3d_b200.so")

KIND_MECH, KIND_THERMAL = 1, 2
ELASTIC, J2, DAMAGE = 0, 1, 2
FP64, FP32, FP32_REFINE = 0, 1, 2
CRIT_REFERENCE, CRIT_RESIDUAL = 0, 1
SCHEME_AUTO, SCHEME_PRIMAL, SCHEME_DUAL = 0, 1, 2
FIELD_STRAIN, FIELD_STRESS, FIELD_EPS_P, FIELD_DAMAGE = 0, 1, 2, 3
OK, NOT_CONVERGED, PENDING = 0, 4, 9

_PRECISIONS = {"fp64": FP64, "fp32": FP32, "fp32_refine": FP32_REFINE, FP64: FP64, FP32: FP32, FP32_REFINE: FP32_REFINE}
_BEHAV = {"e": ELASTIC, "ep": J2, "ed": DAMAGE}


class M3DError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{msg} (status {status})")
        self.status = status


class Stats(ctypes.Structure):
    _fields_ = [
        ("sweeps", ctypes.c_longlong), ("sweeps_fp64", ctypes.c_longlong), ("sweeps_fp32", ctypes.c_longlong),
        ("iters", ctypes.c_int), ("scheme", ctypes.c_int), ("status", ctypes.c_int), ("n_increments", ctypes.c_int),
        ("residual", ctypes.c_double), ("eqvar", ctypes.c_double), ("diff_sum", ctypes.c_double),
        ("diff_eq", ctypes.c_double), ("solve_ms", ctypes.c_double), ("la0", ctypes.c_double),
        ("mu0", ctypes.c_double), ("k0", ctypes.c_double), ("vol_fraction", ctypes.c_double * 16),
        ("kernel_launches", ctypes.c_longlong), ("passes_per_sweep", ctypes.c_int),
    ]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_ if k != "vol_fraction"}
        d["vol_fraction"] = list(self.vol_fraction)
        return d


class BatchStats(ctypes.Structure):
    _fields_ = [("sweeps", ctypes.c_longlong), ("sweeps_fp64", ctypes.c_longlong),
                ("sweeps_fp32", ctypes.c_longlong), ("voxel_iters", ctypes.c_longlong),
                ("device_ms", ctypes.c_double), ("wall_ms", ctypes.c_double), ("rves", ctypes.c_int),
                ("groups", ctypes.c_int), ("launches", ctypes.c_int), ("kernel_launches", ctypes.c_longlong),
                ("autotuned", ctypes.c_int), ("concurrent", ctypes.c_int)]


class Tune(ctypes.Structure):
    _fields_ = [("fast", ctypes.c_int), ("tma_y", ctypes.c_int), ("G", ctypes.c_int), ("tzy", ctypes.c_int),
                ("tzx", ctypes.c_int), ("sweep_us", ctypes.c_double), ("candidates", ctypes.c_int),
                ("slab", ctypes.c_int), ("schedule", ctypes.c_int)]


class Request(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("behav", ctypes.c_int), ("Nx", ctypes.c_int), ("Ny", ctypes.c_int),
                ("Nz", ctypes.c_int), ("precision", ctypes.c_int), ("mat", ctypes.c_void_p), ("nph", ctypes.c_int),
                ("km", ctypes.c_double), ("ki", ctypes.c_double), ("phase", ctypes.c_void_p),
                ("scheme", ctypes.c_int), ("E", ctypes.c_void_p), ("X0", ctypes.c_void_p), ("nInc", ctypes.c_int),
                ("tol", ctypes.c_double), ("max_iter", ctypes.c_int), ("keep_field", ctypes.c_int)]


class Result(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("iters", ctypes.c_int), ("sweeps", ctypes.c_longlong),
                ("residual", ctypes.c_double), ("strain_mean", ctypes.c_double * 6),
                ("stress_mean", ctypes.c_double * 6), ("queue_ms", ctypes.c_double),
                ("solve_ms", ctypes.c_double), ("latency_ms", ctypes.c_double)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_}
        d["strain_mean"] = np.array(self.strain_mean[:])
        d["stress_mean"] = np.array(self.stress_mean[:])
        return d


class ServeStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_longlong), ("completed", ctypes.c_longlong), ("failed", ctypes.c_longlong),
                ("queued", ctypes.c_int), ("running", ctypes.c_int), ("peak_running", ctypes.c_int),
                ("resident_solvers", ctypes.c_int), ("resident_bytes", ctypes.c_double),
                ("budget_bytes", ctypes.c_double), ("merged_solves", ctypes.c_longlong),
                ("merged_requests", ctypes.c_longlong)]


class Profile(ctypes.Structure):
    _fields_ = [("ms_fp64", ctypes.c_double), ("n_fp64", ctypes.c_longlong),
                ("ms_fp32", ctypes.c_double), ("n_fp32", ctypes.c_longlong),
                ("pass_ms_fp64", ctypes.c_double * 5), ("pass_ms_fp32", ctypes.c_double * 5)]


_lib = None

# every symbol the C ABI header declares
EXPORTS = [
    "m3d_create", "m3d_destroy", "m3d_set_material_mech", "m3d_set_material_thermal", "m3d_set_load", "m3d_run",
    "m3d_homogenize", "m3d_get_field", "m3d_get_field_async", "m3d_wait_field", "m3d_get_means", "m3d_get_stats", "m3d_get_increments",
    "m3d_status_string", "m3d_last_error", "m3d_abi_version", "m3d_get_stream", "m3d_set_stream",
    "m3d_set_profiling", "m3d_get_profile", "m3d_thermal_solve_noalloc", "m3d_get_entry_stats",
    "m3d_create_multi", "m3d_set_material_mech_rve", "m3d_set_material_thermal_rve", "m3d_footprint_bytes",
    "m3d_batch_create", "m3d_batch_add_mech", "m3d_batch_add_thermal", "m3d_batch_homogenize",
    "m3d_batch_get_stats", "m3d_batch_clear", "m3d_batch_destroy",
    "m3d_autotune", "m3d_batch_set_autotune",
    "m3d2d_create", "m3d2d_destroy", "m3d2d_material", "m3d2d_set_load", "m3d2d_run", "m3d2d_homogenize",
    "m3d2d_get_fields", "m3d2d_kernel_launches", "m3d2d_get_stream",
    "m3d_serve_create", "m3d_serve_submit", "m3d_serve_poll", "m3d_serve_wait", "m3d_serve_get_field",
    "m3d_serve_get_stats", "m3d_serve_destroy",
    "m3drec_create", "m3drec_destroy", "m3drec_seed", "m3drec_run", "m3drec_iterate", "m3drec_threshold",
    "m3drec_set_state", "m3drec_get_state", "m3drec_get_field", "m3drec_get_error", "m3drec_set_profiling",
    "m3drec_profile", "m3drec_kernel_launches", "m3drec_get_stream", "m3drec_fftshift", "m3drec_ifftshift",
    "m3drec_create_from_sections", "m3drec_estimate_norm", "m3drec_get_norm", "m3drec_save_images",
    "m3drec_write_vti", "m3drec_fft3",
]


def load_library(path: str | None = None):
    """Load libmat3d_b200.so (built in-tree by ``python -m mat3d_b200.build``).
    With ``path``, load that build instead and use it for every object created
    afterwards."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise ImportError(f"{p} is missing: build it with `python -m mat3d_b200.build` (no CPU fallback exists)")
    L = ctypes.CDLL(p)
    vp, i, d, dp = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.POINTER(ctypes.c_double)
    L.m3d_create.argtypes = [i, i, i, i, i, i, i, ctypes.POINTER(vp)]
    L.m3d_destroy.argtypes = [vp]
    L.m3d_set_material_mech.argtypes = [vp, vp, i, vp, i]
    L.m3d_set_material_thermal.argtypes = [vp, d, d, vp, i]
    L.m3d_set_load.argtypes = [vp, i, vp, vp]
    L.m3d_run.argtypes = [vp, d, d, i, i, i]
    L.m3d_homogenize.argtypes = [vp, d, d, i, i, vp, vp, vp, vp]
    L.m3d_get_field.argtypes = [vp, i, i, vp]
    L.m3d_get_field_async.argtypes = [vp, i, i, vp]
    L.m3d_wait_field.argtypes = [vp]
    L.m3d_get_means.argtypes = [vp, i, vp, vp]
    L.m3d_get_stats.argtypes = [vp, ctypes.POINTER(Stats)]
    L.m3d_get_increments.argtypes = [vp, vp, i]
    L.m3d_get_entry_stats.argtypes = [vp, i, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_longlong),
                                      ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)]
    L.m3d_status_string.restype = ctypes.c_char_p
    L.m3d_status_string.argtypes = [i]
    L.m3d_last_error.restype = ctypes.c_char_p
    L.m3d_abi_version.restype = i
    for name in EXPORTS:
        if name not in ("m3d_status_string", "m3d_last_error", "m3d_get_stream", "m3d_footprint_bytes",
                        "m3d2d_kernel_launches", "m3d2d_get_stream", "m3drec_kernel_launches",
                        "m3drec_get_stream"):
            getattr(L, name).restype = ctypes.c_int
    L.m3d_get_stream.restype = vp
    L.m3d_get_stream.argtypes = [vp]
    L.m3d_set_stream.argtypes = [vp, vp]
    L.m3d_thermal_solve_noalloc.argtypes = [i, i, i, d, d, vp, vp, d, i, vp, ctypes.POINTER(ctypes.c_int),
                                            ctypes.POINTER(ctypes.c_double), vp]
    L.m3d_create_multi.argtypes = [i, i, i, i, i, i, i, ctypes.POINTER(vp)]
    L.m3d_set_material_mech_rve.argtypes = [vp, i, vp, i, vp, i]
    L.m3d_set_material_thermal_rve.argtypes = [vp, i, d, d, vp, i]
    L.m3d_footprint_bytes.argtypes = [i, i, i, i, i, i, i, i]
    L.m3d_footprint_bytes.restype = ctypes.c_longlong
    L.m3d_batch_create.argtypes = [i, i, d, ctypes.POINTER(vp)]
    L.m3d_batch_add_mech.argtypes = [vp, i, i, i, vp, i, vp, i, ctypes.POINTER(ctypes.c_int)]
    L.m3d_batch_add_thermal.argtypes = [vp, i, i, i, d, d, vp, i, ctypes.POINTER(ctypes.c_int)]
    L.m3d_batch_homogenize.argtypes = [vp, d, i, vp, vp]
    L.m3d_batch_get_stats.argtypes = [vp, ctypes.POINTER(BatchStats)]
    L.m3d_batch_clear.argtypes = [vp]
    L.m3d_batch_destroy.argtypes = [vp]
    L.m3d2d_create.argtypes = [i, i, ctypes.POINTER(vp)]
    L.m3d2d_destroy.argtypes = [vp]
    L.m3d2d_material.argtypes = [vp, vp, vp]
    L.m3d2d_set_load.argtypes = [vp, vp]
    L.m3d2d_run.argtypes = [vp, i]
    L.m3d2d_homogenize.argtypes = [vp, i, vp, vp, vp]
    L.m3d2d_get_fields.argtypes = [vp, vp, vp]
    L.m3d2d_kernel_launches.argtypes = [vp]
    L.m3d2d_kernel_launches.restype = ctypes.c_longlong
    L.m3d2d_get_stream.argtypes = [vp]
    L.m3d2d_get_stream.restype = vp
    L.m3d_autotune.argtypes = [vp, i, ctypes.POINTER(Tune)]
    L.m3d_batch_set_autotune.argtypes = [vp, i]
    L.m3d_serve_create.argtypes = [d, i, ctypes.POINTER(vp)]
    L.m3d_serve_submit.argtypes = [vp, ctypes.POINTER(Request), ctypes.POINTER(ctypes.c_longlong)]
    L.m3d_serve_poll.argtypes = [vp, ctypes.c_longlong, ctypes.POINTER(Result)]
    L.m3d_serve_wait.argtypes = [vp, ctypes.c_longlong, d, ctypes.POINTER(Result)]
    L.m3d_serve_get_field.argtypes = [vp, ctypes.c_longlong, vp]
    L.m3d_serve_get_stats.argtypes = [vp, ctypes.POINTER(ServeStats)]
    L.m3d_serve_destroy.argtypes = [vp]
    L.m3d_set_profiling.argtypes = [vp, i]
    L.m3d_get_profile.argtypes = [vp, ctypes.POINTER(Profile)]
    u64, ip = ctypes.c_ulonglong, ctypes.POINTER(ctypes.c_int)
    L.m3drec_create.argtypes = [i, i, i, vp, i, ctypes.POINTER(vp)]
    L.m3drec_destroy.argtypes = [vp]
    L.m3drec_seed.argtypes = [vp, u64]
    L.m3drec_run.argtypes = [vp, i, d]
    L.m3drec_iterate.argtypes = [vp, i, d]
    L.m3drec_threshold.argtypes = [vp]
    L.m3drec_set_state.argtypes = [vp, vp, i, i, u64]
    L.m3drec_get_state.argtypes = [vp, vp, ip, ip, ctypes.POINTER(u64)]
    L.m3drec_get_field.argtypes = [vp, vp]
    L.m3drec_get_error.argtypes = [vp, vp, i, ip]
    L.m3drec_set_profiling.argtypes = [vp, i]
    L.m3drec_profile.argtypes = [vp, vp, ctypes.POINTER(ctypes.c_longlong)]
    L.m3drec_kernel_launches.argtypes = [vp]
    L.m3drec_kernel_launches.restype = ctypes.c_longlong
    L.m3drec_get_stream.argtypes = [vp]
    L.m3drec_get_stream.restype = vp
    L.m3drec_fftshift.argtypes = [vp, vp, i, i, i]
    L.m3drec_ifftshift.argtypes = [vp, vp, i, i, i]
    L.m3drec_create_from_sections.argtypes = [vp, i, i, vp, i, i, i, ctypes.POINTER(vp)]
    L.m3drec_estimate_norm.argtypes = [vp]
    L.m3drec_get_norm.argtypes = [vp, vp]
    L.m3drec_save_images.argtypes = [vp, ctypes.c_char_p]
    L.m3drec_write_vti.argtypes = [vp, ctypes.c_char_p, vp]
    L.m3drec_fft3.argtypes = [vp, vp, i, i, i, i, i]
    _lib = L
    return L


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def _check(L, rc, what, allow_not_converged=True):
    if rc == OK or (allow_not_converged and rc == NOT_CONVERGED):
        return rc
    raise M3DError(rc, f"{what}: {L.m3d_status_string(rc).decode()}: {L.m3d_last_error().decode()}")


class Solver:
    """Thin handle over the C ABI (one CUDA stream, `batch` solves at once)."""

    def __init__(self, kind, Nx, Ny, Nz, behav=ELASTIC, precision=FP64, batch=1, nrve=None, nload=None):
        self.L = load_library()
        self.kind, self.shape = kind, (Nx, Ny, Nz)
        self.V = Nx * Ny * Nz
        self.C = 6 if kind == KIND_MECH else 3
        self.behav = behav
        h = ctypes.c_void_p()
        if nrve is None:
            self.nrve, self.batch = 1, batch
            rc = self.L.m3d_create(kind, Nx, Ny, Nz, behav, _PRECISIONS[precision], batch, ctypes.byref(h))
        else:
            # many RVEs of one grid size, nload load cases each (linear solves only)
            nload = self.C if nload is None else nload
            self.nrve, self.batch = nrve, nrve * nload
            rc = self.L.m3d_create_multi(kind, Nx, Ny, Nz, _PRECISIONS[precision], nrve, nload, ctypes.byref(h))
        _check(self.L, rc, "m3d_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.L.m3d_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_material_mech(self, mat, phase, scheme=SCHEME_AUTO, rve=0):
        mat = np.ascontiguousarray(mat, np.float64)
        ph = np.ascontiguousarray(np.asarray(phase).ravel(), np.int32)
        _check(self.L, self.L.m3d_set_material_mech_rve(self.h, rve, _ptr(mat), mat.shape[0], _ptr(ph), scheme),
               "material")

    def set_material_thermal(self, km, ki, phase, scheme=SCHEME_AUTO, rve=0):
        ph = np.ascontiguousarray(np.asarray(phase).ravel(), np.int32)
        _check(self.L, self.L.m3d_set_material_thermal_rve(self.h, rve, float(km), float(ki), _ptr(ph), scheme),
               "material")

    def set_load(self, E, X0=None, b=-1):
        E = np.ascontiguousarray(E, np.float64)
        X = None if X0 is None else np.ascontiguousarray(X0, np.float64)
        _check(self.L, self.L.m3d_set_load(self.h, b, _ptr(E), _ptr(X)), "setLoad")

    def run(self, tol_field, tol_eq=0.0, nInc=1, criterion=CRIT_RESIDUAL, max_iter=0):
        return _check(self.L, self.L.m3d_run(self.h, tol_field, tol_eq, nInc, criterion, max_iter), "run")

    def homogenize(self, tol_field, tol_eq=0.0, criterion=CRIT_RESIDUAL, max_iter=0):
        """Effective tensors; on a multi-RVE solver each array is (nrve, C, C)."""
        C = self.C
        Ce, Se, ep, sg = (np.zeros((self.nrve, C, C)) for _ in range(4))
        rc = _check(self.L, self.L.m3d_homogenize(self.h, tol_field, tol_eq, criterion, max_iter,
                                                  _ptr(Ce), _ptr(Se), _ptr(ep), _ptr(sg)), "homogenize")
        if self.nrve == 1:
            Ce, Se, ep, sg = Ce[0], Se[0], ep[0], sg[0]
        return Ce, Se, ep, sg, rc

    def field(self, which=FIELD_STRAIN, b=0, out=None):
        """The field as a (C, V) view of voxel-major (AoS) data, or (V,) for
        scalar fields.  ``out``: a caller-owned contiguous float64 buffer of
        V*C (or V) elements to write into (e.g. pinned host memory, so the
        device-to-host copy runs at full speed with no extra host copy)."""
        scalar = which in (FIELD_EPS_P, FIELD_DAMAGE)
        n = self.V if scalar else self.V * self.C
        if out is None:
            out = np.empty(n)
        elif out.dtype != np.float64 or out.size != n or not out.flags.c_contiguous:
            raise ValueError(f"out must be a contiguous float64 array of {n} elements")
        _check(self.L, self.L.m3d_get_field(self.h, which, b, _ptr(out)), "get_field")
        flat = out.reshape(-1)
        return flat if scalar else flat.reshape(self.V, self.C).T  # (C, V) view of AoS data

    def field_async(self, out, which=FIELD_STRAIN, b=0):
        """Enqueue the field's copy into ``out`` (a contiguous float64 array of
        V*C elements, page-locked for an asynchronous copy) and return at once;
        the copy overlaps the handle's next work.  ``out`` is complete after
        wait_field()."""
        n = self.V * self.C
        if out.dtype != np.float64 or out.size != n or not out.flags.c_contiguous:
            raise ValueError(f"out must be a contiguous float64 array of {n} elements")
        _check(self.L, self.L.m3d_get_field_async(self.h, which, b, _ptr(out)), "get_field_async")
        return out.reshape(-1).reshape(self.V, self.C).T

    def wait_field(self):
        _check(self.L, self.L.m3d_wait_field(self.h), "wait_field")

    def means(self, b=0):
        e = np.zeros(self.C)
        s = np.zeros(self.C)
        _check(self.L, self.L.m3d_get_means(self.h, b, _ptr(e), _ptr(s)), "get_means")
        return e, s

    def stats(self):
        st = Stats()
        _check(self.L, self.L.m3d_get_stats(self.h, ctypes.byref(st)), "get_stats")
        return st.as_dict()

    def entry_stats(self, b):
        """Batch entry b's own iterations, sweeps, residual and status of the last run."""
        it, sw, res, stt = ctypes.c_int(), ctypes.c_longlong(), ctypes.c_double(), ctypes.c_int()
        _check(self.L, self.L.m3d_get_entry_stats(self.h, b, ctypes.byref(it), ctypes.byref(sw), ctypes.byref(res),
                                                  ctypes.byref(stt)), "get_entry_stats")
        return {"iters": it.value, "sweeps": sw.value, "residual": res.value, "status": stt.value}

    def autotune(self, sweeps=3):
        """Time the launch schedules and keep the fastest (sweeps = 0: apply
        the schedule remembered for this shape)."""
        t = Tune()
        _check(self.L, self.L.m3d_autotune(self.h, sweeps, ctypes.byref(t)), "autotune")
        return {k: getattr(t, k) for k, _ in t._fields_}

    def set_profiling(self, enable=True):
        _check(self.L, self.L.m3d_set_profiling(self.h, 1 if enable else 0), "set_profiling")

    def profile(self):
        p = Profile()
        _check(self.L, self.L.m3d_get_profile(self.h, ctypes.byref(p)), "get_profile")
        d = {k: getattr(p, k) for k, _ in p._fields_}
        d["pass_ms_fp64"] = list(p.pass_ms_fp64)
        d["pass_ms_fp32"] = list(p.pass_ms_fp32)
        return d

    def stream_ptr(self):
        """cudaStream_t of the handle (for timing with events on the launching stream)."""
        return self.L.m3d_get_stream(self.h)

    def increments(self, max_rows=100000):
        st = self.stats()
        n = max(st["n_increments"], 0)
        out = np.zeros((max(n, 1), 9))
        rows = self.L.m3d_get_increments(self.h, _ptr(out), n)
        return out[:rows]


def footprint_bytes(kind, shape, behav=ELASTIC, precision=FP64, nrve=1, batch=1):
    """Device bytes a solver of this shape holds (admission by HBM footprint)."""
    L = load_library()
    return int(L.m3d_footprint_bytes(kind, *shape, behav, _PRECISIONS[precision], nrve, batch))


class Batch:
    """Many RVEs of mixed grid sizes homogenized together (m3d_batch_*)."""

    def __init__(self, kind, precision=FP32_REFINE, mem_budget_bytes=0.0):
        self.L = load_library()
        self.kind = kind
        self.C = 6 if kind == KIND_MECH else 3
        self.n = 0
        h = ctypes.c_void_p()
        _check(self.L, self.L.m3d_batch_create(kind, _PRECISIONS[precision], float(mem_budget_bytes),
                                               ctypes.byref(h)), "batch_create")
        self.h = h

    def add_mech(self, shape, mat, phase, scheme=SCHEME_AUTO):
        mat = np.ascontiguousarray(mat, np.float64)
        ph = np.ascontiguousarray(np.asarray(phase).ravel(), np.int32)
        idx = ctypes.c_int()
        _check(self.L, self.L.m3d_batch_add_mech(self.h, *shape, _ptr(mat), mat.shape[0], _ptr(ph), scheme,
                                                 ctypes.byref(idx)), "batch_add")
        self.n += 1
        return idx.value

    def add_thermal(self, shape, km, ki, phase, scheme=SCHEME_AUTO):
        ph = np.ascontiguousarray(np.asarray(phase).ravel(), np.int32)
        idx = ctypes.c_int()
        _check(self.L, self.L.m3d_batch_add_thermal(self.h, *shape, float(km), float(ki), _ptr(ph), scheme,
                                                    ctypes.byref(idx)), "batch_add")
        self.n += 1
        return idx.value

    def set_autotune(self, on=True):
        _check(self.L, self.L.m3d_batch_set_autotune(self.h, 1 if on else 0), "batch_set_autotune")

    def homogenize(self, tol_field, max_iter=0):
        C = self.C
        Ce = np.zeros((self.n, C, C))
        Se = np.zeros((self.n, C, C))
        rc = _check(self.L, self.L.m3d_batch_homogenize(self.h, tol_field, max_iter, _ptr(Ce), _ptr(Se)),
                    "batch_homogenize")
        return Ce, Se, rc

    def stats(self):
        st = BatchStats()
        _check(self.L, self.L.m3d_batch_get_stats(self.h, ctypes.byref(st)), "batch_stats")
        return {k: getattr(st, k) for k, _ in st._fields_}

    def clear(self):
        _check(self.L, self.L.m3d_batch_clear(self.h), "batch_clear")
        self.n = 0

    def close(self):
        if getattr(self, "h", None):
            self.L.m3d_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Solver2D:
    """The 2-D elastic solver (m3d2d_*): complex FP64 fields, basic scheme."""

    def __init__(self, Nx, Ny):
        self.L = load_library()
        self.Nx, self.Ny, self.xy = Nx, Ny, Nx * Ny
        h = ctypes.c_void_p()
        _check(self.L, self.L.m3d2d_create(Nx, Ny, ctypes.byref(h)), "m3d2d_create")
        self.h = h

    def material(self, props, phase):
        p = np.ascontiguousarray(props, np.float64)
        ph = np.ascontiguousarray(np.asarray(phase).ravel(), np.int32)
        _check(self.L, self.L.m3d2d_material(self.h, _ptr(p), _ptr(ph)), "material")

    def set_load(self, E):
        e = np.ascontiguousarray(np.asarray(E, np.complex128))
        _check(self.L, self.L.m3d2d_set_load(self.h, _ptr(e)), "setLoad")

    def run(self, iterations=25):
        _check(self.L, self.L.m3d2d_run(self.h, iterations), "runAnalysis")

    def homogenize(self, iterations=25):
        C, ep, sg = np.zeros((3, 3)), np.zeros((3, 3)), np.zeros((3, 3))
        _check(self.L, self.L.m3d2d_homogenize(self.h, iterations, _ptr(C), _ptr(ep), _ptr(sg)), "homogenization")
        return C, ep, sg

    def fields(self):
        """epsilon, sigma as (3, Nx*Ny) complex arrays."""
        e = np.zeros(3 * self.xy, np.complex128)
        s = np.zeros(3 * self.xy, np.complex128)
        _check(self.L, self.L.m3d2d_get_fields(self.h, _ptr(e), _ptr(s)), "get_fields")
        return e.reshape(self.xy, 3).T.copy(), s.reshape(self.xy, 3).T.copy()

    def kernel_launches(self):
        return int(self.L.m3d2d_kernel_launches(self.h))

    def stream_ptr(self):
        return self.L.m3d2d_get_stream(self.h)

    def close(self):
        if getattr(self, "h", None):
            self.L.m3d2d_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class FFT_Analysis2D:
    """Drop-in mirror of the reference's ``FFT_Analysis2D``
    (include/FFT_analysis2D.hpp:20-100): material(q, RVE) with
    q = [E_m, nu_m, E_i, nu_i] and RVE 1 = matrix; setLoad(E) with E = 3
    complex strains [E11, E22, E12]; runAnalysis() runs 25 iterations;
    homogenization() fills CHomo, SHomo, epHomo, sigHomo."""

    ITERATIONS = 25

    def __init__(self, Nx, Ny):
        self.Nx, self.Ny, self.xy = Nx, Ny, Nx * Ny
        self._s = Solver2D(Nx, Ny)

    def material(self, properties, RVE):
        q = [float(v) for v in properties[:4]]
        self.Em, self.vm, self.Ei, self.vi = q
        self.mum, self.lam = q[0] / (1 + q[1]) / 2, q[1] * q[0] / (1 + q[1]) / (1 - 2 * q[1])
        self.mui, self.lai = q[2] / (1 + q[3]) / 2, q[3] * q[2] / (1 + q[3]) / (1 - 2 * q[3])
        self.Cm = np.array([[self.lam + 2 * self.mum, self.lam, 0], [self.lam, self.lam + 2 * self.mum, 0],
                            [0, 0, 2 * self.mum]])
        self.Ci = np.array([[self.lai + 2 * self.mui, self.lai, 0], [self.lai, self.lai + 2 * self.mui, 0],
                            [0, 0, 2 * self.mui]])
        self.C0 = (self.Cm + self.Ci) / 2.0
        self.la0, self.mu0 = (self.lai + self.lam) / 2.0, (self.mui + self.mum) / 2.0
        self.RVE = np.asarray(RVE).ravel()
        self._s.material(q, (self.RVE == 1).astype(np.int32))

    def setLoad(self, E):
        self.E = np.asarray(E, np.complex128).ravel()[:3]
        self._s.set_load(self.E)

    def runAnalysis(self):
        self._s.run(self.ITERATIONS)
        self.epsilon, self.sigma = self._s.fields()

    def homogenization(self):
        self.CHomo, self.epHomo, self.sigHomo = self._s.homogenize(self.ITERATIONS)
        self.SHomo = np.linalg.inv(self.CHomo)
        self.epsilon, self.sigma = self._s.fields()
        return self.CHomo


class Server:
    """Device-resident serving loop (m3d_serve_*): submit RVE solves from any
    thread, poll or wait for their results."""

    def __init__(self, mem_budget_bytes=0.0, workers=8):
        self.L = load_library()
        h = ctypes.c_void_p()
        _check(self.L, self.L.m3d_serve_create(float(mem_budget_bytes), workers, ctypes.byref(h)), "serve_create")
        self.h = h
        self.fields = {}

    def submit(self, kind, shape, phase, E, *, mat=None, km=0.0, ki=0.0, behav=ELASTIC, precision=FP32_REFINE,
               scheme=SCHEME_AUTO, X0=None, nInc=1, tol=1e-6, max_iter=0, keep_field=False):
        ph = np.ascontiguousarray(np.asarray(phase).ravel(), np.int32)
        Ea = np.ascontiguousarray(E, np.float64)
        ma = None if mat is None else np.ascontiguousarray(mat, np.float64)
        Xa = None if X0 is None else np.ascontiguousarray(X0, np.float64)
        r = Request(kind, behav, *shape, _PRECISIONS[precision], _ptr(ma), 0 if ma is None else ma.shape[0],
                    float(km), float(ki), _ptr(ph), scheme, _ptr(Ea), _ptr(Xa), nInc, float(tol), max_iter,
                    1 if keep_field else 0)
        t = ctypes.c_longlong()
        _check(self.L, self.L.m3d_serve_submit(self.h, ctypes.byref(r), ctypes.byref(t)), "serve_submit")
        if keep_field:
            self.fields[t.value] = (6 if kind == KIND_MECH else 3, int(np.prod(shape)))
        return t.value

    def poll(self, ticket):
        r = Result()
        rc = self.L.m3d_serve_poll(self.h, ticket, ctypes.byref(r))
        if rc == PENDING:
            return None
        _check(self.L, rc, "serve_poll")
        return r.as_dict()

    def wait(self, ticket, timeout_ms=-1.0):
        r = Result()
        rc = self.L.m3d_serve_wait(self.h, ticket, float(timeout_ms), ctypes.byref(r))
        if rc == PENDING:
            return None
        _check(self.L, rc, "serve_wait")
        return r.as_dict()

    def field(self, ticket):
        """(c, V) strain field of a finished keep_field request (released after the call)."""
        c, V = self.fields.pop(ticket)
        out = np.zeros(c * V)
        _check(self.L, self.L.m3d_serve_get_field(self.h, ticket, _ptr(out)), "serve_get_field")
        return out.reshape(V, c).T

    def stats(self):
        st = ServeStats()
        _check(self.L, self.L.m3d_serve_get_stats(self.h, ctypes.byref(st)), "serve_stats")
        return {k: getattr(st, k) for k, _ in st._fields_}

    def close(self):
        if getattr(self, "h", None):
            self.L.m3d_serve_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _iso_C(la, mu):
    C = np.zeros((6, 6))
    C[:3, :3] = la
    C[[0, 1, 2], [0, 1, 2]] = la + 2 * mu
    C[[3, 4, 5], [3, 4, 5]] = 2 * mu
    return C


class FFT_Analysis3D:
    """Drop-in mirror of the reference's ``FFT_Analysis3D`` (include/FFT_analysis3D.hpp:36-215)."""

    def __init__(self, Nx, Ny, Nz, mater_behav="e", precision="fp64", criterion=CRIT_REFERENCE):
        if mater_behav not in _BEHAV:
            raise ValueError('mater_behav must be "e", "ep" or "ed"')
        self.Nx, self.Ny, self.Nz = Nx, Ny, Nz
        self.xyz = Nx * Ny * Nz
        self.mater_behav = mater_behav
        self.precision = precision
        self.criterion = criterion
        self._s = Solver(KIND_MECH, Nx, Ny, Nz, _BEHAV[mater_behav], precision, 1)
        self.epsilon = np.zeros((6, self.xyz))
        self.sigma = np.zeros((6, self.xyz))

    # material(), src/3d/FFT_analysis3D.cpp:420-549
    def material(self, mat, RVE, noPhases=None):
        mat = np.asarray(mat, np.float64)
        self.noPhases = mat.shape[0] if noPhases is None else noPhases
        self._mat = mat[: self.noPhases].copy()
        self._rve = np.asarray(RVE).ravel().astype(np.int32)
        self._s.set_material_mech(self._mat, self._rve)
        st = self._s.stats()
        self.strainBase = st["scheme"] == 1
        self.stressBase = not self.strainBase
        self.la0, self.mu0 = st["la0"], st["mu0"]
        self.vol_fractions = np.array(st["vol_fraction"][: self.noPhases])
        El, v = self._mat[:, 0], self._mat[:, 1]
        self.mu = El / (1 + v) / 2.0
        self.la = v * El / (1 + v) / (1 - 2 * v)
        self.K = self.la + 2.0 / 3.0 * self.mu
        self.C = [_iso_C(self.la[i], self.mu[i]) for i in range(self.noPhases)]
        self.S = [np.linalg.inv(c) for c in self.C]
        self.C0 = _iso_C(self.la0, self.mu0)
        self.S0 = np.linalg.inv(self.C0)

    def setLoad(self, E, X0=None):
        self.E = np.asarray(E, np.float64).ravel().copy()
        self.X0 = np.zeros(6) if X0 is None else np.asarray(X0, np.float64).ravel().copy()
        self._s.set_load(self.E, self.X0)

    def runAnalysis(self, tol_field, tol_eq, nInc=1):
        rc = self._s.run(tol_field, tol_eq, nInc, self.criterion)
        self._fetch()
        return rc

    def _fetch(self, b=0):
        self.epsilon = np.ascontiguousarray(self._s.field(FIELD_STRAIN, b))
        self.sigma = np.ascontiguousarray(self._s.field(FIELD_STRESS, b))
        if self.mater_behav == "ep":
            self.epsilon_p_eff = self._s.field(FIELD_EPS_P, b)
        if self.mater_behav == "ed":
            self.d = self._s.field(FIELD_DAMAGE, b)
        if self.mater_behav != "e":
            self.prop_homogenized = self._s.increments()
        self.itNo = self._s.stats()["iters"]

    # homogenization(), src/3d/FFT_analysis3D.cpp:856-999
    def homogenization(self, tol_field, tol_eq, outputName=None):
        if self.mater_behav != "e":
            s = Solver(KIND_MECH, self.Nx, self.Ny, self.Nz, ELASTIC, self.precision, 6)
            s.set_material_mech(self._mat, self._rve)
            self._s, self.mater_behav = s, "e"
        Ce, Se, ep, sg, _ = self._s.homogenize(tol_field, tol_eq, self.criterion)
        self.CHomo, self.SHomo, self.epHomo, self.sigHomo = Ce, Se, ep, sg
        self.E11, self.E22, self.E33 = 1 / Se[0, 0], 1 / Se[1, 1], 1 / Se[2, 2]
        self._fetch(5)
        return self.E11 + self.E22 + self.E33

    def stats(self):
        return self._s.stats()


class FFT_analysis3d_thermal:
    """Drop-in mirror of the reference's ``FFT_analysis3d_thermal`` (include/FFT_thermal3D.hpp:37-154)."""

    def __init__(self, Nx, Ny, Nz, precision="fp64", criterion=CRIT_REFERENCE):
        self.Nx, self.Ny, self.Nz = Nx, Ny, Nz
        self.xyz = Nx * Ny * Nz
        self.criterion = criterion
        self._s = Solver(KIND_THERMAL, Nx, Ny, Nz, ELASTIC, precision, 1)
        self._E = None

    def material(self, km, ki, RVE):
        self._s.set_material_thermal(km, ki, np.asarray(RVE).ravel().astype(np.int32))
        st = self._s.stats()
        self.tempGradientBase = st["scheme"] == 1
        self.heatFluxBase = not self.tempGradientBase
        self.k0 = st["k0"]
        self.Km, self.Ki, self.K0 = np.eye(3) * km, np.eye(3) * ki, np.eye(3) * self.k0
        if self._E is not None:
            self._s.set_load(self._E)

    def setLoad(self, E):
        self._E = np.asarray(E, np.float64).ravel().copy()
        self.E = self._E
        try:
            self._s.set_load(self._E)
        except M3DError:
            pass

    def runAnalysis(self, tol_field, tol_eq):
        rc = self._s.run(tol_field, tol_eq, 1, self.criterion)
        self._fetch()
        return rc

    def _fetch(self, b=0):
        self.tempGradient = np.ascontiguousarray(self._s.field(FIELD_STRAIN, b))
        self.heatFlux = np.ascontiguousarray(self._s.field(FIELD_STRESS, b))
        self.itNo = self._s.stats()["iters"]

    def homogenization(self, tol_field, tol_eq, filename=None):
        K, R, g, q, _ = self._s.homogenize(tol_field, tol_eq, self.criterion)
        self.KHomo, self.RHomo, self.tempGradHomo, self.heatFluxHomo = K, R, g, q
        self.K11, self.K22, self.K33 = K[0, 0], K[1, 1], K[2, 2]
        self._fetch(2)
        return K

    def stats(self):
        return self._s.stats()


# ---- microstructure reconstruction (m3drec_*) -------------------------------
def _shift(name, a, Nx, Ny, Nz):
    L = load_library()
    x = np.ascontiguousarray(np.asarray(a, np.float64).ravel())
    if x.size != Nx * Ny * Nz:
        raise ValueError("size does not match Nx * Ny * Nz")
    out = np.empty_like(x)
    _check(L, getattr(L, name)(_ptr(x), _ptr(out), Nx, Ny, Nz), name)
    return out


def fftshift(a, Nx, Ny, Nz):
    """recon::fftshift (src/rec/reconstruction.cpp:47-90) of an Nx*Ny*Nz array."""
    return _shift("m3drec_fftshift", a, Nx, Ny, Nz)


def ifftshift(a, Nx, Ny, Nz):
    """recon::ifftshift (src/rec/reconstruction.cpp:97-140)."""
    return _shift("m3drec_ifftshift", a, Nx, Ny, Nz)


def fft3(a, shape, sign=-1, device=0):
    """One unnormalised 3-D complex transform on the GPU (m3drec_fft3)."""
    L = load_library()
    x = np.ascontiguousarray(np.asarray(a, np.complex128).ravel())
    out = np.empty_like(x)
    _check(L, L.m3drec_fft3(_ptr(x), _ptr(out), *shape, int(sign), device), "m3drec_fft3")
    return out


class Reconstruction:
    """Phase-retrieval reconstruction of a two-phase field from its two-point
    correlation function on the GPU (m3drec_*).  ``sections=(c1, c2)`` (2-D
    uint8 arrays indexed [y, x], i.e. images of height x width) builds the
    plan from two cut sections instead; call ``estimate_norm`` before ``run``."""

    def __init__(self, tpcf, Nx=None, Ny=None, Nz=None, device=0, sections=None):
        self.L = load_library()
        h = ctypes.c_void_p()
        if sections is not None:
            c1, c2 = (np.ascontiguousarray(np.asarray(c, np.uint8)) for c in sections)
            (h1, w1), (h2, w2) = c1.shape, c2.shape
            _check(self.L, self.L.m3drec_create_from_sections(_ptr(c1), w1, h1, _ptr(c2), w2, h2, device,
                                                              ctypes.byref(h)), "m3drec_create_from_sections")
            Nx, Ny, Nz = w1, h1, h2
        else:
            t = np.ascontiguousarray(np.asarray(tpcf, np.float64).ravel())
            if t.size != Nx * Ny * Nz:
                raise ValueError("tpcf must hold Nx * Ny * Nz values")
            _check(self.L, self.L.m3drec_create(Nx, Ny, Nz, _ptr(t), device, ctypes.byref(h)), "m3drec_create")
        self.Nx, self.Ny, self.Nz, self.xyz = Nx, Ny, Nz, Nx * Ny * Nz
        self.h = h

    def estimate_norm(self):
        _check(self.L, self.L.m3drec_estimate_norm(self.h), "estimateNormFFT_RVE")

    def norm(self):
        out = np.zeros(self.xyz)
        _check(self.L, self.L.m3drec_get_norm(self.h, _ptr(out)), "get_norm")
        return out

    def save_images(self, folder):
        _check(self.L, self.L.m3drec_save_images(self.h, str(folder).encode()), "saveRecImages")

    def write_vti(self, path, tpcf):
        t = np.ascontiguousarray(np.asarray(tpcf, np.float64).ravel())
        _check(self.L, self.L.m3drec_write_vti(self.h, str(path).encode(), _ptr(t)), "vtiWriter")

    def seed(self, seed):
        _check(self.L, self.L.m3drec_seed(self.h, int(seed)), "seed")

    def run(self, n, beta):
        _check(self.L, self.L.m3drec_run(self.h, int(n), float(beta)), "runRec")

    def iterate(self, iters, beta):
        _check(self.L, self.L.m3drec_iterate(self.h, int(iters), float(beta)), "iterate")

    def threshold(self):
        _check(self.L, self.L.m3drec_threshold(self.h), "threshold")

    def set_state(self, field, i, j, call):
        f = np.ascontiguousarray(np.asarray(field, np.complex128).ravel())
        if f.size != self.xyz:
            raise ValueError("field must hold Nx * Ny * Nz complex values")
        _check(self.L, self.L.m3drec_set_state(self.h, _ptr(f), int(i), int(j), int(call)), "set_state")

    def get_state(self):
        f = np.zeros(self.xyz, np.complex128)
        i, j, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_ulonglong()
        _check(self.L, self.L.m3drec_get_state(self.h, _ptr(f), ctypes.byref(i), ctypes.byref(j), ctypes.byref(c)),
               "get_state")
        return dict(field=f, i=i.value, j=j.value, call=c.value)

    def field(self):
        out = np.zeros(self.xyz)
        _check(self.L, self.L.m3drec_get_field(self.h, _ptr(out)), "get_field")
        return out

    def errors(self):
        n = ctypes.c_int()
        _check(self.L, self.L.m3drec_get_error(self.h, None, 0, ctypes.byref(n)), "get_error")
        out = np.zeros(n.value)
        _check(self.L, self.L.m3drec_get_error(self.h, _ptr(out), n.value, ctypes.byref(n)), "get_error")
        return out

    def set_profiling(self, on):
        _check(self.L, self.L.m3drec_set_profiling(self.h, 1 if on else 0), "set_profiling")

    def profile(self):
        ms = np.zeros(6)
        n = ctypes.c_longlong()
        _check(self.L, self.L.m3drec_profile(self.h, _ptr(ms), ctypes.byref(n)), "profile")
        return ms, n.value

    def kernel_launches(self):
        return int(self.L.m3drec_kernel_launches(self.h))

    def stream_ptr(self):
        return self.L.m3drec_get_stream(self.h)

    def close(self):
        if getattr(self, "h", None):
            self.L.m3drec_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class recPlan:
    """Drop-in mirror of ``recon::recPlan`` built from a two-point correlation
    function (include/reconstruction.hpp:46-96): ``recPlan(TPCF, Nx, Ny, Nz)``,
    ``runRec(n, b)``, the members ``mTilda`` (the reconstructed field, real
    part; 0/1 after runRec) and ``trackrealerrorA`` (error of every pass run).
    ``seed`` picks the random draws (the reference's come from std::rand)."""

    def __init__(self, TPCF, Nx1, Ny1, Nz1, seed=1):
        self.Nx, self.Ny, self.Nz = Nx1, Ny1, Nz1
        self._r = Reconstruction(TPCF, Nx1, Ny1, Nz1)
        self._r.seed(seed)
        self.trackrealerrorA = np.zeros(0)
        self.mTilda = None

    @classmethod
    def from_sections(cls, c1, c2, seed=1):
        """recPlan(CImg c1, CImg c2): two cut sections (uint8, [y, x])."""
        self = cls.__new__(cls)
        self._r = Reconstruction(None, sections=(c1, c2))
        self._r.seed(seed)
        self.Nx, self.Ny, self.Nz = self._r.Nx, self._r.Ny, self._r.Nz
        self.trackrealerrorA = np.zeros(0)
        self.mTilda = None
        return self

    def estimateNormFFT_RVE(self):
        self._r.estimate_norm()

    def runRec(self, n, b):
        self._r.run(n, b)
        e = self._r.errors()
        self.trackrealerrorA = np.zeros(n)
        self.trackrealerrorA[:min(n, e.size)] = e[:n]
        self.mTilda = self._r.field()

    def saveRecImages(self, locFldr):
        self._r.save_images(locFldr)

    def vtiWriter(self, fileName, tpcf):
        self._r.write_vti(fileName, tpcf)

    def close(self):
        self._r.close()
