"""ctypes mirror of include/gizmo_hydro.h and the loader for the CUDA library.

The C-ABI library ``gizmo_b200/lib/libgizmo_hydro.so`` is the product: the
neighbour grid and the density / gradient / force kernels for sm_100a behind
the ``gz_*`` entry points. This module only declares the structures and
argument types; it never falls back to anything when the library is absent
(``load_library`` raises).
"""
from __future__ import annotations

import ctypes as C
import os

KERNEL_CUBIC = 3
KERNEL_WENDLAND_C2 = 6
METHOD_MFM = 0
METHOD_MFV = 1
PRECISION_FP64 = 0
PRECISION_MIXED = 1

OK = 0
ERR_ARG = 1
ERR_CUDA = 2
ERR_NO_DEVICE = 3
ERR_ORDER = 4
ERR_CAPACITY = 5
ERR_INTERNAL = 6
ERR_DENSITY_MAXITER = 1155
ERR_EMPTY_BRACKET = 90001009
ERR_RIEMANN = 1234
ERR_NO_PAST_DRIFT = 90001004
ERR_MIN_TIMESTEP = 888
ERR_END_OF_TIMELINE = 90001005

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class GzParams(C.Structure):
    _fields_ = [
        ("kernel", C.c_int),
        ("method", C.c_int),
        ("precision", C.c_int),
        ("first_step", C.c_int),
        ("selfgravity_off", C.c_int),
        ("reserved", C.c_int),
        ("box_size", C.c_double),
        ("gamma", C.c_double),
        ("des_num_ngb", C.c_double),
        ("max_num_ngb_dev", C.c_double),
        ("min_kernel_radius", C.c_double),
        ("max_kernel_radius", C.c_double),
    ]


class GzParticles(C.Structure):
    _fields_ = [
        ("n", C.c_int64),
        ("pos", _dp),
        ("vel", _dp),
        ("mass", _dp),
        ("u", _dp),
        ("dt", _dp),
        ("h", _dp),
        ("cond", _dp),
        ("timebin", _ip),
        ("vsig", _dp),
    ]


OUTPUT_FIELDS = [
    ("h", 1), ("num_ngb", 1), ("drkern", 1), ("divvel", 1), ("rho", 1), ("pressure", 1),
    ("nvt", 6), ("cond", 1), ("fce", 1), ("pvel", 3), ("grad_rho", 3), ("grad_p", 3),
    ("grad_v", 9), ("accel", 3), ("dudt", 1), ("vsig", 1), ("dtmass", 1), ("dmass", 1),
    ("gravwork", 3),
]
# downloaded only when asked for by name (no reference counterpart)
DIAGNOSTIC_FIELDS = [("flux_abs", 3)]


class GzOutputs(C.Structure):
    _fields_ = [(name, _dp) for name, _ in OUTPUT_FIELDS] + [("iters", _ip), ("wakeup", _ip), ("flux_abs", _dp)]


class GzStatusInfo(C.Structure):
    _fields_ = [
        ("code", C.c_int),
        ("index", C.c_int),
        ("density_iterations", C.c_int),
        ("reserved", C.c_int),
        ("pairs_density", C.c_int64),
        ("pairs_symmetric", C.c_int64),
        ("device_bytes", C.c_int64),
        ("kernel_launches", C.c_int64),
        ("message", C.c_char * 256),
        ("h_iter_max", C.c_double),
        ("pairs_refined", C.c_int64),
    ]


class GzKickFields(C.Structure):
    """gz_kick_fields: device pointers (as integers) of one half-step kick."""
    _fields_ = [("n", C.c_int64)] + [(name, C.c_void_p) for name in (
        "vel", "u", "mass", "mass_true", "dmass", "dtmass", "accel", "dudt", "grav", "gravwork", "vel_pred",
        "u_pred", "dp", "tstart", "tend", "active")]


class GzDriftFields(C.Structure):
    """gz_drift_fields: device pointers (as integers) of one drift."""
    _fields_ = [("n", C.c_int64)] + [(name, C.c_void_p) for name in (
        "pos", "vel", "pvel", "vel_pred", "grav", "accel", "divvel", "mass", "dtmass", "mass_true", "rho", "u_pred",
        "dudt", "h", "pressure", "ti_current", "status")]


class GzTuning(C.Structure):
    _fields_ = [("leaf_max", C.c_int), ("reserved", C.c_int), ("row_slots", C.c_double)]


class GzGraphInfo(C.Structure):
    """gz_graph_info."""
    _fields_ = [("captures", C.c_int64), ("replays", C.c_int64), ("fallbacks", C.c_int64),
                ("kernels_top", C.c_int64), ("kernels_per_iteration", C.c_int64), ("kernels_after", C.c_int64)]


class GzTimestepParams(C.Structure):
    """gz_timestep_params."""
    _fields_ = [("err_tol_int_accuracy", C.c_double), ("courant_fac", C.c_double),
                ("max_size_timestep", C.c_double), ("min_size_timestep", C.c_double), ("timebase", C.c_double),
                ("ti_current", C.c_int64), ("bin_active", C.c_int32 * 60)]


class GzTimestepFields(C.Structure):
    """gz_timestep_fields: device pointers (as integers) of one timestep update."""
    _fields_ = [("n", C.c_int64)] + [(name, C.c_void_p) for name in (
        "grav", "accel", "vsig", "h", "num_ngb", "divvel", "mass", "softening", "aphys", "ti_want", "bin",
        "ti_begstep", "dt_step", "status")]


EXPORTED_SYMBOLS = [
    "gz_create", "gz_destroy", "gz_set_params", "gz_set_diagnostics", "gz_upload", "gz_restage", "gz_hydro_density",
    "gz_hydro_gradients", "gz_hydro_force", "gz_download", "gz_status", "gz_stream", "gz_kernel_timing",
    "gz_kernel_time",
    "gz_neighbors", "gz_density_sums", "gz_density_sums_noalloc", "gz_kick",
    "gz_drift", "gz_set_bin_active", "gz_active_list", "gz_wakeup_bins", "gz_timestep",
    "gz_upload_device", "gz_download_device", "gz_get_tuning", "gz_set_tuning", "gz_autotune",
    "gz_hydro_pass", "gz_graph_stats", "gz_upload_async", "gz_download_async", "gz_wait", "gz_set_boxes",
]
PASS_GRAPH = 1  # GZ_PASS_GRAPH
PASS_RESTAGE = 2  # GZ_PASS_RESTAGE
TIMEBINS = 60  # GZ_TIMEBINS
NOALLOC_MAX_PARTICLES = 65536  # GZ_NOALLOC_MAX_PARTICLES
DIAG_FLUX_ABS = 1  # GZ_DIAG_FLUX_ABS
TIMERS = {"density_sums": 0, "walk": 1, "gradients": 2, "force": 3}  # GZ_TIMER_*

LIB_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib")
LIB_PATH = os.path.join(LIB_DIR, "libgizmo_hydro.so")

_lib = None


def load_library(path: str | None = None) -> C.CDLL:
    """Load the CUDA C-ABI library (raises when it has not been built)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(
            f"gizmo_b200: CUDA library {p} is missing; run __graft_entry__.build() "
            "(nvcc, sm_100a). There is no CPU fallback.")
    lib = C.CDLL(p)
    vp = C.c_void_p
    lib.gz_create.argtypes = [C.POINTER(GzParams), C.c_int, C.POINTER(vp)]
    lib.gz_destroy.argtypes = [vp]
    lib.gz_set_params.argtypes = [vp, C.POINTER(GzParams)]
    lib.gz_set_diagnostics.argtypes = [vp, C.c_int]
    lib.gz_kernel_timing.argtypes = [vp, C.c_int]
    lib.gz_kernel_time.argtypes = [vp, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    lib.gz_upload.argtypes = [vp, C.POINTER(GzParticles)]
    lib.gz_upload_device.argtypes = [vp, C.POINTER(GzParticles)]
    lib.gz_get_tuning.argtypes = [vp, C.POINTER(GzTuning)]
    lib.gz_set_tuning.argtypes = [vp, C.POINTER(GzTuning)]
    lib.gz_autotune.argtypes = [vp, C.POINTER(GzTuning)]
    lib.gz_download_device.argtypes = [vp, C.POINTER(GzOutputs)]
    lib.gz_restage.argtypes = [vp]
    for name in ("gz_hydro_density", "gz_hydro_gradients", "gz_hydro_force"):
        getattr(lib, name).argtypes = [vp, _ip, C.c_int]
    lib.gz_download.argtypes = [vp, C.POINTER(GzOutputs)]
    lib.gz_status.argtypes = [vp, C.POINTER(GzStatusInfo)]
    lib.gz_stream.argtypes = [vp]
    lib.gz_stream.restype = vp
    lib.gz_neighbors.argtypes = [vp, _ip, C.c_int, C.c_int, C.POINTER(C.c_int64), _ip]
    lib.gz_density_sums.argtypes = [vp, _ip, C.c_int, _dp, _dp]
    lib.gz_density_sums_noalloc.argtypes = [C.POINTER(GzParams), C.c_int, vp, vp, vp, vp, vp, vp, vp]
    lib.gz_kick.argtypes = [C.POINTER(GzParams), C.POINTER(GzKickFields), C.c_int, C.c_double, C.c_double, vp]
    lib.gz_drift.argtypes = [C.POINTER(GzParams), C.POINTER(GzDriftFields), C.c_int64, C.c_double, C.c_double,
                             vp]
    lib.gz_timestep.argtypes = [C.POINTER(GzParams), C.POINTER(GzTimestepParams), C.POINTER(GzTimestepFields), vp]
    lib.gz_set_bin_active.argtypes = [vp, _ip]
    lib.gz_active_list.argtypes = [vp, _ip, _ip, _ip]
    lib.gz_wakeup_bins.argtypes = [vp, _ip, C.c_int, C.c_int, _ip, _ip]
    for name in EXPORTED_SYMBOLS:
        if name != "gz_stream":
            getattr(lib, name).restype = C.c_int
    if path is None:
        _lib = lib
    return lib
