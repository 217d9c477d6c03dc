"""Python binding of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Loads ``oracle/liboracle.so`` (the C restatement, gizmo_oracle.c) and the
reference's own pair bodies compiled by ``oracle/build_ref.sh`` into
``oracle/_ref/libgizmo_ref_<config>.so``. Only tests/, __graft_entry__.smoke()
and bench.py's CPU-baseline leg use this module: it is the checker, never the
thing measured or shipped.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from gizmo_b200.abi import GzParams, METHOD_MFM, METHOD_MFV

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_ORACLE = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)

STATE_FIELDS = [  # (name, components, dtype)
    ("pos", 3, np.float64), ("vel", 3, np.float64), ("mass", 1, np.float64), ("u", 1, np.float64),
    ("dt", 1, np.float64), ("h", 1, np.float64), ("cond", 1, np.float64),
    ("num_ngb", 1, np.float64), ("drkern", 1, np.float64), ("divvel", 1, np.float64),
    ("rho", 1, np.float64), ("pressure", 1, np.float64), ("nvt", 6, np.float64), ("fce", 1, np.float64),
    ("pvel", 3, np.float64), ("iters", 1, np.int32),
    ("grad_rho", 3, np.float64), ("grad_p", 3, np.float64), ("grad_v", 9, np.float64),
    ("accel", 3, np.float64), ("dudt", 1, np.float64), ("vsig", 1, np.float64),
    ("dtmass", 1, np.float64), ("dmass", 1, np.float64), ("gravwork", 3, np.float64),
    ("timebin", 1, np.int32), ("wakeup", 1, np.int32),
]


class OrcState(C.Structure):
    _fields_ = [("n", C.c_int)] + [(name, _ip if dt == np.int32 else _dp) for name, _, dt in STATE_FIELDS]


KICK_FIELDS = [  # (name, components, dtype), the order of orc_kick_state
    ("vel", 3, np.float64), ("u", 1, np.float64), ("mass", 1, np.float64), ("mass_true", 1, np.float64),
    ("dmass", 1, np.float64), ("dtmass", 1, np.float64), ("accel", 3, np.float64), ("dudt", 1, np.float64),
    ("grav", 3, np.float64), ("gravwork", 3, np.float64), ("vel_pred", 3, np.float64), ("u_pred", 1, np.float64),
    ("dp", 3, np.float64), ("tstart", 1, np.int64), ("tend", 1, np.int64), ("active", 1, np.int32),
]
_CTYPE = {np.float64: _dp, np.int64: C.POINTER(C.c_longlong), np.int32: _ip}


class OrcKickState(C.Structure):
    _fields_ = [("n", C.c_int)] + [(name, _CTYPE[dt]) for name, _, dt in KICK_FIELDS]


def new_kick_state(n: int, inputs: dict) -> dict:
    """All kick arrays for n particles, zero except what `inputs` fills."""
    st = {}
    for name, k, dt in KICK_FIELDS:
        st[name] = np.zeros((n,) if k == 1 else (n, k), dtype=dt)
    for name, arr in inputs.items():
        st[name][...] = arr
    return st


def _c_kick_state(st: dict) -> OrcKickState:
    s = OrcKickState()
    s.n = int(st["u"].shape[0])
    for name, _, dt in KICK_FIELDS:
        a = st[name]
        assert a.flags["C_CONTIGUOUS"] and a.dtype == dt and a.shape[0] == s.n, name
        setattr(s, name, a.ctypes.data_as(_CTYPE[dt]))
    return s


DRIFT_FIELDS = [  # (name, components, dtype), the order of orc_drift_state
    ("pos", 3, np.float64), ("vel", 3, np.float64), ("pvel", 3, np.float64), ("vel_pred", 3, np.float64),
    ("grav", 3, np.float64), ("accel", 3, np.float64), ("divvel", 1, np.float64), ("mass", 1, np.float64),
    ("dtmass", 1, np.float64), ("mass_true", 1, np.float64), ("rho", 1, np.float64), ("u_pred", 1, np.float64),
    ("dudt", 1, np.float64), ("h", 1, np.float64), ("pressure", 1, np.float64), ("ti_current", 1, np.int64),
]


class OrcDriftState(C.Structure):
    _fields_ = [("n", C.c_int)] + [(name, _CTYPE[dt]) for name, _, dt in DRIFT_FIELDS]


def new_drift_state(n: int, inputs: dict) -> dict:
    """All drift arrays for n particles, zero except what `inputs` fills."""
    st = {}
    for name, k, dt in DRIFT_FIELDS:
        st[name] = np.zeros((n,) if k == 1 else (n, k), dtype=dt)
    for name, arr in inputs.items():
        st[name][...] = arr
    return st


def _c_drift_state(st: dict) -> OrcDriftState:
    s = OrcDriftState()
    s.n = int(st["mass"].shape[0])
    for name, _, dt in DRIFT_FIELDS:
        a = st[name]
        assert a.flags["C_CONTIGUOUS"] and a.dtype == dt and a.shape[0] == s.n, name
        setattr(s, name, a.ctypes.data_as(_CTYPE[dt]))
    return s


TIMESTEP_FIELDS = [  # (name, components, dtype), the order of orc_timestep_state
    ("grav", 3, np.float64), ("accel", 3, np.float64), ("vsig", 1, np.float64), ("h", 1, np.float64),
    ("num_ngb", 1, np.float64), ("divvel", 1, np.float64), ("mass", 1, np.float64), ("softening", 1, np.float64),
    ("aphys", 1, np.float64), ("ti_want", 1, np.int64), ("bin", 1, np.int32), ("ti_begstep", 1, np.int64),
    ("dt_step", 1, np.int64),
]
TIMEBINS = 60  # declarations/typedefs.h:8


class OrcTimestepState(C.Structure):
    _fields_ = [("n", C.c_int)] + [(name, _CTYPE[dt]) for name, _, dt in TIMESTEP_FIELDS]


class OrcTimestepParams(C.Structure):
    _fields_ = [("err_tol_int_accuracy", C.c_double), ("courant_fac", C.c_double),
                ("max_size_timestep", C.c_double), ("min_size_timestep", C.c_double), ("timebase", C.c_double),
                ("ti_current", C.c_longlong), ("bin_active", C.c_int * TIMEBINS)]


def new_timestep_state(n: int, inputs: dict) -> dict:
    """All timestep arrays for n cells, zero except what `inputs` fills."""
    st = {}
    for name, k, dt in TIMESTEP_FIELDS:
        st[name] = np.zeros((n,) if k == 1 else (n, k), dtype=dt)
    for name, arr in inputs.items():
        st[name][...] = arr
    return st


def _c_timestep_state(st: dict) -> OrcTimestepState:
    s = OrcTimestepState()
    s.n = int(st["mass"].shape[0])
    for name, _, dt in TIMESTEP_FIELDS:
        a = st[name]
        assert a.flags["C_CONTIGUOUS"] and a.dtype == dt and a.shape[0] == s.n, name
        setattr(s, name, a.ctypes.data_as(_CTYPE[dt]))
    return s


class OrcCsr(C.Structure):
    _fields_ = [("offsets", C.POINTER(C.c_longlong)), ("nbrs", _ip), ("n_rows", C.c_int)]


def new_state(n: int, inputs: dict) -> dict:
    """All state arrays for n particles; `inputs` fills pos/vel/mass/u/dt/h/cond."""
    st = {}
    for name, k, dt in STATE_FIELDS:
        shape = (n,) if k == 1 else (n, k)
        st[name] = np.zeros(shape, dtype=dt)
    for name, arr in inputs.items():
        st[name][...] = arr
    return st


def _c_state(st: dict) -> OrcState:
    s = OrcState()
    s.n = int(st["pos"].shape[0])
    for name, _, dt in STATE_FIELDS:
        a = st[name]
        assert a.flags["C_CONTIGUOUS"] and a.dtype == dt, name
        setattr(s, name, a.ctypes.data_as(_ip if dt == np.int32 else _dp))
    return s


def build_oracle() -> None:
    subprocess.run(["make", "-s", "liboracle.so"], cwd=HERE, check=True)


def build_reference() -> None:
    subprocess.run([os.path.join(HERE, "build_ref.sh")], check=True)


def _setup(lib: C.CDLL, prefix: str) -> C.CDLL:
    for name in ("density", "gradients", "force"):
        f = getattr(lib, f"{prefix}_{name}")
        f.argtypes = [C.POINTER(GzParams), C.POINTER(OrcState), _ip, C.c_int, C.c_int]
        f.restype = C.c_int
    f = getattr(lib, f"{prefix}_force_wakeup")
    f.argtypes = [C.POINTER(GzParams), C.POINTER(OrcState), _ip, C.c_int, C.c_int, _ip]
    f.restype = C.c_int
    f = getattr(lib, f"{prefix}_density_sums")
    f.argtypes = [C.POINTER(GzParams), C.POINTER(OrcState), _ip, C.c_int, _dp, _dp, C.c_int]
    f.restype = C.c_int
    f = getattr(lib, f"{prefix}_kick")
    f.argtypes = [C.POINTER(GzParams), C.POINTER(OrcKickState), C.c_int, C.c_double, C.c_double]
    f.restype = C.c_int
    f = getattr(lib, f"{prefix}_drift")
    f.argtypes = [C.POINTER(GzParams), C.POINTER(OrcDriftState), C.c_longlong, C.c_double, C.c_double]
    f.restype = C.c_int
    f = getattr(lib, f"{prefix}_timestep")
    f.argtypes = [C.POINTER(GzParams), C.POINTER(OrcTimestepParams), C.POINTER(OrcTimestepState)]
    f.restype = C.c_int
    if hasattr(lib, f"{prefix}_active_list"):
        f = getattr(lib, f"{prefix}_active_list")
        f.argtypes = [C.c_int, _ip, _dp, _ip, _ip]
        f.restype = C.c_int
        f = getattr(lib, f"{prefix}_wakeup_bins")
        f.argtypes = [C.c_int, _ip, _ip, _dp, _ip, C.c_int, C.c_int, _ip]
        f.restype = C.c_int
    if hasattr(lib, f"{prefix}_riemann_branches"):
        f = getattr(lib, f"{prefix}_riemann_branches")
        f.argtypes = [C.POINTER(C.c_longlong)]
        f.restype = None
    if hasattr(lib, f"{prefix}_density_h_iter_max"):
        f = getattr(lib, f"{prefix}_density_h_iter_max")
        f.argtypes = []
        f.restype = C.c_double
    f = getattr(lib, f"{prefix}_full_pass_seconds")
    f.argtypes = [C.POINTER(GzParams), C.POINTER(OrcState), _ip, C.c_int, C.c_int, _ip]
    f.restype = C.c_double
    return lib


_libs: dict = {}


def ref_config_name(params: GzParams) -> str:
    g = {5.0 / 3.0: "g53", 1.0001: "g1"}.get(float(params.gamma))
    m = {METHOD_MFM: "mfm", METHOD_MFV: "mfv"}[params.method]
    if g is None:
        raise ValueError(f"no reference build for gamma={params.gamma}")
    return f"{m}_k{params.kernel}_{g}"


def ref_available(params: GzParams) -> bool:
    try:
        return os.path.exists(os.path.join(REF_DIR, f"libgizmo_ref_{ref_config_name(params)}.so"))
    except ValueError:
        return False


class Oracle:
    """The C restatement (kind='port') or the compiled reference (kind='reference')."""

    def __init__(self, params: GzParams, kind: str = "port", n_threads: int = 0):
        self.params = params
        self.kind = kind
        self.n_threads = n_threads
        if kind == "port":
            key = LIB_ORACLE
            if key not in _libs:
                if not os.path.exists(LIB_ORACLE):
                    build_oracle()
                _libs[key] = _setup(C.CDLL(LIB_ORACLE), "orc")
            self.prefix = "orc"
        elif kind == "reference":
            key = os.path.join(REF_DIR, f"libgizmo_ref_{ref_config_name(params)}.so")
            if key not in _libs:
                if not os.path.exists(key):
                    raise FileNotFoundError(key)
                _libs[key] = _setup(C.CDLL(key), "ref")
            self.prefix = "ref"
        else:
            raise ValueError(kind)
        self.lib = _libs[key]

    def _act(self, active):
        if active is None:
            return None, 0
        a = np.ascontiguousarray(active, dtype=np.int32)
        return a, len(a)

    def _run(self, name: str, st: dict, active=None) -> int:
        a, na = self._act(active)
        cs = _c_state(st)
        f = getattr(self.lib, f"{self.prefix}_{name}")
        return int(f(C.byref(self.params), C.byref(cs), a.ctypes.data_as(_ip) if a is not None else None, na,
                     self.n_threads))

    def density(self, st, active=None):
        return self._run("density", st, active)

    def riemann_branches(self) -> dict:
        """Pair evaluations of the last force pass per rare Riemann branch (port only)."""
        out = (C.c_longlong * 4)()
        getattr(self.lib, f"{self.prefix}_riemann_branches")(out)
        return dict(zip(("kt", "exact", "retry_centred", "retry_at_rest"), (int(v) for v in out)))

    def density_h_iter_max(self) -> float:
        """The largest kernel length at which the last density pass took sums (port only)."""
        return float(getattr(self.lib, f"{self.prefix}_density_h_iter_max")())

    def gradients(self, st, active=None):
        return self._run("gradients", st, active)

    def force(self, st, active=None):
        return self._run("force", st, active)

    def force_wakeup(self, st, bin_active, active=None):
        """The force pass with the wake-up of inactive neighbours (TimeBinActive = bin_active[60])."""
        a, na = self._act(active)
        cs = _c_state(st)
        bins = np.ascontiguousarray(bin_active, dtype=np.int32)
        assert bins.shape == (TIMEBINS,)
        f = getattr(self.lib, f"{self.prefix}_force_wakeup")
        return int(f(C.byref(self.params), C.byref(cs), a.ctypes.data_as(_ip) if a is not None else None, na,
                     self.n_threads, bins.ctypes.data_as(_ip)))

    def density_sums(self, st, active=None):
        a, na = self._act(active)
        n_rows = na if a is not None else st["pos"].shape[0]
        acc = np.zeros((n_rows, 14))
        pv = np.zeros((n_rows, 3))
        cs = _c_state(st)
        f = getattr(self.lib, f"{self.prefix}_density_sums")
        rc = f(C.byref(self.params), C.byref(cs), a.ctypes.data_as(_ip) if a is not None else None, na,
               acc.ctypes.data_as(_dp), pv.ctypes.data_as(_dp), self.n_threads)
        if rc:
            raise RuntimeError(f"density_sums failed: {rc}")
        return acc, pv

    def kick(self, st: dict, mode: int, timebase: float, min_egy_spec: float = 0.0) -> int:
        """One half-step kick (mode 0 first, 1 second) of the kick state, in place."""
        cs = _c_kick_state(st)
        f = getattr(self.lib, f"{self.prefix}_kick")
        return int(f(C.byref(self.params), C.byref(cs), int(mode), float(timebase), float(min_egy_spec)))

    def drift(self, st: dict, time1: int, timebase: float, min_egy_spec: float = 0.0) -> int:
        """Drift every cell of the drift state to the integer time `time1`, in place."""
        cs = _c_drift_state(st)
        f = getattr(self.lib, f"{self.prefix}_drift")
        return int(f(C.byref(self.params), C.byref(cs), int(time1), float(timebase), float(min_egy_spec)))

    def timestep(self, st: dict, tp: "OrcTimestepParams") -> int:
        """New timesteps and bins of every cell of the timestep state, in place."""
        cs = _c_timestep_state(st)
        f = getattr(self.lib, f"{self.prefix}_timestep")
        return int(f(C.byref(self.params), C.byref(tp), C.byref(cs)))

    def full_pass_seconds(self, st, active=None):
        a, na = self._act(active)
        cs = _c_state(st)
        status = C.c_int(0)
        f = getattr(self.lib, f"{self.prefix}_full_pass_seconds")
        t = f(C.byref(self.params), C.byref(cs), a.ctypes.data_as(_ip) if a is not None else None, na,
              self.n_threads, C.byref(status))
        return float(t), int(status.value)


def neighbors(params: GzParams, st: dict, mode: int, active=None, n_threads: int = 0):
    """Exact neighbour sets (CSR, original indices, sorted rows) from the C oracle."""
    lib = Oracle(params, "port").lib
    lib.orc_neighbors.argtypes = [C.POINTER(GzParams), C.POINTER(OrcState), _ip, C.c_int, C.c_int,
                                  C.POINTER(OrcCsr), C.c_int]
    lib.orc_neighbors.restype = C.c_int
    lib.orc_csr_free.argtypes = [C.POINTER(OrcCsr)]
    a = None if active is None else np.ascontiguousarray(active, dtype=np.int32)
    na = 0 if a is None else len(a)
    cs = _c_state(st)
    out = OrcCsr()
    rc = lib.orc_neighbors(C.byref(params), C.byref(cs), a.ctypes.data_as(_ip) if a is not None else None, na, mode,
                           C.byref(out), n_threads)
    if rc:
        raise RuntimeError(f"orc_neighbors failed: {rc}")
    n_rows = out.n_rows
    off = np.ctypeslib.as_array(out.offsets, shape=(n_rows + 1,)).astype(np.int64).copy()
    nb = np.ctypeslib.as_array(out.nbrs, shape=(max(int(off[-1]), 1),))[: int(off[-1])].astype(np.int32).copy()
    lib.orc_csr_free(C.byref(out))
    return off, nb


def active_list(timebin, mass, bin_active) -> np.ndarray:
    """make_list_of_active_particles (core/run.cc:997-1010), ascending indices."""
    lib = Oracle(GzParams(), "port").lib
    tb = np.ascontiguousarray(timebin, dtype=np.int32)
    m = np.ascontiguousarray(mass, dtype=np.float64)
    ba = np.ascontiguousarray(bin_active, dtype=np.int32)
    out = np.zeros(max(len(tb), 1), dtype=np.int32)
    k = lib.orc_active_list(len(tb), tb.ctypes.data_as(_ip), m.ctypes.data_as(_dp), ba.ctypes.data_as(_ip),
                            out.ctypes.data_as(_ip))
    return out[:k]


def wakeup_bins(timebin, wakeup, mass, bin_active, max_time_bin_active: int, lowest_occupied_active_bin: int):
    """(new timebins, cells moved) by process_wake_ups' rule (core/timestep.cc:1565-1700)."""
    lib = Oracle(GzParams(), "port").lib
    tb = np.ascontiguousarray(timebin, dtype=np.int32)
    wk = np.ascontiguousarray(wakeup, dtype=np.int32)
    m = np.ascontiguousarray(mass, dtype=np.float64)
    ba = np.ascontiguousarray(bin_active, dtype=np.int32)
    out = np.zeros(len(tb), dtype=np.int32)
    moved = lib.orc_wakeup_bins(len(tb), tb.ctypes.data_as(_ip), wk.ctypes.data_as(_ip), m.ctypes.data_as(_dp),
                                ba.ctypes.data_as(_ip), int(max_time_bin_active), int(lowest_occupied_active_bin),
                                out.ctypes.data_as(_ip))
    return out, int(moved)
