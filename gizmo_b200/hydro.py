"""Host-side mirror of GIZMO's hydro entry points over the B200 C ABI.

``HydroPass`` holds one device context (its own CUDA stream) and exposes the
reference's three entry points under their own names:

    density()              src/hydro/density_loop.cc:764
    hydro_gradient_calc()  src/hydro/gradients_loop.cc:458
    hydro_force()          src/hydro/hydro_force_loop.cc:423

The reference reads the global P[] / CellP[] arrays; here the caller uploads
the same fields (``upload``) and reads the results back (``download``). A
reference stop (endrun) becomes a ``GizmoHydroError`` carrying the same code
(1155 density did not converge, 90001009 empty bracket, 1234 no positive
Riemann pressure). All work runs in the CUDA library; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi


class GizmoHydroError(RuntimeError):
    def __init__(self, code: int, message: str = ""):
        super().__init__(f"gizmo_b200 error {code}: {message}")
        self.code = code


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def _f64(a, shape):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if a.shape != shape:
        a = a.reshape(shape)
    return a


class HydroPass:
    """One device-resident particle set and the density -> gradient -> force pass."""

    def __init__(self, params: abi.GzParams, device: int = 0):
        self.lib = abi.load_library()
        self.params = params
        self._ctx = C.c_void_p()
        rc = self.lib.gz_create(C.byref(params), int(device), C.byref(self._ctx))
        if rc:
            raise GizmoHydroError(rc, "gz_create failed")
        self.n = 0
        self._keep = []

    # -- lifecycle --------------------------------------------------------
    def close(self):
        if self._ctx:
            self.lib.gz_destroy(self._ctx)
            self._ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_params(self, params: abi.GzParams):
        self._check(self.lib.gz_set_params(self._ctx, C.byref(params)))
        self.params = params

    def set_diagnostics(self, flux_abs: bool = False):
        """Diagnostics of the force pass beyond the reference's outputs (off by
        default): flux_abs, the per-row sums of |pair flux|."""
        self._check(self.lib.gz_set_diagnostics(self._ctx, abi.DIAG_FLUX_ABS if flux_abs else 0))

    def kernel_timing(self, enable: bool = True):
        """Start (clearing the totals) or stop CUDA-event timing of the main kernels."""
        self._check(self.lib.gz_kernel_timing(self._ctx, 1 if enable else 0))

    def kernel_times(self) -> dict:
        """Per timer since the last read: kernel milliseconds, launches and work
        units (rows, targets or pair evaluations); clears the totals."""
        out = {}
        for name, t in abi.TIMERS.items():
            ms, nl, un = C.c_double(), C.c_int64(), C.c_int64()
            self._check(self.lib.gz_kernel_time(self._ctx, t, C.byref(ms), C.byref(nl), C.byref(un)))
            out[name] = {"ms": ms.value, "launches": nl.value, "units": un.value}
        return out

    @property
    def stream(self) -> int:
        return int(self.lib.gz_stream(self._ctx) or 0)

    # -- data ---------------------------------------------------------------
    def upload(self, pos, vel, mass, u, dt, h, cond=None, timebin=None, vsig=None):
        """Inputs in the caller's order; timebin (P.TimeBin) and vsig (the stored
        CellP.MaxSignalVel) are for the individual-timestep wake-up (optional)."""
        n = int(np.asarray(mass).shape[0])
        arrs = dict(pos=_f64(pos, (n, 3)), vel=_f64(vel, (n, 3)), mass=_f64(mass, (n,)), u=_f64(u, (n,)),
                    dt=_f64(dt, (n,)), h=_f64(h, (n,)),
                    cond=_f64(np.zeros(n) if cond is None else cond, (n,)))
        p = abi.GzParticles()
        p.n = n
        for k, a in arrs.items():
            setattr(p, k, _dp(a))
        keep = [arrs]
        if timebin is not None:
            tb = np.ascontiguousarray(timebin, dtype=np.int32).reshape(n)
            p.timebin = _ip(tb)
            keep.append(tb)
            if vsig is not None:
                vs = _f64(vsig, (n,))
                p.vsig = _dp(vs)
                keep.append(vs)
        self._check(self.lib.gz_upload(self._ctx, C.byref(p)))
        self.n = n

    def upload_raw(self, n: int, ptrs: dict):
        """Upload from caller-owned host buffers (e.g. pinned memory): ptrs maps
        pos/vel/mass/u/dt/h/cond to addresses of row-major FP64 arrays."""
        p = self._raw_particles(n, ptrs)
        self._check(self.lib.gz_upload(self._ctx, C.byref(p)))
        self.n = int(n)

    @staticmethod
    def _raw_particles(n: int, ptrs: dict):
        p = abi.GzParticles()
        p.n = int(n)
        for k in ("pos", "vel", "mass", "u", "dt", "h", "cond"):
            if ptrs.get(k):
                setattr(p, k, C.cast(C.c_void_p(int(ptrs[k])), C.POINTER(C.c_double)))
        return p

    @staticmethod
    def _raw_outputs(ptrs: dict):
        o = abi.GzOutputs()
        for k, v in ptrs.items():
            if k in ("iters", "wakeup"):
                setattr(o, k, C.cast(C.c_void_p(int(v)), C.POINTER(C.c_int)))
            else:
                setattr(o, k, C.cast(C.c_void_p(int(v)), C.POINTER(C.c_double)))
        return o

    def download_raw(self, ptrs: dict):
        """Download into caller-owned host buffers (addresses per output field)."""
        self._check(self.lib.gz_download(self._ctx, C.byref(self._raw_outputs(ptrs))))

    def upload_raw_async(self, n: int, ptrs: dict):
        """gz_upload_async from caller-owned (pinned) host buffers: the copies run
        beside the current pass; the next restage() takes them. The buffers must
        stay untouched until that restage returns."""
        p = self._raw_particles(n, ptrs)
        self._check(self.lib.gz_upload_async(self._ctx, C.byref(p)))
        self.n = int(n)

    def download_raw_async(self, ptrs: dict):
        """gz_download_async into caller-owned (pinned) host buffers; they are
        filled when wait() returns."""
        self._check(self.lib.gz_download_async(self._ctx, C.byref(self._raw_outputs(ptrs))))

    def wait(self):
        self._check(self.lib.gz_wait(self._ctx))

    def restage(self):
        """Rebuild grid + sorted mirror from the resident inputs (no host traffic)."""
        self._check(self.lib.gz_restage(self._ctx))

    def upload_workload(self, wl):
        self.upload(wl.pos, wl.vel, wl.mass, wl.u, wl.dt, wl.h, wl.cond)

    def download(self, fields=None) -> dict:
        n = self.n
        names = [f for f, _ in abi.OUTPUT_FIELDS] + ["iters"]
        want = names if fields is None else list(fields)
        out = {}
        o = abi.GzOutputs()
        for name, k in abi.OUTPUT_FIELDS + abi.DIAGNOSTIC_FIELDS:
            if name in want:
                a = np.zeros((n,) if k == 1 else (n, k))
                out[name] = a
                setattr(o, name, _dp(a))
        for name in ("iters", "wakeup"):
            if name in want:
                a = np.zeros(n, dtype=np.int32)
                out[name] = a
                setattr(o, name, _ip(a))
        self._check(self.lib.gz_download(self._ctx, C.byref(o)))
        return out

    # -- the three entry points ---------------------------------------------
    def _active(self, active):
        if active is None:
            return None, 0
        a = np.ascontiguousarray(active, dtype=np.int32)
        self._keep = [a]
        return _ip(a), int(a.shape[0])

    def density(self, active=None):
        ap, na = self._active(active)
        self._check(self.lib.gz_hydro_density(self._ctx, ap, na))

    def hydro_gradient_calc(self, active=None):
        ap, na = self._active(active)
        self._check(self.lib.gz_hydro_gradients(self._ctx, ap, na))

    def hydro_force(self, active=None):
        ap, na = self._active(active)
        self._check(self.lib.gz_hydro_force(self._ctx, ap, na))

    def full_pass(self, active=None):
        self.density(active)
        self.hydro_gradient_calc(active)
        self.hydro_force(active)

    def hydro_pass(self, graph: bool = True, restage: bool = False):
        """density -> gradients -> force over every particle in one call
        (gz_hydro_pass); with graph=True as one CUDA graph once a plain pass
        has sized its buffers; with restage=True the restage first (in the
        graph). Results equal full_pass()'s (after restage())."""
        flags = (abi.PASS_GRAPH if graph else 0) | (abi.PASS_RESTAGE if restage else 0)
        self._check(self.lib.gz_hydro_pass(self._ctx, flags))

    def set_boxes(self, counts=None):
        """Box sets (gz_set_boxes): the next uploads hold len(counts) consecutive
        runs of counts[b] particles, each its own periodic box; None: one box."""
        if counts is None or len(counts) <= 1:
            self._check(self.lib.gz_set_boxes(self._ctx, 0, None))
            return
        a = np.ascontiguousarray(counts, dtype=np.int64)
        self._keep.append(a)
        self._check(self.lib.gz_set_boxes(self._ctx, int(a.shape[0]), a.ctypes.data_as(C.POINTER(C.c_int64))))

    def graph_stats(self) -> dict:
        g = abi.GzGraphInfo()
        self._check(self.lib.gz_graph_stats(self._ctx, C.byref(g)))
        return {k: int(getattr(g, k)) for k, _ in abi.GzGraphInfo._fields_}

    # -- walk tuning ------------------------------------------------------------
    def tuning(self) -> dict:
        t = abi.GzTuning()
        self._check(self.lib.gz_get_tuning(self._ctx, C.byref(t)))
        return {"leaf_max": t.leaf_max, "row_slots": t.row_slots}

    def set_tuning(self, leaf_max: int, row_slots: float):
        """Walk settings for the next upload/restage (no result depends on them)."""
        t = abi.GzTuning()
        t.leaf_max, t.row_slots = int(leaf_max), float(row_slots)
        self._check(self.lib.gz_set_tuning(self._ctx, C.byref(t)))

    def autotune(self) -> dict:
        """Time the walk settings on the uploaded set and keep the fastest."""
        t = abi.GzTuning()
        self._check(self.lib.gz_autotune(self._ctx, C.byref(t)))
        return {"leaf_max": t.leaf_max, "row_slots": t.row_slots}

    # -- individual timesteps ---------------------------------------------------
    def set_bin_active(self, bin_active):
        """TimeBinActive[60] for the wake-up test of the following force passes
        over active subsets (None: off)."""
        if bin_active is None:
            self._check(self.lib.gz_set_bin_active(self._ctx, None))
            return
        b = np.ascontiguousarray(bin_active, dtype=np.int32).reshape(abi.TIMEBINS)
        self._check(self.lib.gz_set_bin_active(self._ctx, _ip(b)))

    def active_list(self, bin_active) -> np.ndarray:
        """make_list_of_active_particles on the device: ascending original indices."""
        b = np.ascontiguousarray(bin_active, dtype=np.int32).reshape(abi.TIMEBINS)
        k = C.c_int()
        self._check(self.lib.gz_active_list(self._ctx, _ip(b), None, C.byref(k)))
        out = np.zeros(max(k.value, 1), dtype=np.int32)
        self._check(self.lib.gz_active_list(self._ctx, _ip(b), _ip(out), C.byref(k)))
        return out[: k.value]

    def wakeup_bins(self, bin_active, max_time_bin_active: int, lowest_occupied_active_bin: int):
        """(new timebin of every cell, cells moved) by process_wake_ups' bin rule."""
        b = np.ascontiguousarray(bin_active, dtype=np.int32).reshape(abi.TIMEBINS)
        out = np.zeros(self.n, dtype=np.int32)
        m = C.c_int()
        self._check(self.lib.gz_wakeup_bins(self._ctx, _ip(b), int(max_time_bin_active),
                                            int(lowest_occupied_active_bin), _ip(out), C.byref(m)))
        return out, m.value

    # -- diagnostics ----------------------------------------------------------
    def neighbors(self, mode: int, active=None):
        ap, na = self._active(active)
        rows = na if active is not None else self.n
        off = np.zeros(rows + 1, dtype=np.int64)
        self._check(self.lib.gz_neighbors(self._ctx, ap, na, int(mode),
                                          off.ctypes.data_as(C.POINTER(C.c_int64)), None))
        nb = np.zeros(max(int(off[-1]), 1), dtype=np.int32)
        self._check(self.lib.gz_neighbors(self._ctx, ap, na, int(mode),
                                          off.ctypes.data_as(C.POINTER(C.c_int64)), _ip(nb)))
        return off, nb[: int(off[-1])]

    def density_sums(self, active=None):
        ap, na = self._active(active)
        rows = na if active is not None else self.n
        acc = np.zeros((rows, 14))
        pv = np.zeros((rows, 3))
        self._check(self.lib.gz_density_sums(self._ctx, ap, na, _dp(acc), _dp(pv)))
        return acc, pv

    def status(self) -> dict:
        s = abi.GzStatusInfo()
        self.lib.gz_status(self._ctx, C.byref(s))
        return dict(code=s.code, index=s.index, density_iterations=s.density_iterations,
                    pairs_density=s.pairs_density, pairs_symmetric=s.pairs_symmetric,
                    device_bytes=s.device_bytes, kernel_launches=s.kernel_launches,
                    message=s.message.decode(errors="replace"), h_iter_max=s.h_iter_max,
                    pairs_refined=s.pairs_refined)

    def _check(self, rc: int):
        if rc:
            st = self.status()
            raise GizmoHydroError(int(rc), st.get("message", ""))


KICK_DTYPES = {name: "torch.float64" for name in (
    "vel", "u", "mass", "mass_true", "dmass", "dtmass", "accel", "dudt", "grav", "gravwork", "vel_pred", "u_pred",
    "dp")}
KICK_DTYPES.update({"tstart": "torch.int64", "tend": "torch.int64", "active": "torch.int32"})
KICK_VECTORS = ("vel", "accel", "grav", "gravwork", "vel_pred", "dp")


def kick(params: abi.GzParams, fields: dict, mode: int, timebase: float, min_egy_spec: float = 0.0,
         stream: int | None = None) -> None:
    """One half-step kick of a particle set held in device memory, in place:
    do_the_kick (src/core/kicks.cc:284-545) as do_first_halfstep_kick (mode 0)
    and do_second_halfstep_kick (mode 1) apply it.

    ``fields`` maps the gz_kick_fields names to contiguous CUDA tensors in the
    caller's order ([n] or [n, 3]; FP64, ``tstart``/``tend`` int64, ``active``
    int32); ``grav``, ``gravwork`` and ``active`` may be left out, and the MFV
    fields under MFM. The work is queued on ``stream`` (a cudaStream_t handle,
    None for the default stream) and this returns without waiting."""
    n = int(fields["u"].shape[0])
    f = abi.GzKickFields()
    f.n = n
    for name, dtype in KICK_DTYPES.items():
        t = fields.get(name)
        if t is None:
            continue
        rows = 3 if name in KICK_VECTORS else 1
        if (not t.is_cuda or not t.is_contiguous() or int(t.shape[0]) != n or t.numel() != rows * n
                or str(t.dtype) != dtype):
            raise ValueError(f"kick field {name}: want a contiguous CUDA {dtype} tensor of shape "
                             f"{(n, 3) if rows == 3 else (n,)}")
        setattr(f, name, t.data_ptr())
    rc = abi.load_library().gz_kick(C.byref(params), C.byref(f), int(mode), float(timebase), float(min_egy_spec),
                                    stream)
    if rc:
        raise GizmoHydroError(rc, "gz_kick")


DRIFT_DTYPES = {name: "torch.float64" for name in (
    "pos", "vel", "pvel", "vel_pred", "grav", "accel", "divvel", "mass", "dtmass", "mass_true", "rho", "u_pred",
    "dudt", "h", "pressure")}
DRIFT_DTYPES.update({"ti_current": "torch.int64", "status": "torch.int32"})
DRIFT_VECTORS = ("pos", "vel", "pvel", "vel_pred", "grav", "accel")


def drift(params: abi.GzParams, fields: dict, time1: int, timebase: float, min_egy_spec: float = 0.0,
          stream: int | None = None) -> None:
    """Drift a particle set held in device memory to the integer time
    ``time1``, in place: drift_particle_impl
    (src/core/drift_particle_functions.h:86-260) for every gas cell, as
    move_particles (src/core/predict.cc:171) applies it.

    ``fields`` maps the gz_drift_fields names to contiguous CUDA tensors in the
    caller's order ([n] or [n, 3]; FP64, ``ti_current`` int64); ``status`` is a
    one-element int32 CUDA tensor that receives GZ_ERR_NO_PAST_DRIFT (90001004)
    if a cell's Ti_current lies after ``time1`` (that cell is left as it was).
    ``grav`` may be left out, the MFV fields under MFM, ``vel`` under MFV and
    ``pvel`` under MFM. Queued on ``stream`` without waiting."""
    n = int(fields["mass"].shape[0])
    f = abi.GzDriftFields()
    f.n = n
    for name, dtype in DRIFT_DTYPES.items():
        t = fields.get(name)
        if t is None:
            continue
        rows = 3 if name in DRIFT_VECTORS else 1
        want = 1 if name == "status" else rows * n
        if (not t.is_cuda or not t.is_contiguous() or t.numel() != want or str(t.dtype) != dtype
                or (name != "status" and int(t.shape[0]) != n)):
            raise ValueError(f"drift field {name}: want a contiguous CUDA {dtype} tensor of {want} elements")
        setattr(f, name, t.data_ptr())
    rc = abi.load_library().gz_drift(C.byref(params), C.byref(f), int(time1), float(timebase), float(min_egy_spec),
                                     stream)
    if rc:
        raise GizmoHydroError(rc, "gz_drift")


TIMESTEP_DTYPES = {name: "torch.float64" for name in (
    "grav", "accel", "vsig", "h", "num_ngb", "divvel", "mass", "softening", "aphys")}
TIMESTEP_DTYPES.update({"ti_want": "torch.int64", "bin": "torch.int32", "ti_begstep": "torch.int64",
                        "dt_step": "torch.int64", "status": "torch.int32"})
TIMESTEP_VECTORS = ("grav", "accel")


def timestep(params: abi.GzParams, tp: abi.GzTimestepParams, fields: dict, stream: int | None = None) -> None:
    """New timesteps and bins of a particle set held in device memory, in
    place: get_timestep (src/core/timestep.cc:357-1416) and the per-particle
    binning of find_timesteps (timestep.cc:176-215, 265-270).

    ``fields`` maps the gz_timestep_fields names to contiguous CUDA tensors in
    the caller's order ([n] or [n, 3]); ``grav``, ``softening``, ``aphys``,
    ``ti_want`` and ``status`` (a one-element int32 tensor that receives 888 or
    90001005) may be left out. Queued on ``stream`` without waiting."""
    n = int(fields["mass"].shape[0])
    f = abi.GzTimestepFields()
    f.n = n
    for name, dtype in TIMESTEP_DTYPES.items():
        t = fields.get(name)
        if t is None:
            continue
        rows = 3 if name in TIMESTEP_VECTORS else 1
        want = 1 if name == "status" else rows * n
        if (not t.is_cuda or not t.is_contiguous() or t.numel() != want or str(t.dtype) != dtype
                or (name != "status" and int(t.shape[0]) != n)):
            raise ValueError(f"timestep field {name}: want a contiguous CUDA {dtype} tensor of {want} elements")
        setattr(f, name, t.data_ptr())
    rc = abi.load_library().gz_timestep(C.byref(params), C.byref(tp), C.byref(f), stream)
    if rc:
        raise GizmoHydroError(rc, "gz_timestep")
