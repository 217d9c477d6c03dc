"""One integration step of the gas on the device, in the reference's loop order.

The reference's main loop (src/core/run.cc:148-489) takes, per step: the
timesteps (find_timesteps -> get_timestep, src/core/timestep.cc), the first
half kick (do_first_halfstep_kick, src/core/kicks.cc:34-97), the drift to the
new time (move_particles, src/core/predict.cc:171), the hydro pass on the
predicted state (density, hydro_gradient_calc, hydro_force) and the second
half kick (do_second_halfstep_kick, src/core/kicks.cc:99-182). ``DeviceStep``
runs that sequence for gas cells held as CUDA tensors, through gz_timestep,
gz_kick, gz_drift and a HydroPass fed by gz_upload_device / read by
gz_download_device, so no particle field leaves the GPU between steps.

Scope: one global step (every cell on the smallest step the timestep
criterion gives, as the reference runs with all bins active), no gravity, a
periodic box (positions are wrapped into [0, box) for the pass), the
integer timeline of the reference (Timebase_interval per tick).
"""
from __future__ import annotations

import ctypes as C

from . import abi
from .hydro import HydroPass, drift, kick, timestep

PASS_OUT = ("accel", "dudt", "dtmass", "dmass", "gravwork", "vsig", "divvel", "rho", "pressure", "num_ngb", "pvel",
            "h", "cond")
_VEC = {"accel": 3, "gravwork": 3, "pvel": 3}


class DeviceStep:
    """Gas cells on the device and the state a step carries between passes.

    ``state`` holds CUDA tensors in the caller's order: pos, vel (P.Vel), u
    (CellP.InternalEnergy), mass (P.Mass), mass_true (MFV CellP.MassTrue),
    vel_pred, u_pred, h, cond and the pass outputs of PASS_OUT.
    """

    def __init__(self, params: abi.GzParams, tp: abi.GzTimestepParams, pos, vel, mass, u, h, device: int = 0):
        import torch

        self.torch = torch
        self.params = params
        self.tp = tp
        self.dev = torch.device("cuda", device)
        t = lambda a: torch.as_tensor(a, dtype=torch.float64, device=self.dev).contiguous()  # noqa: E731
        self.n = int(mass.shape[0])
        self.mfv = params.method == abi.METHOD_MFV
        s = {"pos": t(pos), "vel": t(vel), "mass": t(mass), "u": t(u), "h": t(h)}
        s["mass_true"] = s["mass"].clone()
        s["vel_pred"] = s["vel"].clone()
        s["u_pred"] = s["u"].clone()
        s["cond"] = torch.zeros(self.n, dtype=torch.float64, device=self.dev)
        for k in PASS_OUT:
            if k not in s:
                s[k] = torch.zeros((self.n, _VEC[k]) if k in _VEC else (self.n,), dtype=torch.float64, device=self.dev)
        self.state = s
        self.ti = 0
        self.hp = HydroPass(params, device=device)
        self.stream = torch.cuda.ExternalStream(self.hp.stream, device=self.dev)
        self.status = torch.zeros(1, dtype=torch.int32, device=self.dev)
        self._pass(0.0)  # at start-up no step has been assigned (dt_step = 0): the first pass books no dMass

    def close(self):
        self.hp.close()

    def _pass(self, dt_phys: float):
        """The hydro pass on the predicted state, device arrays in and out."""
        torch, s = self.torch, self.state
        with torch.cuda.stream(self.stream):
            box = self.params.box_size
            pos = torch.remainder(s["pos"], box).contiguous()
            dt = torch.full((self.n,), dt_phys, dtype=torch.float64, device=self.dev)
            p = abi.GzParticles()
            p.n = self.n
            keep = {"pos": pos, "vel": s["vel_pred"], "mass": s["mass"], "u": s["u_pred"], "dt": dt, "h": s["h"],
                    "cond": s["cond"]}
            for k, v in keep.items():
                setattr(p, k, C.cast(C.c_void_p(v.data_ptr()), C.POINTER(C.c_double)))
        self.stream.synchronize()  # the inputs are written on this stream before the library reads them
        self.hp._check(self.hp.lib.gz_upload_device(self.hp._ctx, C.byref(p)))
        self.hp.n = self.n
        self.hp.full_pass()
        o = abi.GzOutputs()
        for k in PASS_OUT:
            setattr(o, k, C.cast(C.c_void_p(s[k].data_ptr()), C.POINTER(C.c_double)))
        self.hp._check(self.hp.lib.gz_download_device(self.hp._ctx, C.byref(o)))
        self.stream.synchronize()
        del keep

    def step(self) -> int:
        """One global step; returns its length in integer ticks."""
        torch, s, tp = self.torch, self.state, self.tp
        n = self.n
        tp.ti_current = self.ti
        i64 = lambda v: torch.full((n,), v, dtype=torch.int64, device=self.dev)  # noqa: E731
        f = {"accel": s["accel"], "vsig": s["vsig"], "h": s["h"], "num_ngb": s["num_ngb"], "divvel": s["divvel"],
             "mass": s["mass"], "bin": torch.zeros(n, dtype=torch.int32, device=self.dev), "ti_begstep": i64(0),
             "dt_step": i64(0), "status": self.status}
        sid = self.stream.cuda_stream
        with torch.cuda.stream(self.stream):
            timestep(self.params, tp, f, sid)
            step = int(f["dt_step"].min().item())  # one global step: every cell on the smallest bin
            half = step // 2
            kf = {"vel": s["vel"], "u": s["u"], "mass": s["mass"], "accel": s["accel"], "dudt": s["dudt"],
                  "vel_pred": s["vel_pred"], "u_pred": s["u_pred"], "dp": torch.zeros_like(s["vel"]),
                  "tstart": i64(self.ti), "tend": i64(self.ti + half)}
            if self.mfv:
                kf.update({"mass_true": s["mass_true"], "dmass": s["dmass"], "dtmass": s["dtmass"],
                           "gravwork": s["gravwork"]})
            kick(self.params, kf, 0, tp.timebase, 0.0, sid)
            df = {"pos": s["pos"], "vel_pred": s["vel_pred"], "accel": s["accel"], "divvel": s["divvel"],
                  "mass": s["mass"], "rho": s["rho"], "u_pred": s["u_pred"], "dudt": s["dudt"], "h": s["h"],
                  "pressure": s["pressure"], "ti_current": i64(self.ti), "status": self.status}
            if self.mfv:
                df.update({"pvel": s["pvel"], "dtmass": s["dtmass"], "mass_true": s["mass_true"]})
            else:
                df["vel"] = s["vel"]
            drift(self.params, df, self.ti + step, tp.timebase, 0.0, sid)
        self._pass(step * tp.timebase)
        with torch.cuda.stream(self.stream):
            kf["tstart"], kf["tend"] = i64(self.ti + half), i64(self.ti + step)
            kf["dp"] = torch.zeros_like(s["vel"])
            kf["dmass"] = s["dmass"]
            kick(self.params, kf, 1, tp.timebase, 0.0, sid)
        self.stream.synchronize()
        code = int(self.status.item())
        if code:
            from .hydro import GizmoHydroError
            raise GizmoHydroError(code, "device step")
        self.ti += step
        return step
