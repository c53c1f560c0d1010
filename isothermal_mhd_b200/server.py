"""Serving loop: box-solve requests with continuous batching (imhd_server_*).

    with Server(precision=32, hbm_budget=150e9) as srv:
        rid = srv.submit(spec)              # from any thread
        state, info, out = srv.poll(rid, fetch=True)

A request is a :class:`~isothermal_mhd_b200.workloads.BoxSpec` (edge, B0,
rms Mach, Riemann solver, passive scalars, steps) or the explicit fields of
:meth:`Server.submit_raw`.  The worker thread admits requests in arrival order
while their device bytes fit the budget, keeps them resident and advances all
of them together; a result does not depend on what else was resident.
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import IMHD_E_PHYSICS, REQ_STATES, SERVER_NSTATS, ImhdRequest, ImhdServerConfig, check, lib
from .batch import make_config
from .box import _dptr

STAT_NAMES = ("queued", "resident", "admitted", "completed", "failed", "graph_replays", "kernel_launches",
              "table_rebuilds", "resident_bytes", "peak_resident_bytes", "peak_resident_boxes", "build_s",
              "rebuild_s", "step_s", "retire_s", "harvest_s")
_FLOAT_STATS = ("resident_bytes", "peak_resident_bytes", "build_s", "rebuild_s", "step_s", "retire_s", "harvest_s")


class Server:
    def __init__(self, precision=32, hbm_budget=150e9, max_resident_cells=0, steps_per_round=4, device=0):
        c = ImhdServerConfig()
        lib().imhd_server_default_config(ctypes.byref(c))
        c.device = int(device)
        c.precision = int(precision)
        c.hbm_budget_bytes = float(hbm_budget)
        c.max_resident_cells = int(max_resident_cells)
        c.steps_per_round = int(steps_per_round)
        self.precision = precision
        self._cfgs = {}
        self._h = ctypes.c_void_p()
        check(lib().imhd_server_start(ctypes.byref(c), ctypes.byref(self._h)))

    # -------------------------------------------------------------- requests
    def submit_raw(self, cfg, steps, rho=1.0, b0=(0.0, 0.0, 0.0), kvec=None, amp_velocity=None, scale_velocity=0.0,
                   amp_force=None, scale_force=0.0, forcing=False, t_end=0.0, dt0=0.0):
        r = ImhdRequest()
        r.box = cfg
        r.steps = int(steps)
        r.t_end = float(t_end)
        r.dt0 = float(dt0)
        r.rho = float(rho)
        for d in range(3):
            r.b0[d] = float(b0[d])
        keep = []
        if kvec is not None:
            kv = np.ascontiguousarray(kvec, dtype=np.int32).reshape(-1, 3)
            keep.append(kv)
            r.nmodes = len(kv)
            r.kvec = kv.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
            if amp_velocity is not None:
                av = np.ascontiguousarray(amp_velocity, dtype=np.float64).reshape(-1, 6)
                keep.append(av)
                r.amp_velocity = _dptr(av)
            if amp_force is not None:
                af = np.ascontiguousarray(amp_force, dtype=np.float64).reshape(-1, 6)
                keep.append(af)
                r.amp_force = _dptr(af)
        r.scale_velocity = float(scale_velocity)
        r.scale_force = float(scale_force)
        r.forcing = 1 if forcing else 0
        rid = ctypes.c_longlong()
        check(lib().imhd_server_submit(self._h, ctypes.byref(r), ctypes.byref(rid)))
        self._cfgs[rid.value] = (cfg.nx, cfg.ny, cfg.nz, cfg.npass, cfg.ng, cfg.ng_pass)
        return rid.value

    def submit(self, spec, cour=0.4, forcing=True):
        """Queue the driven-turbulence box of a BoxSpec."""
        kv, av, sv, af, sf = spec.fields()
        cfg = make_config(spec.n, precision=self.precision, riemann=spec.riemann, npass=spec.npass, cour=cour,
                          edot=spec.edot if forcing else 0.0, dt_turb=spec.dt_turb, recon=spec.recon)
        return self.submit_raw(cfg, spec.steps, rho=1.0, b0=spec.b0, kvec=kv, amp_velocity=av, scale_velocity=sv,
                               amp_force=af if forcing else None, scale_force=sf, forcing=forcing)

    def poll(self, rid, fetch=False):
        """(state, info, arrays): state in queued/running/done/failed/cancelled;
        info {t, steps, latency_s, queue_wait_s, status[, error]}; arrays
        (q, bface, qpass) when fetch and done -- the result is then released.
        A failed request (physics error, or larger than the budget) returns
        state "failed" with the reason in info["error"]."""
        st = ctypes.c_int()
        info = np.zeros(5)
        q = b = p = None
        nx, ny, nz, npass, ng, ngp = self._cfgs[rid]
        args = [None, None, None]
        if fetch:
            # look first, allocate the result arrays only once it is done
            state, inf, _ = self.poll(rid, fetch=False)
            if state != "done":
                return state, inf, None
            q = np.empty((7, nz + 2 * ng, ny + 2 * ng, nx + 2 * ng))
            b = np.empty((3, nz + 2 * ng, ny + 2 * ng, nx + 2 * ng))
            p = np.empty((npass, nz + 2 * ngp, ny + 2 * ngp, nx + 2 * ngp)) if npass else None
            args = [_dptr(q), _dptr(b), _dptr(p)]
        rc = lib().imhd_server_poll(self._h, int(rid), ctypes.byref(st), *args, _dptr(info))
        state = REQ_STATES.get(st.value, "unknown")
        inf = {"t": info[0], "steps": int(info[1]), "latency_s": info[2], "queue_wait_s": info[3],
               "status": int(info[4])}
        if rc == IMHD_E_PHYSICS and state == "failed":
            # the box stopped on a physics error (NaN / zero speed) or was refused
            inf["error"] = lib().imhd_last_error().decode(errors="replace")
            return state, inf, None
        check(rc)
        if fetch and state == "done":
            self._cfgs.pop(rid, None)
            return state, inf, (q, b, p)
        return state, inf, None

    def stats(self):
        out = np.zeros(SERVER_NSTATS)
        check(lib().imhd_server_stats(self._h, _dptr(out), SERVER_NSTATS))
        return {k: (float(v) if k in _FLOAT_STATS else int(v)) for k, v in zip(STAT_NAMES, out)}

    def stop(self, drain=True):
        check(lib().imhd_server_stop(self._h, 1 if drain else 0))

    def close(self):
        if self._h:
            lib().imhd_server_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
