"""Many independent periodic boxes advanced together on one GPU.

One :class:`Batch` holds boxes of different sizes, Riemann solvers and passive
counts.  Every kernel launch of a step covers all of them, each box runs the
reference driver loop (first dt, forcing schedule, dt clamps of
3D_MPI/src/driver.f90:35-186) on its own device clock, and one step of the
whole batch is a CUDA graph replay.  See imhd_batch_* in include/imhd.h.
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import IMHD_E_PHYSICS, RECON, ImhdConfig, check, lib
from .box import RIEMANN, _dptr


def make_config(n, precision=32, riemann="roe", npass=0, sound_speed=1.0, cour=0.4, edot=0.0, dt_turb=0.05,
                ng=0, ng_pass=None, device=0, recon="plm", protect=False):
    nx, ny, nz = (n, n, n) if np.isscalar(n) else tuple(n)
    c = ImhdConfig()
    lib().imhd_default_config(ctypes.byref(c))
    c.nx, c.ny, c.nz = int(nx), int(ny), int(nz)
    c.precision = int(precision)
    c.riemann = RIEMANN[riemann] if isinstance(riemann, str) else int(riemann)
    c.recon = RECON[recon] if isinstance(recon, str) else int(recon)
    c.npass = int(npass)
    c.sound_speed = float(sound_speed)
    c.cour = float(cour)
    c.edot = float(edot)
    c.dt_turb = float(dt_turb)
    c.ng = int(ng)
    c.ng_pass = int(ng if ng_pass is None else ng_pass)
    c.device = int(device)
    c.protect = 1 if protect else 0
    return c


class Batch:
    def __init__(self, configs):
        self.cfgs = list(configs)
        arr = (ImhdConfig * len(self.cfgs))(*self.cfgs)
        self._h = ctypes.c_void_p()
        check(lib().imhd_batch_create(arr, len(self.cfgs), ctypes.byref(self._h)))

    def __len__(self):
        return len(self.cfgs)

    def close(self):
        if self._h:
            lib().imhd_batch_destroy(self._h)
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

    def _shape(self, i, nvar, g):
        c = self.cfgs[i]
        return (nvar, c.nz + 2 * g, c.ny + 2 * g, c.nx + 2 * g)

    def upload(self, i, q, b, p=None):
        c = self.cfgs[i]
        q = np.ascontiguousarray(q, dtype=np.float64)
        b = np.ascontiguousarray(b, dtype=np.float64)
        p = np.ascontiguousarray(p, dtype=np.float64) if c.npass else None
        check(lib().imhd_batch_upload(self._h, i, _dptr(q), _dptr(b), _dptr(p)))

    def set_force(self, i, delv):
        d = np.ascontiguousarray(delv, dtype=np.float64)
        check(lib().imhd_batch_set_force(self._h, i, _dptr(d)))

    def download(self, i):
        c = self.cfgs[i]
        q = np.empty(self._shape(i, 7, c.ng))
        b = np.empty(self._shape(i, 3, c.ng))
        p = np.empty(self._shape(i, c.npass, c.ng_pass)) if c.npass else None
        check(lib().imhd_batch_download(self._h, i, _dptr(q), _dptr(b), _dptr(p)))
        return q, b, p

    def schedule(self, i, steps, t0=0.0, t_end=1.0e30, dt0=1.0e-15, forcing=False):
        check(lib().imhd_batch_schedule(self._h, i, float(t0), float(t_end), int(steps), float(dt0),
                                        1 if forcing else 0))

    def run(self, replays):
        check(lib().imhd_batch_run(self._h, int(replays)))

    def clock(self, i):
        t = ctypes.c_double()
        s = ctypes.c_longlong()
        dt = ctypes.c_double()
        a = ctypes.c_int()
        rc = lib().imhd_batch_clock(self._h, i, ctypes.byref(t), ctypes.byref(s), ctypes.byref(dt), ctypes.byref(a))
        if rc not in (0, IMHD_E_PHYSICS):
            check(rc)
        # failed: the box stopped on a physics error (NaN or zero max speed)
        return {"t": t.value, "steps": s.value, "dt": dt.value, "active": bool(a.value),
                "failed": rc == IMHD_E_PHYSICS}

    def init_uniform(self, i, rho=1.0, b0=(0.0, 0.0, 0.0)):
        b = np.ascontiguousarray(b0, dtype=np.float64)
        check(lib().imhd_batch_init_uniform(self._h, i, float(rho), _dptr(b)))

    def fourier_field(self, i, target, kvec, amp, scale):
        kv = np.ascontiguousarray(kvec, dtype=np.int32).reshape(-1, 3)
        am = np.ascontiguousarray(amp, dtype=np.float64).reshape(-1, 6)
        check(lib().imhd_batch_fourier_field(self._h, i, {"velocity": 0, "force": 1}[target],
                                             kv.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), _dptr(am), len(kv),
                                             float(scale)))

    def tuning(self, enable=None):
        """Online decomposition tuning: enable / disable (None leaves it) and
        the current setting {done, tile_policy, sweep_segment, z_column}."""
        d, tp, sg, zc = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        e = -1 if enable is None else (1 if enable else 0)
        check(lib().imhd_batch_tuning(self._h, e, ctypes.byref(d), ctypes.byref(tp), ctypes.byref(sg),
                                      ctypes.byref(zc)))
        return {"done": bool(d.value), "tile_policy": tp.value, "sweep_segment": sg.value, "z_column": zc.value}

    def set_stream(self, stream_handle):
        check(lib().imhd_batch_set_stream(self._h, ctypes.c_void_p(stream_handle) if stream_handle else None))

    @property
    def launch_count(self):
        return int(lib().imhd_batch_launch_count(self._h))
