"""One periodic isothermal-MHD box on a B200, driven through the C ABI.

This is the host-side mirror of the reference's hot-path interface
(3D_MPI/src): the module procedures that the Fortran driver calls once per
time step act on module-global arrays there; here they act on the state of a
:class:`Box` kept resident in HBM.

=====================================  =========================================
reference (3D_MPI/src)                 here
=====================================  =========================================
create_grid_arrays, init_solver_*      ``Box(...)``  (imhd_create)
q_3d / bface_3d / qpass_3d hand-over   ``Box.upload`` / ``Box.download``
generate_rand_force -> delv_re         ``Box.set_force``  (imhd_set_force)
copy_velocity + vanleer_solve_3d +     ``Box.step(dt, drive_next)``  (imhd_step)
passive_solve_3d + boundary fill +
compute_new_time_step
get_max_speed_vanleer                  ``Box.max_speed``
compute_KE, compute_divB               ``Box.diagnostics``
=====================================  =========================================

Host arrays use the reference's layout: numpy C-order ``(nvar, nz+2g, ny+2g,
nx+2g)`` float64 is exactly Fortran ``q_3d(1-g:nx+g, 1-g:ny+g, 1-g:nz+g, nvar)``.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import ImhdConfig, check, lib

RIEMANN = {"roe": 1, "hlld": 2, "hlle": 3}


def _dptr(a):
    if a is None:
        return None
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Box:
    """A periodic box with nx*ny*nz interior cells, dx = 1/max(n)."""

    def __init__(self, n, precision=64, riemann="hlld", recon="plm", npass=1, sound_speed=1.0, cour=0.35,
                 edot=1.0e-3, dt_turb=0.05, ng=0, ng_pass=None, device=0, protect=False):
        nx, ny, nz = (n, n, n) if np.isscalar(n) else tuple(n)
        cfg = ImhdConfig()
        lib().imhd_default_config(ctypes.byref(cfg))
        cfg.nx, cfg.ny, cfg.nz = int(nx), int(ny), int(nz)
        cfg.precision = int(precision)
        cfg.riemann = RIEMANN[riemann] if isinstance(riemann, str) else int(riemann)
        cfg.recon = _lib.RECON[recon]
        cfg.npass = int(npass)
        cfg.sound_speed = float(sound_speed)
        cfg.cour = float(cour)
        cfg.edot = float(edot)
        cfg.dt_turb = float(dt_turb)
        cfg.ng = int(ng)
        cfg.ng_pass = int(ng if ng_pass is None else ng_pass)
        cfg.device = int(device)
        cfg.protect = 1 if protect else 0     # flux_protection of a Roe box (vanleer_mod.f90:81)
        self.cfg = cfg
        self.shape = (int(nz), int(ny), int(nx))
        self.npass = int(npass)
        self.precision = int(precision)
        self._h = ctypes.c_void_p()
        check(lib().imhd_create(ctypes.byref(cfg), ctypes.byref(self._h)))
        self.dx = 1.0 / max(nx, ny, nz)

    # ------------------------------------------------------------- lifetime
    def close(self):
        if self._h:
            lib().imhd_destroy(self._h)
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

    # ------------------------------------------------------------- layout
    def padded_shape(self, nvar, g):
        nz, ny, nx = self.shape
        return (nvar, nz + 2 * g, ny + 2 * g, nx + 2 * g)

    def _as_host(self, a, nvar, g, name):
        a = np.ascontiguousarray(a, dtype=np.float64)
        if a.shape != self.padded_shape(nvar, g):
            raise ValueError(f"{name} has shape {a.shape}, expected {self.padded_shape(nvar, g)}")
        return a

    # ------------------------------------------------------------- transfer
    def upload(self, q, bface, qpass=None):
        g, gp = self.cfg.ng, self.cfg.ng_pass
        q = self._as_host(q, 7, g, "q")
        b = self._as_host(bface, 3, g, "bface")
        p = self._as_host(qpass, self.npass, gp, "qpass") if self.npass else None
        check(lib().imhd_upload(self._h, _dptr(q), _dptr(b), _dptr(p)))

    def download(self, q=None, bface=None, qpass=None):
        g, gp = self.cfg.ng, self.cfg.ng_pass
        q = np.empty(self.padded_shape(7, g)) if q is None else q
        b = np.empty(self.padded_shape(3, g)) if bface is None else bface
        p = (np.empty(self.padded_shape(self.npass, gp)) if qpass is None else qpass) if self.npass else None
        check(lib().imhd_download(self._h, _dptr(q), _dptr(b), _dptr(p)))
        return q, b, p

    def set_force(self, delv):
        d = self._as_host(delv, 3, self.cfg.ng, "delv")
        check(lib().imhd_set_force(self._h, _dptr(d)))

    # ------------------------------------------------------------- stepping
    def step(self, dt, drive_next=False):
        """One reference time step; returns the next local dt (COUR*dx/cmax)."""
        out = ctypes.c_double()
        check(lib().imhd_step(self._h, float(dt), 1 if drive_next else 0, ctypes.byref(out)))
        return out.value

    def max_speed(self):
        out = ctypes.c_double()
        check(lib().imhd_max_speed(self._h, ctypes.byref(out)))
        return out.value

    def diagnostics(self):
        out = (ctypes.c_double * 6)()
        check(lib().imhd_diagnostics(self._h, out))
        keys = ("kinetic_energy", "vrms_sq", "momx", "momy", "momz", "divB")
        return dict(zip(keys, list(out)))

    def status(self, reset=False):
        f = ctypes.c_uint()
        h = ctypes.c_longlong()
        check(lib().imhd_status(self._h, ctypes.byref(f), ctypes.byref(h), 1 if reset else 0))
        return {"flags": f.value, "floor_hits": h.value,
                "floored": bool(f.value & _lib.S_FLOOR), "nan": bool(f.value & _lib.S_NAN)}

    def wave_speeds(self):
        s = ctypes.c_double()
        d = ctypes.c_double()
        check(lib().imhd_wave_speeds(self._h, ctypes.byref(s), ctypes.byref(d)))
        return s.value, d.value

    @property
    def launch_count(self):
        return int(lib().imhd_launch_count(self._h))

    def set_stream(self, stream_handle):
        """Run on an external CUDA stream (an integer cudaStream_t, e.g.
        ``torch.cuda.current_stream().cuda_stream``); None restores the box's own."""
        check(lib().imhd_set_stream(self._h, ctypes.c_void_p(stream_handle) if stream_handle else None))

    def init_turb(self, seeds=(1234, 5678, 9123), k_max=2):
        """Seed the reference force generator (taus88) and set k_max."""
        check(lib().imhd_init_turb(self._h, int(seeds[0]), int(seeds[1]), int(seeds[2]), int(k_max)))

    def generate_force(self):
        """Next reference force field (generate_rand_force) into the box."""
        check(lib().imhd_generate_force(self._h))

    def set_geometry(self, dx, zlo, zhi):
        """Global cell size and the own z planes [zlo, zhi) of a slab."""
        check(lib().imhd_set_geometry(self._h, float(dx), int(zlo), int(zhi)))

    def pack_planes(self, z0, nplanes, out=None):
        """Planes [z0, z0+nplanes) of every state field as a flat uint8 CUDA
        tensor (field-major), for halo exchange."""
        import torch
        esz = 8 if self.cfg.precision == 64 else 4
        nbytes = (10 + self.cfg.npass) * nplanes * self.cfg.nx * self.cfg.ny * esz
        if out is None:
            out = torch.empty(nbytes, dtype=torch.uint8, device=torch.device("cuda", self.cfg.device))
        check(lib().imhd_pack_planes(self._h, int(z0), int(nplanes), ctypes.c_void_p(out.data_ptr())))
        return out

    def unpack_planes(self, z0, nplanes, src):
        check(lib().imhd_unpack_planes(self._h, int(z0), int(nplanes), ctypes.c_void_p(src.data_ptr())))

    def force_sums(self):
        """This box's forcing sums over its own planes (get_rho_turb's five
        terms before the all-reduce), as a float64 array of 5."""
        out = np.empty(5)
        check(lib().imhd_force_sums(self._h, _dptr(out)))
        return out

    def set_force_sums(self, sums):
        """All ranks' forcing sums, used by the next drive step's kick."""
        s = np.ascontiguousarray(np.asarray(sums, dtype=np.float64).reshape(5))
        check(lib().imhd_set_force_sums(self._h, _dptr(s)))

    def get_force(self):
        """The force field (3, nz+2g, ny+2g, nx+2g) in FP64."""
        g = self.cfg.ng
        out = np.empty((3, self.cfg.nz + 2 * g, self.cfg.ny + 2 * g, self.cfg.nx + 2 * g))
        check(lib().imhd_get_force(self._h, _dptr(out)))
        return out

    def turb_seeds(self):
        a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(lib().imhd_turb_seeds(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
        return a.value, b.value, c.value

    def init_uniform(self, rho=1.0, b0=(0.0, 0.0, 0.0)):
        """Density rho, zero momentum, uniform field b0, passive scalars 0."""
        b = np.ascontiguousarray(b0, dtype=np.float64)
        check(lib().imhd_init_uniform(self._h, float(rho), _dptr(b)))

    def fourier_field(self, target, kvec, amp, scale):
        """Fill from Fourier modes on the device: target "velocity" adds
        rho * scale * v to the momentum, "force" sets the force field to scale * v
        (v = sum_m 2 Re(amp_m exp(2 pi i k_m . x)), see imhd_fourier_field)."""
        kv = np.ascontiguousarray(kvec, dtype=np.int32).reshape(-1, 3)
        am = np.ascontiguousarray(amp, dtype=np.float64).reshape(-1, 6)
        check(lib().imhd_fourier_field(self._h, {"velocity": 0, "force": 1}[target],
                                       kv.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), _dptr(am), len(kv),
                                       float(scale)))

    def profile(self, enable=True):
        check(lib().imhd_profile(self._h, 1 if enable else 0))

    def stage_times(self, reset=False):
        """{stage: (total_ms, timed_steps)} accumulated since the last reset."""
        ms = (ctypes.c_double * _lib.NSTAGES)()
        cnt = (ctypes.c_longlong * _lib.NSTAGES)()
        check(lib().imhd_stage_times(self._h, ms, cnt, _lib.NSTAGES, 1 if reset else 0))
        return {name: (ms[s], cnt[s]) for s, name in enumerate(_lib.STAGES)}
