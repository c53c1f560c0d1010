"""ctypes wrapper of the FP64 oracle library (test infrastructure only).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline and
reference legs import this module.  The product package never does.

The oracle restates the reference's van Leer + CT step
(3D_MPI/src/vanleer_mod.f90, passive_mod.f90, turb_driver_mod.f90,
boundary_conditions_mod.f90, driver.f90).  Parity against the reference itself
is unpinned: no Fortran compiler exists here and the reference ships no golden
vectors.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle_imhd.so")
_lib = None


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (g++, -ffp-contract=off)."""
    if force or not os.path.exists(_LIB_PATH):
        subprocess.check_call(["make", "-s", "-C", _HERE])
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        vp, d, i = ctypes.c_void_p, ctypes.c_double, ctypes.c_int
        dp = ctypes.POINTER(ctypes.c_double)
        L.oracle_create.restype = vp
        L.oracle_create.argtypes = [i, i, i, i, i, i, d, i]
        L.oracle_destroy.argtypes = [vp]
        L.oracle_set_threads.argtypes = [vp, i]
        L.oracle_set_force_params.argtypes = [vp, d, d]
        L.oracle_set_state.argtypes = [vp, dp, dp, dp]
        L.oracle_get_state.argtypes = [vp, dp, dp, dp]
        L.oracle_set_force.argtypes = [vp, dp]
        L.oracle_get_force.argtypes = [vp, dp]
        L.oracle_init_turb.argtypes = [vp, i, i, i]
        L.oracle_generate_force.argtypes = [vp]
        L.oracle_step.restype = d
        L.oracle_step.argtypes = [vp, d, i]
        for name in ("oracle_smax", "oracle_delv_max", "oracle_dx", "oracle_max_speed"):
            getattr(L, name).restype = d
            getattr(L, name).argtypes = [vp]
        L.oracle_floor_hits.restype = ctypes.c_long
        L.oracle_floor_hits.argtypes = [vp]
        L.oracle_prot_cells.restype = ctypes.c_long
        L.oracle_prot_cells.argtypes = [vp]
        L.oracle_force_error.restype = i
        L.oracle_force_error.argtypes = [vp]
        L.oracle_diagnostics.argtypes = [vp, dp]
        _lib = L
    return _lib


def _ptr(a):
    if a is None:
        return None
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


RIEMANN = {"roe": 1, "hlld": 2, "hlle": 3}
# reconstruction code of oracle_create: bit 0 PPM, bit 1 primitive variables
RECON = {"plm": 0, "ppm": 1, "plm-prim": 2, "ppm-prim": 3}


def recon_code(recon, protect=False):
    return RECON[recon] | (4 if protect else 0)


class Oracle:
    """One periodic box advanced by the CPU restatement of the reference."""

    def __init__(self, n, riemann="roe", recon="plm", npass=0, sound_speed=1.0, nthreads=1, protect=False):
        """recon: "plm" / "ppm" characteristic (the reference default) or
        "plm-prim" / "ppm-prim" primitive-variable reconstruction; protect:
        the HLLE protection fluxes of a Roe run (flux_protection)."""
        nx, ny, nz = (n, n, n) if np.isscalar(n) else n
        self.shape = (nz, ny, nx)
        self.npass = npass
        self.h = lib().oracle_create(nx, ny, nz, RIEMANN[riemann], recon_code(recon, protect),
                                     npass, float(sound_speed), int(nthreads))
        if not self.h:
            raise ValueError("oracle needs every edge >= 12 cells (nb = 6 ghost layers)")

    def close(self):
        if self.h:
            lib().oracle_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def dx(self):
        return lib().oracle_dx(self.h)

    def set_threads(self, n):
        lib().oracle_set_threads(self.h, int(n))

    def set_state(self, q, bface, qpass=None):
        q = np.ascontiguousarray(q, dtype=np.float64)
        bface = np.ascontiguousarray(bface, dtype=np.float64)
        qp = None if qpass is None or self.npass == 0 else np.ascontiguousarray(qpass, dtype=np.float64)
        lib().oracle_set_state(self.h, _ptr(q), _ptr(bface), _ptr(qp))

    def get_state(self):
        q = np.empty((7,) + self.shape)
        b = np.empty((3,) + self.shape)
        p = np.empty((self.npass,) + self.shape) if self.npass else None
        lib().oracle_get_state(self.h, _ptr(q), _ptr(b), _ptr(p))
        return q, b, p

    def set_force(self, delv, edot=None, dt_turb=None):
        delv = np.ascontiguousarray(delv, dtype=np.float64)
        lib().oracle_set_force(self.h, _ptr(delv))
        if edot is not None:
            lib().oracle_set_force_params(self.h, float(edot), float(dt_turb))

    def set_force_params(self, edot, dt_turb):
        lib().oracle_set_force_params(self.h, float(edot), float(dt_turb))

    def generate_ref_force(self, seeds=(1234, 5678, 9123), init=True):
        if init:
            lib().oracle_init_turb(self.h, *[int(s) for s in seeds])
        lib().oracle_generate_force(self.h)
        out = np.empty((3,) + self.shape)
        lib().oracle_get_force(self.h, _ptr(out))
        return out

    def step(self, dt, drive=False):
        """One reference driver step; returns cmax (dt_next = COUR*dx/cmax)."""
        return lib().oracle_step(self.h, float(dt), 1 if drive else 0)

    @property
    def smax(self):
        return lib().oracle_smax(self.h)

    @property
    def delv_max(self):
        return lib().oracle_delv_max(self.h)

    def max_speed(self):
        return lib().oracle_max_speed(self.h)

    @property
    def floor_hits(self):
        return lib().oracle_floor_hits(self.h)

    @property
    def prot_cells(self):
        """Interior cells the protection re-updated (counted per update)."""
        return lib().oracle_prot_cells(self.h)

    @property
    def force_error(self):
        return lib().oracle_force_error(self.h)

    def diagnostics(self):
        out = np.zeros(6)
        lib().oracle_diagnostics(self.h, _ptr(out))
        return out
