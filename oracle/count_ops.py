"""Arithmetic of one reference step per interior cell-update, from the
op-counting build of the oracle (count_ops.cpp).  TEST INFRASTRUCTURE ONLY.

    python oracle/count_ops.py [--out oracle/op_counts.json]

The reference computes every stage over its padded arrays (nb = 6 ghost
layers, vanleer_mod.f90:279-426), so a step's tally at edge N is a cubic
polynomial in N whose leading coefficient is the work per interior cell; the
lower terms are the ghost-region work, which a periodic box does not need.
For each configuration (Riemann solver, reconstruction, passive scalars) the
undriven step after the 1e-15 warm-up step (driver.f90:249) is tallied at
several edges on the same physics (rms Mach 2 solenoidal velocity, B0 =
(0.5, 0, 0), passive scalars U[0, 1)), and the cubic's leading coefficient
is fitted by least squares.  The count covers additions and subtractions,
multiplications, divisions, square roots, comparisons (the reference's MAX /
MIN and its limiter and upwind tests), ABS and SIGN, each as one op.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

LIB = os.path.join(HERE, "libops_imhd.so")
CATEGORIES = ("add", "mul", "div", "sqrt", "cmp", "abs", "sign", "transc")
EDGES = (16, 20, 24, 28, 32)
COUR = 0.4
_lib = None


def lib():
    global _lib
    if _lib is None:
        subprocess.check_call(["make", "-s", "-C", HERE, "libops_imhd.so"])
        L = ctypes.CDLL(LIB)
        vp, d, i = ctypes.c_void_p, ctypes.c_double, ctypes.c_int
        dp = ctypes.POINTER(ctypes.c_double)
        L.ops_create.restype = vp
        L.ops_create.argtypes = [i, i, i, i, i, i, d]
        L.ops_destroy.argtypes = [vp]
        L.ops_set_state.argtypes = [vp, dp, dp, dp]
        L.ops_step.restype = d
        L.ops_step.argtypes = [vp, d, dp]
        L.ops_dx.restype = d
        L.ops_dx.argtypes = [vp]
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if a is not None else None


def tally_step(n, riemann, recon, npass, seed=20261203):
    """Tallies of the second step (after the 1e-15 warm-up) of an n^3 box."""
    from isothermal_mhd_b200 import forcing
    q, b, p = forcing.turbulent_box(n, mach=2.0, b0=(0.5, 0.0, 0.0), npass=npass, seed=seed)
    L = lib()
    code = {"plm": 0, "ppm": 1, "plm-prim": 2, "ppm-prim": 3}[recon]
    h = L.ops_create(n, n, n, {"roe": 1, "hlld": 2, "hlle": 3}[riemann], code, npass, 1.0)
    try:
        q, b = np.ascontiguousarray(q), np.ascontiguousarray(b)
        p = np.ascontiguousarray(p) if npass else None
        L.ops_set_state(h, _ptr(q), _ptr(b), _ptr(p))
        out = np.zeros(8)
        cmax = L.ops_step(h, 1e-15, _ptr(out))
        cmax = L.ops_step(h, COUR * L.ops_dx(h) / cmax, _ptr(out))
    finally:
        L.ops_destroy(h)
    return dict(zip(CATEGORIES, out.tolist()))


def per_cell(riemann, recon, npass, edges=EDGES):
    """Leading coefficient of the cubic fit of each tally over the edges, and
    the largest relative residual of the fit of the total."""
    rows = [tally_step(n, riemann, recon, npass) for n in edges]
    x = np.array(edges, dtype=np.float64)
    A = np.stack([x ** 3, x ** 2, x, np.ones_like(x)], axis=1)
    out = {}
    for c in CATEGORIES:
        y = np.array([r[c] for r in rows])
        coef, *_ = np.linalg.lstsq(A, y, rcond=None)
        out[c] = float(coef[0])
    tot = np.array([sum(r[c] for c in CATEGORIES if c != "transc") for r in rows])
    coef, *_ = np.linalg.lstsq(A, tot, rcond=None)
    resid = float(np.max(np.abs(A @ coef - tot) / tot))
    out["ops"] = float(coef[0])
    out["fit_max_rel_residual"] = resid
    out["raw_per_interior_cell_at_largest_edge"] = float(tot[-1] / edges[-1] ** 3)
    return out


CONFIGS = [(r, rc, npass) for r in ("roe", "hlld", "hlle") for rc in ("plm", "ppm") for npass in (0, 2, 4)]


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "op_counts.json"))
    a = ap.parse_args(argv)
    table = {"edges": list(EDGES), "categories": list(CATEGORIES),
             "physics": "rms Mach 2 solenoidal velocity, B0 = (0.5, 0, 0), passives U[0,1), undriven step",
             "configs": {}}
    for r, rc, npass in CONFIGS:
        key = f"{r}-{rc}-np{npass}"
        table["configs"][key] = per_cell(r, rc, npass)
        print(key, "%.0f ops / cell-update" % table["configs"][key]["ops"],
              "(fit residual %.1e)" % table["configs"][key]["fit_max_rel_residual"], flush=True)
    with open(a.out, "w") as f:
        json.dump(table, f, indent=1)


if __name__ == "__main__":
    main()
