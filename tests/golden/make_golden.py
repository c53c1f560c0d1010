"""Generate tests/golden/oracle_digests.json: SHA-256 digests (plus norms and
the dt sequence) of the FP64 oracle's state after N reference steps for a set
of cases.  The CUDA FP64 path must reproduce the same digests bit for bit.

    python tests/golden/make_golden.py [--threads 8]

The digest hashes the little-endian float64 bytes of q (7 fields), bface (3)
and qpass (npass), unpadded, x fastest, after x + 0.0 (so that a signed zero
hashes like an unsigned one).  Deterministic inputs only: no seeds.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (ROOT, os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)

from isothermal_mhd_b200 import problems  # noqa: E402

CASES = [
    dict(name="smooth16_roe", ic="smooth", n=[16, 16, 16], riemann="roe", steps=6, npass=1, cour=0.4),
    dict(name="smooth16_hlld", ic="smooth", n=[16, 16, 16], riemann="hlld", steps=6, npass=1, cour=0.4),
    dict(name="smooth16_hlle", ic="smooth", n=[16, 16, 16], riemann="hlle", steps=6, npass=1, cour=0.4),
    dict(name="shockx16_roe", ic="shock_x", n=[16, 16, 16], riemann="roe", steps=8, npass=1, cour=0.4),
    dict(name="smooth_noncubic_hlld", ic="smooth", n=[24, 16, 20], riemann="hlld", steps=4, npass=2, cour=0.4),
    # the 64^3 parity configuration: FP64 Roe + CT, COUR 0.4, 100 steps, one passive scalar
    dict(name="c1_smooth64_roe_100", ic="smooth", n=[64, 64, 64], riemann="roe", steps=100, npass=1, cour=0.4),
]


def make_ic(case):
    n = tuple(case["n"])
    if case["ic"] == "smooth":
        return problems.smooth_wave_box(n, npass=case["npass"])
    if case["ic"] == "shock_x":
        return problems.shock_tube(n, axis=0, npass=case["npass"])
    raise ValueError(case["ic"])


def digest(q, b, p):
    h = hashlib.sha256()
    for a in (q, b) + ((p,) if p is not None and len(p) else ()):
        h.update(np.ascontiguousarray(np.asarray(a, dtype="<f8") + 0.0).tobytes())
    return h.hexdigest()


def run_case(case, threads=4):
    from helpers import oracle_run
    ic = make_ic(case)
    n = tuple(case["n"])
    r = oracle_run(ic, n, case["riemann"], case["steps"], cour=case["cour"], npass=case["npass"], nthreads=threads)
    return dict(sha256=digest(r["q"], r["b"], r["p"]), dts=[float(x) for x in r["dts"]],
                dt_next=float(r["dt_next"]),
                l1=[float(np.sum(np.abs(a))) for a in list(r["q"]) + list(r["b"]) + (list(r["p"]) if r["p"] is not None else [])],
                diag=[float(x) for x in r["diag"]])


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 4)
    a = ap.parse_args(argv)
    out = {"format": "sha256 of float64 LE bytes of (q, bface, qpass) after x + 0.0", "cases": []}
    for case in CASES:
        r = run_case(case, threads=a.threads)
        c = dict(case)
        c["cells"] = int(np.prod(case["n"]))
        c.update(r)
        out["cases"].append(c)
        print(case["name"], r["sha256"][:16], "dt_next", r["dt_next"], flush=True)
    with open(os.path.join(HERE, "oracle_digests.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
