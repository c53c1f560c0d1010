"""Build libimhd.so (the CUDA kernels + C ABI) in-tree for sm_100a with nvcc.

    python -m isothermal_mhd_b200.build [--verbose]

The FP64 translation unit is compiled with --fmad=false so that no product is
contracted into an FMA: every FP64 operation is a separately rounded IEEE-754
operation, which is what bit parity with the FP64 oracle needs.  The FP32 unit
keeps FMA contraction and uses approximate single-precision division and
square root (its accuracy is checked against the FP64 oracle instead).
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libimhd.so")
BUILD_DIR = os.path.join(HERE, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"] + ARCH

UNITS = {
    "imhd_f64.cu": ["--fmad=false", "-prec-div=true", "-prec-sqrt=true"],
    # FP32: FMA contraction, approximate (<= 2 ulp) division and square root,
    # denormals flushed; the FP64 pieces of this unit are unaffected
    "imhd_f32.cu": ["--fmad=true", "-prec-div=false", "-prec-sqrt=false", "-ftz=true"],
    "imhd_capi.cu": [],
    "imhd_static.cu": [],
    "imhd_batch.cu": [],
    "imhd_server.cu": [],
    "imhd_io.cu": [],
}
HEADERS = ["imhd_physics.cuh", "imhd_physics_fast.cuh", "imhd_types.cuh", "imhd_table.h", "imhd_kernels.cuh", "imhd_launch.cuh"]


def nvcc() -> str:
    p = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(p):
        raise RuntimeError("nvcc not found")
    return p


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False, ptxas_verbose: bool = False) -> str:
    os.makedirs(BUILD_DIR, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(HERE, "..", "include", "imhd.h")]
    objs = []
    jobs = []
    for unit, flags in UNITS.items():
        src = os.path.join(CSRC, unit)
        obj = os.path.join(BUILD_DIR, unit.replace(".cu", ".o"))
        objs.append(obj)
        if force or ptxas_verbose or _stale(obj, [src, __file__] + hdrs):
            cmd = [nvcc()] + COMMON + flags + ["-c", src, "-o", obj]
            if ptxas_verbose:
                cmd += ["-Xptxas", "-v"]
            if verbose:
                print(" ".join(cmd), flush=True)
            jobs.append(cmd)
    if ptxas_verbose:
        for cmd in jobs:   # one at a time, so that the resource reports do not interleave
            subprocess.check_call(cmd)
    else:
        # the translation units compile in parallel (the two precisions dominate)
        procs = [subprocess.Popen(cmd) for cmd in jobs]
        failed = [cmd for cmd, p in zip(jobs, procs) if p.wait() != 0]
        if failed:
            raise subprocess.CalledProcessError(1, failed[0])
    if force or _stale(LIB, objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas", action="store_true", help="print register / spill usage (-Xptxas -v)")
    a = ap.parse_args(argv)
    print(build(verbose=a.verbose, force=a.force, ptxas_verbose=a.ptxas))


if __name__ == "__main__":
    sys.exit(main())
