"""Shared helpers of the parity tests: run the same case through the FP64
oracle (CPU) and through the CUDA library (C ABI), step by step, with the
reference driver's dt rule (first dt = 1e-15, then COUR*dx/cmax with COUR
halved after a drive step)."""
from __future__ import annotations

import numpy as np

from isothermal_mhd_b200 import problems


def rel_l1(a, b):
    """Relative L1 of a against b per field (leading axis)."""
    out = []
    for x, y in zip(a, b):
        den = np.sum(np.abs(y))
        num = np.sum(np.abs(x - y))
        out.append(num / den if den > 0 else num)
    return np.array(out)


def oracle_run(ic, n, riemann, steps, cour=0.4, npass=None, dt0=1e-15, force=None, drive_at=(), edot=1e-3,
               dt_turb=0.05, nthreads=4, recon="plm"):
    from oracle.pyoracle import Oracle
    q, b, p = ic
    npass = p.shape[0] if npass is None else npass
    o = Oracle(n, riemann=riemann, recon=recon, npass=npass, nthreads=nthreads)
    o.set_state(q, b, p if npass else None)
    if force is not None:
        o.set_force(force, edot=edot, dt_turb=dt_turb)
    dts, smaxs = [], []
    dt = dt0
    for s in range(steps):
        drive = s in drive_at
        cmax = o.step(dt, drive)
        dts.append(dt)
        smaxs.append(o.smax)
        c = 0.5 * cour if drive else cour
        dt = c * o.dx / cmax
    qo, bo, po = o.get_state()
    diag = o.diagnostics()
    o.close()
    return dict(q=qo, b=bo, p=po, dts=dts, smax=smaxs, dt_next=dt, diag=diag)


def gpu_run(ic, n, riemann, steps, precision=64, cour=0.4, npass=None, dt0=1e-15, force=None, drive_at=(),
            edot=1e-3, dt_turb=0.05, dts=None, ng=0, recon="plm"):
    from isothermal_mhd_b200 import Box
    q, b, p = ic
    npass = p.shape[0] if npass is None else npass
    box = Box(n, precision=precision, riemann=riemann, recon=recon, npass=npass, cour=cour, edot=edot,
              dt_turb=dt_turb, ng=ng)
    box.upload(problems.pad(q, ng), problems.pad(b, ng), problems.pad(p, ng) if npass else None)
    if force is not None:
        box.set_force(problems.pad(force, ng))
    out_dts, smaxs = [], []
    dt = dt0
    for s in range(steps):
        if dts is not None:
            dt = dts[s]
        drive = s in drive_at
        dt_next = box.step(dt, drive)
        out_dts.append(dt)
        smaxs.append(box.wave_speeds()[0])
        dt = dt_next
    qg, bg, pg = box.download()
    diag = box.diagnostics()
    st = box.status()
    launches = box.launch_count
    box.close()
    return dict(q=problems.unpad(qg, ng), b=problems.unpad(bg, ng), p=problems.unpad(pg, ng) if npass else None,
                dts=out_dts, smax=smaxs, dt_next=dt, diag=diag, status=st, launches=launches)
