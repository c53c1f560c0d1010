"""Flux protection (flux_protection, vanleer_mod.f90:81, 2086-2202; off in
the reference) on the GPU against the FP64 oracle: HLLE fluxes of the same
interface states beside the Roe fluxes (their wave speeds enter smax), and
after each update the cells whose density fell below 1e-20 and their six
neighbours updated again with the HLLE fluxes on the bad cells' faces and the
HLLE corner EMFs.  FP64 bit for bit, every dt included, on a smooth run (no
bad cells), on a strong rarefaction along each axis (two planes of bad cells
every step from the third on), with PPM and primitive reconstruction, and as
one box of a batch."""
import ctypes

import numpy as np
import pytest

from helpers import oracle_run, rel_l1
from isothermal_mhd_b200 import problems

pytestmark = pytest.mark.gpu


def rarefaction(n, axis, rho_lo=0.05, v=1.5, bx=0.3, by=0.2, width=0.07):
    """A band of density rho_lo between two streams leaving it at speed v."""
    nx, ny, nz = n
    shape = (nz, ny, nx)
    q = np.zeros((7,) + shape)
    b = np.zeros((3,) + shape)
    L = n[axis]
    x = (np.arange(L) + 0.5) / L
    sh = [1, 1, 1]
    sh[2 - axis] = L
    q[0] = np.broadcast_to(np.where(np.abs(x - 0.5) < width, rho_lo, 1.0).reshape(sh), shape)
    q[1 + axis] = q[0] * np.broadcast_to(np.where(x < 0.5, -v, v).reshape(sh), shape)
    b[axis] = q[4 + axis] = bx
    b[(axis + 1) % 3] = q[4 + (axis + 1) % 3] = by
    return q, b, np.zeros((0,) + shape)


def run_pair(ic, n, steps, recon="plm", npass=0, precision=64):
    from oracle.pyoracle import Oracle
    from isothermal_mhd_b200 import Box
    q, b, p = ic
    o = Oracle(n, riemann="roe", recon=recon, npass=npass, protect=True, nthreads=4)
    o.set_state(q, b, p if npass else None)
    dt = 0.4 * o.dx / o.max_speed()
    dts, cells = [], []
    for _ in range(steps):
        dts.append(dt)
        dt = 0.4 * o.dx / o.step(dt)
        cells.append(o.prot_cells)
    ref = o.get_state() + (dt, o.smax)
    o.close()
    with Box(n, precision=precision, riemann="roe", recon=recon, npass=npass, cour=0.4, protect=True) as box:
        box.upload(q, b, p if npass else None)
        gdt = []
        g = dts[0]
        for s in range(steps):
            gdt.append(g)
            g = box.step(dts[s] if precision == 32 else g)
        got = box.download() + (g, box.wave_speeds()[0])
        st = box.status()
    return ref, got, dts, gdt, cells, st


@pytest.mark.parametrize("recon", ["plm", "ppm", "plm-prim"])
def test_protected_smooth_run_bit_exact(recon):
    n = (16, 20, 12)
    ref, got, dts, gdt, cells, _ = run_pair(problems.smooth_wave_box(n, npass=1), n, 5, recon=recon, npass=1)
    assert cells[-1] == 0
    for a, b in zip(got[:3], ref[:3]):
        assert np.array_equal(a, b)
    assert gdt == dts and got[3] == ref[3] and got[4] == ref[4]


@pytest.mark.parametrize("axis", [0, 1, 2])
def test_protected_rarefaction_bit_exact(axis):
    n = (16, 16, 16)
    ref, got, dts, gdt, cells, st = run_pair(rarefaction(n, axis), n, 5)
    assert cells[-1] > 0, "the case must exercise the protected update"
    assert np.all(np.isfinite(ref[0]))
    for a, b in zip(got[:2], ref[:2]):
        assert np.array_equal(a, b), np.max(np.abs(a - b))
    assert gdt == dts and got[3] == ref[3]
    assert st["floor_hits"] == 0


def test_protected_rarefaction_ppm_prim_bit_exact():
    n = (16, 16, 16)
    ref, got, dts, gdt, cells, _ = run_pair(rarefaction(n, 0), n, 4, recon="ppm-prim")
    for a, b in zip(got[:2], ref[:2]):
        assert np.array_equal(a, b), np.max(np.abs(a - b))
    assert gdt == dts


def test_protected_fp32_smooth_within_1e5():
    n = 24
    ref, got, _, _, _, _ = run_pair(problems.smooth_wave_box(n, npass=1), n, 10, npass=1, precision=32)
    for a, b in zip(got[:3], ref[:3]):
        assert np.all(rel_l1(a, b) <= 1e-5)


def test_protected_box_in_a_batch_equals_it_alone():
    from isothermal_mhd_b200 import Batch, Box
    from isothermal_mhd_b200.batch import make_config
    n = (16, 16, 16)
    ic = rarefaction(n, 1)
    steps = 5
    cfgs = [make_config(n, precision=64, riemann="roe", npass=0, cour=0.4, protect=True),
            make_config(n, precision=64, riemann="hlld", npass=0, cour=0.4),
            make_config((16, 12, 20), precision=64, riemann="roe", npass=1, cour=0.4)]
    other = problems.smooth_wave_box((16, 12, 20), npass=1)
    with Batch(cfgs) as bt:
        bt.upload(0, ic[0], ic[1])
        bt.upload(1, ic[0], ic[1])
        bt.upload(2, *other)
        for i in range(3):
            bt.schedule(i, steps)
        bt.run(steps)
        qb, bb, _ = bt.download(0)
    with Box(n, precision=64, riemann="roe", npass=0, cour=0.4, protect=True) as box:
        box.upload(ic[0], ic[1])
        dt = 1e-15
        for _ in range(steps):
            dt = box.step(dt)
        qa, ba, _ = box.download()
    assert np.array_equal(qb, qa) and np.array_equal(bb, ba)


def test_protect_needs_the_roe_solver():
    from isothermal_mhd_b200 import Box, ImhdError
    with pytest.raises(ImhdError) as ei:
        Box(16, precision=64, riemann="hlld", protect=True)
    assert "IMHD_E_ARG" in str(ei.value)
