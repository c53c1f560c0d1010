"""Checks of the FP64 oracle itself (CPU only).

The reference ships no golden vectors and cannot be compiled here, so the
oracle is pinned to the invariants its test problems rely on
(3D_MPI/src/init_domain_mod.f90 and driver.f90:492-553) and to the committed
golden digests of tests/golden/ (made by tests/golden/make_golden.py).
"""
import json
import os

import numpy as np
import pytest

from helpers import oracle_run
from isothermal_mhd_b200 import problems
from oracle.pyoracle import Oracle

SOLVERS = ["roe", "hlld", "hlle"]
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("riemann", SOLVERS)
@pytest.mark.parametrize("recon", ["plm", "ppm", "plm-prim", "ppm-prim"])
def test_uniform_state_is_exactly_stationary(riemann, recon):
    n = 12
    q, b, p = problems.uniform_box(n, rho=1.7, v=(0.3, -0.2, 0.1), b0=(0.6, -0.4, 0.2), npass=1, pass_value=0.3)
    o = Oracle(n, riemann=riemann, recon=recon, npass=1)
    o.set_state(q, b, p)
    dt = 1e-3
    for _ in range(3):
        o.step(dt)
    q1, b1, p1 = o.get_state()
    assert np.array_equal(q1, q) and np.array_equal(b1, b) and np.array_equal(p1, p)


@pytest.mark.parametrize("riemann", SOLVERS)
@pytest.mark.parametrize("recon", ["plm", "plm-prim", "ppm-prim"])
def test_conservation_and_divb(riemann, recon):
    n = 16
    ic = problems.smooth_wave_box(n, npass=1)
    q0 = ic[0]
    r = oracle_run(ic, n, riemann, steps=8, recon=recon)
    for v in range(4):   # mass and momentum: telescoping flux sums on a periodic box
        s0, s1 = q0[v].sum(), r["q"][v].sum()
        assert abs(s1 - s0) <= 1e-12 * max(1.0, np.abs(q0[v]).sum()), (v, s0, s1)
    bx, by, bz = r["b"]
    div = (bx - np.roll(bx, 1, 2)) + (by - np.roll(by, 1, 1)) + (bz - np.roll(bz, 1, 0))
    assert np.max(np.abs(div)) < 1e-13
    # the cell-centred field stays the face average
    np.testing.assert_array_equal(r["q"][4:7], problems.cell_centred_b(r["b"]))


def _profile(r, axis):
    """1D profiles along the normal of a planar run, in the rotated frame
    (rho, m_n, m_t1, m_t2, Bc_n, Bc_t1, Bc_t2, Bf_n, Bf_t1, Bf_t2, s)."""
    sl = [0, 0, 0]
    sl[2 - axis] = slice(None)          # arrays are [k, j, i]
    sl = tuple(sl)
    rot = [axis, (axis + 1) % 3, (axis + 2) % 3]
    q, b = r["q"], r["b"]
    rows = [q[0][sl]] + [q[1 + c][sl] for c in rot] + [q[4 + c][sl] for c in rot] + [b[c][sl] for c in rot]
    rows.append(r["p"][0][sl])
    return np.array(rows)


@pytest.mark.parametrize("riemann,recon", [(r, "plm") for r in SOLVERS] + [("roe", "plm-prim"), ("hlld", "ppm-prim")])
def test_cyclic_direction_symmetry(riemann, recon):
    # the three sweeps differ only by a cyclic permutation of the components,
    # so a planar problem along x, y or z gives the same numbers permuted, up
    # to round-off: the corner-EMF averages add their four face values in an
    # order that is not cyclic (Ez: x-faces then y-faces; Ey: x-faces then
    # z-faces; vanleer_mod.f90:1949-1951, 2013-2015, 2067-2069)
    n = 12
    res = [oracle_run(problems.shock_tube(n, axis=a, npass=1), n, riemann, steps=5, recon=recon) for a in range(3)]
    ref = _profile(res[0], 0)
    for a in (1, 2):
        got = _profile(res[a], a)
        assert np.max(np.abs(got - ref)) <= 1e-14 * np.max(np.abs(ref)), a
        np.testing.assert_allclose(res[a]["dts"], res[0]["dts"], rtol=1e-14)
    # planarity: every transverse line of the x problem is identical
    q = res[0]["q"]
    assert np.array_equal(q, np.broadcast_to(q[:, :1, :1, :], q.shape))


def _alfven_error(n, riemann, t_end=0.25, recon="plm"):
    # travelling Alfven wave along (1,1,0): B0 = (1,0,0), dv_z = dB_z, speed |B0.k|/|k| = 1/sqrt2
    TWOPI = 2 * np.pi
    dx = 1.0 / n
    c = (np.arange(n) + 0.5) * dx
    Z, Y, X = np.meshgrid(c, c, c, indexing="ij")
    amp = 1e-3
    phase0 = TWOPI * (X + Y)
    shape = (n, n, n)
    q = np.zeros((7,) + shape)
    b = np.zeros((3,) + shape)
    q[0] = 1.0
    q[3] = amp * np.sin(phase0)
    b[0] = 1.0
    b[2] = -amp * np.sin(phase0)
    q[4:7] = problems.cell_centred_b(b)
    o = Oracle(n, riemann=riemann, recon=recon, npass=0, nthreads=4)
    o.set_state(q, b, None)
    t, dt = 0.0, 0.3 * dx
    while t < t_end - 1e-14:
        dt = min(dt, t_end - t)
        o.step(dt)
        t += dt
    q1, _, _ = o.get_state()
    o.close()
    # dv = -dB/sqrt(rho) travels along +B0: x -> x - v_A t along x, i.e. phase shift 2 pi v_A t
    exact = amp * np.sin(phase0 - TWOPI * 1.0 * t)
    return np.mean(np.abs(q1[3] - exact)) / amp


@pytest.mark.parametrize("riemann,recon", [("roe", "plm"), ("hlld", "plm"), ("roe", "plm-prim"), ("hlld", "ppm-prim")])
def test_alfven_wave_converges_second_order(riemann, recon):
    e16 = _alfven_error(16, riemann, recon=recon)
    e32 = _alfven_error(32, riemann, recon=recon)
    assert e32 < 0.5 * e16, (e16, e32)
    assert e32 < 0.05


def test_taus88_and_reference_force_field():
    n = 16
    o = Oracle(n, riemann="roe", npass=0)
    f1 = o.generate_ref_force(seeds=(1234, 5678, 9123))
    f2 = o.generate_ref_force(seeds=(1234, 5678, 9123))
    f3 = o.generate_ref_force(init=False)
    o.close()
    assert np.array_equal(f1, f2)
    assert not np.array_equal(f1, f3)
    assert np.all(np.isfinite(f1)) and np.max(np.abs(f1)) > 0
    # the k = 0 mode carries no power, so the field has no mean
    assert np.max(np.abs(f1.mean(axis=(1, 2, 3)))) < 1e-12 * np.max(np.abs(f1))


def test_forcing_kick_injects_edot_dt_turb():
    n = 16
    q, b, p = problems.uniform_box(n, rho=1.0, v=(0, 0, 0), b0=(0.5, 0, 0), npass=0)
    o = Oracle(n, riemann="hlld", npass=0)
    o.set_state(q, b, None)
    delv = o.generate_ref_force(seeds=(1234, 5678, 9123))
    o.set_force(delv, edot=1e-3, dt_turb=0.05)
    ke0 = o.diagnostics()[0]
    o.step(1e-6, drive=True)
    ke1 = o.diagnostics()[0]
    # from rest the quadratic gives exactly E dot * dt_turb up to the tiny MHD step
    assert abs((ke1 - ke0) - 1e-3 * 0.05) < 1e-3 * 1e-3 * 0.05
    assert o.delv_max > 0


def test_golden_digests():
    path = os.path.join(GOLDEN, "oracle_digests.json")
    with open(path) as f:
        gold = json.load(f)
    import sys
    sys.path.insert(0, GOLDEN)
    import make_golden
    for case in gold["cases"]:
        if case["cells"] > 40 ** 3:
            continue    # the 64^3 case is checked against the GPU only
        got = make_golden.run_case(case)
        assert got["sha256"] == case["sha256"], case["name"]
        assert got["dts"] == case["dts"], case["name"]


def test_flux_protection_restatement():
    # flux_protection (vanleer_mod.f90:81, 2086-2202), restated for the Roe
    # solver: a uniform state stays uniform; a smooth run conserves mass and
    # momentum and keeps div B at round-off while its dt sees the HLLE speeds
    # too (:2962); on a strong rarefaction the bad cells take the HLLE fluxes
    # and are updated again instead of floored
    n = 12
    q, b, p = problems.uniform_box(n, rho=1.2, v=(0.3, -0.2, 0.1), b0=(0.6, -0.4, 0.2), npass=0)
    o = Oracle(n, riemann="roe", npass=0, protect=True)
    o.set_state(q, b, None)
    for _ in range(3):
        o.step(1e-3)
    q1, b1, _ = o.get_state()
    assert np.array_equal(q1, q) and np.array_equal(b1, b)
    o.close()

    n = 16
    ic = problems.smooth_wave_box(n, npass=0)
    runs = {}
    for prot in (False, True):
        o = Oracle(n, riemann="roe", npass=0, protect=prot)
        o.set_state(ic[0], ic[1], None)
        dt, smax = 1e-15, []
        for _ in range(4):
            dt = 0.4 * o.dx / o.step(dt)
            smax.append(o.smax)
        runs[prot] = (o.get_state(), smax, o.prot_cells)
        o.close()
    (qp, bp, _), smax_p, cells = runs[True]
    assert cells == 0 and all(a >= b for a, b in zip(smax_p, runs[False][1]))
    for v in range(4):
        assert abs(qp[v].sum() - ic[0][v].sum()) <= 1e-12 * max(1.0, np.abs(ic[0][v]).sum())
    div = (bp[0] - np.roll(bp[0], 1, 2)) + (bp[1] - np.roll(bp[1], 1, 1)) + (bp[2] - np.roll(bp[2], 1, 0))
    assert np.max(np.abs(div)) < 1e-13

    # rho = 0.1 band with a diverging flow of speed 1.5 along x
    q = np.zeros((7, n, n, n))
    b = np.zeros((3, n, n, n))
    x = (np.arange(n) + 0.5) / n
    q[0] = np.where(np.abs(x - 0.5) < 0.07, 0.1, 1.0)[None, None, :]
    q[1] = q[0] * np.where(x < 0.5, -1.5, 1.5)[None, None, :]
    b[0] = q[4] = 0.3
    o = Oracle(n, riemann="roe", npass=0, protect=True)
    o.set_state(q, b, None)
    dt = 0.4 * o.dx / o.max_speed()
    for _ in range(3):
        cm = o.step(dt)
        if o.prot_cells:
            break
        dt = 0.4 * o.dx / cm
    assert o.prot_cells > 0 and o.floor_hits == 0
    o.close()
