"""Batches of mixed boxes: every box of a batch ends bit for bit where the
same box ends in a batch of its own, and where it ends alone under imhd_step
with the host driver loop (FP64 bit for bit; FP32 to rounding, since the
single-box kernels are separate instantiations whose FMA contraction may
differ), with and without forcing; the device Fourier-field generator matches
the numpy OU field."""
import numpy as np
import pytest

from isothermal_mhd_b200 import Batch, Box, driver, forcing, problems
from isothermal_mhd_b200.batch import make_config

pytestmark = pytest.mark.gpu

# the 128 x 12 x 18 box has rows of whole 128-cell tiles: its update runs the
# bulk-copy fed kernel, in the batch (table launch) and alone
CASES = [((16, 16, 16), "roe", 1, 6), ((24, 16, 20), "hlld", 2, 4), ((12, 12, 12), "hlle", 0, 8),
         ((128, 12, 18), "roe", 1, 4)]
RECON = ["plm", "ppm", "plm", "plm"]      # a PPM box among PLM boxes


def alone(n, riemann, npass, steps, precision, ic, edot=0.0, delv=None, recon="plm"):
    with Box(n, precision=precision, riemann=riemann, recon=recon, npass=npass, cour=0.4, edot=edot,
             dt_turb=0.03) as box:
        box.upload(ic[0], ic[1], ic[2] if npass else None)
        rec = driver.run(box, t_end=1e30, maxsteps=steps + 1, forcing=(lambda: delv) if delv is not None else None,
                         dt_turb=0.03)
        q, b, p = box.download()
    return q, b, p, rec


def batch_of_one(cfg, ic, npass, steps, delv, driven):
    with Batch([cfg]) as bt:
        bt.upload(0, ic[0], ic[1], ic[2] if npass else None)
        if driven:
            bt.set_force(0, delv)
        bt.schedule(0, steps, forcing=driven)
        bt.run(steps)
        return bt.download(0)


@pytest.mark.parametrize("precision", [64, 32])
@pytest.mark.parametrize("driven", [False, True])
def test_batch_equals_each_box_alone(precision, driven):
    ics = [problems.smooth_wave_box(n, npass=np_) for n, s, np_, _ in CASES]
    edot = 1.0 if driven else 0.0
    forces = []
    for n, s, np_, _ in CASES:
        f = forcing.OUForcing(n, seed=5)
        forces.append(f.field(rms=1.0) if driven else None)
    cfgs = [make_config(n, precision=precision, riemann=s, npass=np_, cour=0.4, edot=edot, dt_turb=0.03, recon=r)
            for (n, s, np_, _), r in zip(CASES, RECON)]
    with Batch(cfgs) as bt:
        for i, (ic, (n, s, np_, st)) in enumerate(zip(ics, CASES)):
            bt.upload(i, ic[0], ic[1], ic[2] if np_ else None)
            if driven:
                bt.set_force(i, forces[i])
            bt.schedule(i, st, forcing=driven)
        bt.run(max(c[3] for c in CASES))
        drove = []
        for i, (ic, (n, s, np_, st)) in enumerate(zip(ics, CASES)):
            q, b, p = bt.download(i)
            clk = bt.clock(i)
            qa, ba, pa, rec = alone(n, s, np_, st, precision, ic, edot=edot, delv=forces[i], recon=RECON[i])
            q1, b1, p1 = batch_of_one(cfgs[i], ic, np_, st, forces[i], driven)
            assert np.array_equal(q, q1) and np.array_equal(b, b1), (i, np.max(np.abs(q - q1)))
            if np_:
                assert np.array_equal(p, p1)
            assert clk["steps"] == st and not clk["active"]
            if precision == 64:
                assert clk["t"] == rec.t
                assert np.array_equal(q, qa) and np.array_equal(b, ba), (i, np.max(np.abs(q - qa)))
                if np_:
                    assert np.array_equal(p, pa)
            else:
                assert abs(clk["t"] - rec.t) <= 1e-5 * rec.t
                for u, v in ((q, qa), (b, ba)) + (((p, pa),) if np_ else ()):
                    assert np.max(np.abs(u - v)) <= 1e-5 * np.max(np.abs(v)), i
            drove.append(len(rec.drive_steps) > 0)
    if driven:
        # the 24x16x20 box ends before its first drive time; the others drive
        assert sum(drove) >= 2, drove


def test_device_fourier_field_matches_numpy_ou_field():
    n = 16
    f = forcing.OUForcing(n, seed=9)
    ref = f.field(rms=2.0)
    q, b, p = problems.uniform_box(n, rho=1.0, b0=(0.5, 0, 0), npass=0)
    with Box(n, precision=64, riemann="roe", npass=0) as box:
        box.upload(q, b)
        kv, amp, scale = f.device_modes(rms=2.0)
        box.fourier_field("velocity", kv, amp, scale)
        qg, _, _ = box.download()
    np.testing.assert_allclose(qg[1:4], ref, rtol=0, atol=1e-12 * np.max(np.abs(ref)))


def test_schedule_without_dt0_uses_cfl_of_the_state():
    n = 16
    ic = problems.smooth_wave_box(n, npass=0)
    with Box(n, precision=64, riemann="roe", npass=0, cour=0.4) as box:
        box.upload(ic[0], ic[1])
        dt_expect = 0.4 * box.dx / box.max_speed()
    with Batch([make_config(n, precision=64, riemann="roe", npass=0, cour=0.4)]) as bt:
        bt.upload(0, ic[0], ic[1])
        bt.schedule(0, 3, dt0=0.0)
        assert bt.clock(0)["dt"] == dt_expect


@pytest.mark.parametrize("precision", [64, 32])
def test_init_uniform_equals_uploaded_uniform_state(precision):
    n = (12, 10, 8)
    b0 = (0.3, -0.2, 0.7)
    q, b, p = problems.uniform_box(n, rho=1.5, b0=b0, npass=2)
    p[...] = 0.0
    with Box(n, precision=precision, riemann="hlld", npass=2) as box:
        box.init_uniform(1.5, b0)
        qg, bg, pg = box.download()
    np.testing.assert_array_equal(qg, q.astype(np.float32) if precision == 32 else q)
    np.testing.assert_array_equal(bg, b.astype(np.float32) if precision == 32 else b)
    np.testing.assert_array_equal(pg, p)
    with Batch([make_config(16, precision=precision, npass=0), make_config(n, precision=precision, npass=2)]) as bt:
        bt.init_uniform(1, 1.5, b0)
        qb, bb, pb = bt.download(1)
    np.testing.assert_array_equal(qb, qg)
    np.testing.assert_array_equal(bb, bg)
    np.testing.assert_array_equal(pb, pg)


@pytest.mark.parametrize("precision", [64, 32])
def test_online_tuning_changes_no_bits(precision):
    # the tuner times eight decomposition settings on the first eight steps;
    # the result equals the untuned run bit for bit
    cases = [((32, 24, 40), "roe", 2, "plm"), ((48, 32, 32), "hlld", 0, "ppm"), ((20, 20, 20), "hlle", 1, "plm"),
             ((128, 12, 16), "roe", 1, "plm"), ((64, 10, 16), "hlld", 1, "plm")]
    out = []
    for tune in (True, False):
        cfgs = [make_config(n, precision=precision, riemann=s, npass=np_, cour=0.4, recon=r) for n, s, np_, r in cases]
        with Batch(cfgs) as bt:
            bt.tuning(tune)
            for i, (n, s, np_, r) in enumerate(cases):
                ic = problems.smooth_wave_box(n, npass=np_)
                bt.upload(i, ic[0], ic[1], ic[2] if np_ else None)
                bt.schedule(i, 12)
            bt.run(12)
            st = bt.tuning()
            assert st["done"] == tune
            out.append([bt.download(i) for i in range(len(cases))])
    for a, b in zip(out[0], out[1]):
        for u, v in zip(a, b):
            if u is not None:
                np.testing.assert_array_equal(u, v)
