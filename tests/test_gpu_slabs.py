"""One box split into z slabs with halo planes (emulated ranks on one
device): every step's dt and the final state equal the single-box run bit
for bit in FP64."""
import numpy as np
import pytest

from isothermal_mhd_b200 import Box, problems
from isothermal_mhd_b200.slabs import LocalSlabs

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("riemann,recon,npass,nranks", [("roe", "plm", 0, 2), ("hlld", "ppm", 1, 3),
                                                         ("hlle", "plm", 2, 4)])
def test_slabs_equal_single_box(riemann, recon, npass, nranks):
    n = (16, 12, 32)
    ic = problems.smooth_wave_box(n, npass=npass)
    steps = 6
    with Box(n, precision=64, riemann=riemann, recon=recon, npass=npass, cour=0.4) as box:
        box.upload(ic[0], ic[1], ic[2] if npass else None)
        dt, dts = 1e-15, []
        for _ in range(steps):
            dts.append(dt)
            dt = box.step(dt)
        q1, b1, p1 = box.download()
    with LocalSlabs(n, nranks, precision=64, riemann=riemann, recon=recon, npass=npass, cour=0.4) as sl:
        sl.upload(ic[0], ic[1], ic[2] if npass else None)
        dt, dts2 = 1e-15, []
        for _ in range(steps):
            dts2.append(dt)
            dt = sl.step(dt)
        q2, b2, p2 = sl.download()
    assert dts2 == dts
    np.testing.assert_array_equal(q2, q1)
    np.testing.assert_array_equal(b2, b1)
    if npass:
        np.testing.assert_array_equal(p2, p1)


@pytest.mark.parametrize("nranks", [2, 3])
def test_driven_slabs_match_single_box(nranks):
    # drive steps add up the slabs' forcing sums (all ranks' totals set the
    # kick); the totals are summed in another order than one box sums its
    # cells, so the states agree to FP64 rounding.  The dt after a drive step
    # is the minimum of the ranks' own dts (each from its own max(c, smax +
    # delv_max)), as in the reference's ranks, so the single box replays the
    # slabs' dt sequence.  No passive scalars: see the note in slabs.py.
    from isothermal_mhd_b200 import forcing
    n = (16, 12, 30)
    ic = problems.smooth_wave_box(n, npass=0)
    delv = forcing.OUForcing(n, seed=11).field(rms=1.0)
    drive_at = (1, 3)
    kw = dict(precision=64, riemann="roe", recon="plm", npass=0, cour=0.4, edot=1.0, dt_turb=0.05)
    with LocalSlabs(n, nranks, **kw) as sl:
        sl.upload(ic[0], ic[1], None)
        sl.set_force(delv)
        dt, dts2 = 1e-15, []
        for s in range(5):
            dts2.append(dt)
            dt = sl.step(dt, s in drive_at)
        q2, b2, p2 = sl.download()
    with Box(n, **kw) as box:
        box.upload(ic[0], ic[1], None)
        box.set_force(delv)
        dts = []
        for s in range(5):
            dts.append(box.step(dts2[s], s in drive_at))
        q1, b1, p1 = box.download()
    # before the first drive step the dts are the single box's
    assert dts[0] == dts2[1]
    # after one, no rank sees a larger speed than the whole box
    assert all(d2 >= d1 * (1 - 1e-12) for d1, d2 in zip(dts[1:4], dts2[2:5]))
    for u, v in ((q2, q1), (b2, b1)):
        for x, y in zip(u, v):
            den = np.sum(np.abs(y))
            assert np.sum(np.abs(x - y)) <= 1e-12 * den, np.sum(np.abs(x - y)) / den
