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
