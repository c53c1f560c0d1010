"""imhd_step_static: the step for callers that cannot allocate device memory.

Such callers (a host whose device buffers all come from its own pool or from
an OpenACC / CUDA Fortran runtime, an allocation-free real-time loop) hand the
library their own input and output state buffers; the step's work arrays come
from a fixed 48 MiB file-scope device array instead of cudaMalloc.  These
tests call the entry point through the C ABI on two steps in a row and
compare each step with the allocating entry point (imhd_create / imhd_step)
on the same input: bit for bit in FP64 (the FP64 parity tolerance) and within
relative L1 1e-5 in FP32.  The largest accepted box (64^3 FP64 with two
passive scalars, which also takes the bulk-copy fed update) is compared bit
for bit, one more scalar must be refused, and a non-finite state must come
back as IMHD_E_PHYSICS.  The file sorts last so that a run stopping at the
first failure has run every other test before it.
"""
import ctypes

import numpy as np
import pytest

from helpers import rel_l1
from isothermal_mhd_b200 import Box, problems
from isothermal_mhd_b200._lib import lib

pytestmark = pytest.mark.gpu


def _static_step(torch, precision, n, riemann, npass, cour, state_in, state_out, dt, expect=0):
    out = ctypes.c_double()
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib().imhd_step_static(precision, n, n, n, {"roe": 1, "hlld": 2, "hlle": 3}[riemann], npass, 1.0, cour,
                                ctypes.c_void_p(state_in.data_ptr()), ctypes.c_void_p(state_out.data_ptr()),
                                float(dt), ctypes.byref(out), ctypes.c_void_p(stream))
    assert rc == expect, lib().imhd_last_error()
    return out.value


def _compare_two_steps(precision, riemann, n, npass, cour=0.4):
    import torch
    q, b, p = problems.smooth_wave_box(n, npass=npass)
    npdt = np.float64 if precision == 64 else np.float32
    tdt = torch.float64 if precision == 64 else torch.float32
    state = np.concatenate([q, b, p]).astype(npdt)
    dev = torch.device("cuda", 0)
    s0 = torch.from_numpy(state).to(dev)
    s1 = torch.empty_like(s0)
    s2 = torch.empty_like(s0)
    dt0 = 1e-15
    dt1 = _static_step(torch, precision, n, riemann, npass, cour, s0, s1, dt0)
    dt2 = _static_step(torch, precision, n, riemann, npass, cour, s1, s2, dt1)
    with Box(n, precision=precision, riemann=riemann, npass=npass, cour=cour) as box:
        box.upload(q, b, p)
        r1 = box.step(dt0)
        q1, b1, p1 = box.download()
        r2 = box.step(r1)
        q2, b2, p2 = box.download()
    assert tdt == s1.dtype
    for got, (qr, br, pr), dtg, dtr in ((s1, (q1, b1, p1), dt1, r1), (s2, (q2, b2, p2), dt2, r2)):
        g = got.double().cpu().numpy()
        ref = np.concatenate([qr, br, pr])
        if precision == 64:
            assert np.array_equal(g, ref)
            assert dtg == dtr
        else:
            assert np.all(rel_l1(g, ref) <= 1e-5)
            assert abs(dtg - dtr) <= 1e-5 * dtr


@pytest.mark.parametrize("precision,riemann", [(64, "roe"), (64, "hlld"), (32, "roe"), (32, "hlle")])
def test_static_step_matches_allocating_step_twice(precision, riemann):
    _compare_two_steps(precision, riemann, 16, 1)


def test_static_step_largest_accepted_box_bit_exact():
    # (21 + 2) * 64^3 * 8 B + 56 KiB = 48.29 MB of the 50.33 MB array; 64-cell
    # rows with an even row count run the bulk-copy fed update
    _compare_two_steps(64, "roe", 64, 2)


def test_static_step_rejects_one_more_scalar():
    import torch
    n = 64   # (21 + 3) * 64^3 * 8 B + 56 KiB = 50.39 MB > 48 MiB
    s = torch.zeros((13, 4, 4, 4), dtype=torch.float64, device="cuda")
    t = torch.zeros_like(s)
    out = ctypes.c_double()
    rc = lib().imhd_step_static(64, n, n, n, 1, 3, 1.0, 0.4, ctypes.c_void_p(s.data_ptr()),
                                ctypes.c_void_p(t.data_ptr()), 1e-3, ctypes.byref(out), None)
    assert rc == 1
    assert b"imhd_step_static holds" in lib().imhd_last_error()


def test_static_step_reports_non_finite_state():
    import torch
    n, npass = 16, 1
    q, b, p = problems.smooth_wave_box(n, npass=npass)
    q[0, 3, 5, 7] = np.nan
    s0 = torch.from_numpy(np.concatenate([q, b, p])).to("cuda")
    s1 = torch.empty_like(s0)
    _static_step(torch, 64, n, "roe", npass, 0.4, s0, s1, 1e-4, expect=4)
    assert b"non-finite" in lib().imhd_last_error()


def test_static_step_rejects_boxes_beyond_its_scratch():
    import torch
    n = 128   # (21 + 2) * 128^3 * 8 B = 386 MB > 48 MiB
    s = torch.zeros((12, 4, 4, 4), dtype=torch.float64, device="cuda")
    t = torch.zeros_like(s)
    out = ctypes.c_double()
    rc = lib().imhd_step_static(64, n, n, n, 1, 2, 1.0, 0.4, ctypes.c_void_p(s.data_ptr()),
                                ctypes.c_void_p(t.data_ptr()), 1e-3, ctypes.byref(out), None)
    assert rc == 1
    assert b"imhd_step_static holds" in lib().imhd_last_error()
