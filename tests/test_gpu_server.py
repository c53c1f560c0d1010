"""Serving loop (imhd_server_*): each request's result is the same alone and
in a mix of concurrently resident requests, equals the single-box path, and
admission respects the HBM budget."""
import time

import numpy as np
import pytest

from isothermal_mhd_b200 import Box, driver
from isothermal_mhd_b200.server import Server
from isothermal_mhd_b200.workloads import BoxSpec

pytestmark = pytest.mark.gpu

A = BoxSpec(n=24, b0=(0.3, -0.4, 0.5), mach=2.5, riemann="roe", npass=1, steps=12, seed=7, dt_turb=0.01)
MIX = [BoxSpec(n=16, b0=(1.0, 0.0, 0.2), mach=1.0, riemann="hlld", npass=0, steps=20, seed=3, dt_turb=0.02),
       BoxSpec(n=32, b0=(0.1, 0.7, 0.0), mach=4.0, riemann="roe", npass=2, steps=9, seed=4, dt_turb=0.01),
       A,
       BoxSpec(n=20, b0=(0.0, 0.0, 1.5), mach=0.7, riemann="hlle", npass=0, steps=15, seed=5, dt_turb=0.03),
       BoxSpec(n=28, b0=(0.5, 0.5, 0.5), mach=3.0, riemann="hlld", npass=1, steps=6, seed=6, dt_turb=0.01)]


def wait(srv, ids, timeout=120.0):
    out = {}
    t0 = time.time()
    while len(out) < len(ids):
        for rid in ids:
            if rid in out:
                continue
            state, info, arr = srv.poll(rid, fetch=True)
            if state == "done":
                out[rid] = (info, arr)
        assert time.time() - t0 < timeout, srv.stats()
        time.sleep(0.002)
    return out


@pytest.mark.parametrize("precision", [32, 64])
def test_result_alone_equals_result_in_mix(precision):
    with Server(precision=precision, hbm_budget=4e9, steps_per_round=3) as srv:
        ra = srv.submit(A)
        alone = wait(srv, [ra])[ra]
        ids = [srv.submit(s) for s in MIX]
        res = wait(srv, ids)
        st = srv.stats()
    assert st["peak_resident_boxes"] >= 2, st       # the mix really ran together
    info_mix, arr_mix = res[ids[2]]
    info_alone, arr_alone = alone
    assert info_alone["steps"] == A.steps == info_mix["steps"]
    assert info_alone["t"] == info_mix["t"]
    for u, v in zip(arr_alone, arr_mix):
        np.testing.assert_array_equal(u, v)


def test_fp64_result_equals_single_box_driver_loop():
    spec = MIX[1]
    with Server(precision=64, hbm_budget=4e9) as srv:
        rid = srv.submit(spec)
        info, (q, b, p) = wait(srv, [rid])[rid]
    kv, av, sv, af, sf = spec.fields()
    with Box(spec.n, precision=64, riemann=spec.riemann, npass=spec.npass, cour=0.4, edot=spec.edot,
             dt_turb=spec.dt_turb) as box:
        box.init_uniform(1.0, spec.b0)
        box.fourier_field("velocity", kv, av, sv)
        box.fourier_field("force", kv, af, sf)
        dt0 = 0.4 * box.dx / box.max_speed()
        rec = driver.run(box, t_end=1e30, maxsteps=spec.steps + 1, dt0=dt0, forcing="device", dt_turb=spec.dt_turb)
        qa, ba, pa = box.download()
    assert info["steps"] == rec.steps and info["t"] == rec.t
    np.testing.assert_array_equal(q, qa)
    np.testing.assert_array_equal(b, ba)
    np.testing.assert_array_equal(p, pa)


def test_budget_admits_one_box_at_a_time():
    specs = [BoxSpec(n=32, b0=(0.5, 0, 0), mach=1.0, steps=4, seed=s) for s in range(4)]
    # one 32^3 FP32 box with forcing needs about 6 MB; the budget holds one
    with Server(precision=32, hbm_budget=8e6) as srv:
        ids = [srv.submit(s) for s in specs]
        res = wait(srv, ids)
        st = srv.stats()
    assert st["peak_resident_boxes"] == 1 and st["completed"] == 4, st
    assert all(r[0]["steps"] == 4 for r in res.values())


def test_oversized_request_fails_and_others_run():
    with Server(precision=32, hbm_budget=8e6) as srv:
        big = srv.submit(BoxSpec(n=64, b0=(0.5, 0, 0), mach=1.0, steps=2, seed=1))
        small = srv.submit(BoxSpec(n=16, b0=(0.5, 0, 0), mach=1.0, steps=2, seed=2))
        res = wait(srv, [small])
        assert res[small][0]["steps"] == 2
        state, info, _ = srv.poll(big)
        assert state == "failed" and "budget" in info["error"]
