"""Primitive-variable reconstruction (compute_interface_states_prim,
vanleer_mod.f90:1144-1485; primitive_reconstruction, :84) on the GPU against
the FP64 oracle: bit for bit in FP64 (every state array, every dt and the
interface wave-speed maximum) for the three solvers with PLM and PPM, shocks
along each axis, rows long enough for the tiled x sweep, and a batch that
mixes the four reconstructions; relative L1 <= 1e-5 in FP32."""
import numpy as np
import pytest

from helpers import gpu_run, oracle_run, rel_l1
from isothermal_mhd_b200 import problems

pytestmark = pytest.mark.gpu

SOLVERS = ["roe", "hlld", "hlle"]
PRIMS = ["plm-prim", "ppm-prim"]


def assert_exact(g, o):
    for name in ("q", "b"):
        assert np.array_equal(g[name], o[name]), (name, np.max(np.abs(g[name] - o[name])))
    if o["p"] is not None:
        assert np.array_equal(g["p"], o["p"]), ("p", np.max(np.abs(g["p"] - o["p"])))
    assert g["dts"] == o["dts"]
    assert g["smax"] == o["smax"]
    assert g["dt_next"] == o["dt_next"]


@pytest.mark.parametrize("recon", PRIMS)
@pytest.mark.parametrize("riemann", SOLVERS)
def test_fp64_bit_exact_prim_noncubic(riemann, recon):
    n = (16, 20, 24)
    ic = problems.smooth_wave_box(n, npass=1)
    o = oracle_run(ic, n, riemann, steps=5, recon=recon)
    g = gpu_run(ic, n, riemann, steps=5, recon=recon)
    assert_exact(g, o)


@pytest.mark.parametrize("recon", PRIMS)
@pytest.mark.parametrize("axis", [0, 1, 2])
def test_fp64_bit_exact_prim_shock(axis, recon):
    # discontinuities: the PLM limiter without a same-sign test, and the PPM
    # constraints (an extremum flattens to the linear profile)
    n = 16
    ic = problems.shock_tube(n, axis=axis, npass=1)
    o = oracle_run(ic, n, "roe", steps=8, recon=recon)
    g = gpu_run(ic, n, "roe", steps=8, recon=recon)
    assert_exact(g, o)


@pytest.mark.parametrize("recon", PRIMS)
def test_fp64_bit_exact_prim_alfven_zero_components(recon):
    n = 16
    ic = problems.alfven_wave(n, npass=0)
    o = oracle_run(ic, n, "hlld", steps=5, npass=0, recon=recon)
    g = gpu_run(ic, n, "hlld", steps=5, npass=0, recon=recon)
    assert_exact(g, o)


@pytest.mark.parametrize("recon", ["plm", "ppm"] + PRIMS)
def test_fp64_bit_exact_long_rows_tiled_x_sweep(recon):
    # rows of more than 945 FP64 cells do not fit the x-row sweep's shared
    # memory: the 128-face tiled x sweep with a staged halo takes them
    n = (960, 12, 12)
    ic = problems.smooth_wave_box(n, npass=1)
    o = oracle_run(ic, n, "roe", steps=2, recon=recon, nthreads=8)
    g = gpu_run(ic, n, "roe", steps=2, recon=recon)
    assert_exact(g, o)


@pytest.mark.parametrize("recon", PRIMS)
def test_fp64_bit_exact_prim_tma_rows(recon):
    n = (128, 12, 18)
    ic = problems.smooth_wave_box(n, npass=2)
    o = oracle_run(ic, n, "hlld", steps=4, recon=recon, nthreads=8)
    g = gpu_run(ic, n, "hlld", steps=4, recon=recon)
    assert_exact(g, o)


@pytest.mark.parametrize("recon", PRIMS)
def test_fp32_prim_within_1e5_of_fp64_oracle(recon):
    n = 32
    ic = problems.smooth_wave_box(n, npass=1)
    o = oracle_run(ic, n, "roe", steps=20, recon=recon, nthreads=8)
    g = gpu_run(ic, n, "roe", steps=20, precision=32, recon=recon, dts=o["dts"])
    for name in ("q", "b", "p"):
        err = rel_l1(g[name], o[name])
        assert np.all(err <= 1e-5), (name, err)


def test_batch_mixing_all_reconstructions_equals_each_box_alone():
    from isothermal_mhd_b200 import Batch
    from isothermal_mhd_b200.batch import make_config
    cases = [((16, 16, 16), "roe", "plm"), ((16, 16, 16), "roe", "ppm"), ((20, 16, 12), "hlld", "plm-prim"),
             ((16, 12, 20), "hlle", "ppm-prim")]
    steps = 4
    ics = [problems.smooth_wave_box(n, npass=1) for n, _, _ in cases]
    cfgs = [make_config(n, precision=64, riemann=r, npass=1, cour=0.4, recon=rc) for n, r, rc in cases]
    with Batch(cfgs) as bt:
        for i, ic in enumerate(ics):
            bt.upload(i, *ic)
            bt.schedule(i, steps)
        bt.run(steps)
        got = [bt.download(i) for i in range(len(cases))]
    for (n, r, rc), ic, (q, b, p) in zip(cases, ics, got):
        o = oracle_run(ic, n, r, steps=steps, recon=rc)
        assert np.array_equal(q, o["q"]) and np.array_equal(b, o["b"]) and np.array_equal(p, o["p"]), (r, rc)
