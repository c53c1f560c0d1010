"""The tiled corner-EMF kernel (single boxes whose rows are whole 32-cell
segments and whose y edge is a multiple of 8: cell-centre EMFs and velocities
computed once per cell into a shared-memory ring) against the FP64 oracle's
compute_cell_corner_emf_3d (vanleer_mod.f90:1823-2076): bit for bit in FP64
on non-cubic boxes whose z edge leaves a partial plane segment, with the
periodic wrap in x and y inside one tile row, for the three solvers and the
reconstructions; the protection EMFs (flux_protection, :2086-2202) on a
rarefaction; a driven run; FP32 within 1e-5."""
import numpy as np
import pytest

from helpers import gpu_run, oracle_run, rel_l1
from isothermal_mhd_b200 import problems

pytestmark = pytest.mark.gpu


def assert_exact(g, o):
    for name in ("q", "b"):
        assert np.array_equal(g[name], o[name]), (name, np.max(np.abs(g[name] - o[name])))
    if o["p"] is not None:
        assert np.array_equal(g["p"], o["p"]), ("p", np.max(np.abs(g["p"] - o["p"])))
    assert g["dts"] == o["dts"]
    assert g["smax"] == o["smax"]
    assert g["dt_next"] == o["dt_next"]


@pytest.mark.parametrize("n,riemann,recon", [
    ((64, 24, 40), "roe", "plm"),        # two tiles across x, three tile rows, segments of 32 + 8 planes
    ((32, 8, 33), "hlld", "ppm"),        # one tile: both wraps inside it, a one-plane segment
    ((96, 16, 20), "hlle", "plm-prim"),  # three tiles across x, fewer planes than a segment
])
def test_fp64_tiled_emf_bit_exact(n, riemann, recon):
    ic = problems.smooth_wave_box(n, npass=1)
    o = oracle_run(ic, n, riemann, steps=4, recon=recon, nthreads=8)
    g = gpu_run(ic, n, riemann, steps=4, recon=recon)
    assert_exact(g, o)


@pytest.mark.parametrize("axis", [0, 1, 2])
def test_fp64_tiled_emf_shock(axis):
    n = (32, 32, 32)
    ic = problems.shock_tube(n, axis=axis, npass=1)
    o = oracle_run(ic, n, "roe", steps=6, nthreads=8)
    g = gpu_run(ic, n, "roe", steps=6)
    assert_exact(g, o)


@pytest.mark.parametrize("axis", [0, 1])
def test_fp64_tiled_protection_emf_bit_exact(axis):
    from test_gpu_protect import rarefaction, run_pair
    n = (32, 16, 16)
    ref, got, dts, gdt, cells, st = run_pair(rarefaction(n, axis), n, 5)
    assert cells[-1] > 0, "the case must exercise the protected update"
    for a, b in zip(got[:2], ref[:2]):
        assert np.array_equal(a, b), np.max(np.abs(a - b))
    assert gdt == dts and got[3] == ref[3]


def test_fp64_tiled_emf_driven():
    from oracle.pyoracle import Oracle
    n = (32, 16, 24)
    ic = problems.smooth_wave_box(n, npass=2)
    gen = Oracle(n, riemann="hlld", npass=2)
    delv = gen.generate_ref_force(seeds=(1234, 5678, 9123))
    gen.close()
    o = oracle_run(ic, n, "hlld", steps=4, force=delv, drive_at=(1,), edot=1.0, nthreads=8)
    g = gpu_run(ic, n, "hlld", steps=4, force=delv, drive_at=(1,), edot=1.0, dts=o["dts"])
    for name in ("q", "b", "p"):
        err = rel_l1(g[name], o[name])
        assert np.all(err <= 1e-12), (name, err)


def test_fp32_tiled_emf_within_1e5():
    n = (64, 32, 24)
    ic = problems.smooth_wave_box(n, npass=1)
    o = oracle_run(ic, n, "roe", steps=10, nthreads=8)
    g = gpu_run(ic, n, "roe", steps=10, precision=32, dts=o["dts"])
    for name in ("q", "b", "p"):
        err = rel_l1(g[name], o[name])
        assert np.all(err <= 1e-5), (name, err)
