"""Parity on box shapes the cubic and 16-cell cases do not reach, against the
FP64 oracle, bit for bit: non-cubic boxes with 32k-cell rows whose z edge
leaves a partial segment of the z-marching kernels, for the three solvers
and the reconstructions; 0 to 5 passive scalars (scalar arrays sized 2, 4 and
8, passive_mod.f90:118-627); shocks along each axis; the protection EMFs
(flux_protection, vanleer_mod.f90:2086-2202) on a rarefaction in a 32-cell
box; a driven run (relative L1 <= 1e-12: the forcing sums reduce in another
order); FP32 within 1e-5; and a batch of such boxes beside boxes of other
shapes, each equal to its run alone."""
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
    ((64, 24, 40), "roe", "plm"),
    ((32, 16, 33), "hlld", "ppm"),       # a one-plane segment
    ((96, 16, 20), "hlle", "plm-prim"),
])
def test_fp64_noncubic_bit_exact(n, riemann, recon):
    ic = problems.smooth_wave_box(n, npass=1)
    o = oracle_run(ic, n, riemann, steps=4, recon=recon, nthreads=8)
    g = gpu_run(ic, n, riemann, steps=4, recon=recon)
    assert_exact(g, o)


@pytest.mark.parametrize("n,npass", [((32, 16, 36), 0), ((32, 16, 36), 2), ((32, 16, 36), 3), ((32, 16, 36), 5),
                                     ((128, 12, 20), 3), ((128, 12, 20), 5), ((128, 13, 16), 2)])
def test_fp64_passive_counts(n, npass):
    # 128-cell rows: the bulk-copy fed passive kernels with scalar arrays sized 4 and 8; an odd
    # row count: the corrector's blocks of one row instead of two
    q, b, p = problems.smooth_wave_box(n, npass=1)
    rng = np.random.default_rng(11)
    p = rng.uniform(0.0, 1.0, (npass,) + q.shape[1:])
    o = oracle_run((q, b, p), n, "roe", steps=4, npass=npass, nthreads=8)
    g = gpu_run((q, b, p), n, "roe", steps=4, npass=npass)
    assert_exact(g, o)


@pytest.mark.parametrize("axis", [0, 1, 2])
def test_fp64_shock_32(axis):
    n = (32, 32, 32)
    ic = problems.shock_tube(n, axis=axis, npass=1)
    o = oracle_run(ic, n, "roe", steps=6, nthreads=8)
    g = gpu_run(ic, n, "roe", steps=6)
    assert_exact(g, o)


@pytest.mark.parametrize("axis", [0, 1])
def test_fp64_protection_32_bit_exact(axis):
    from test_gpu_protect import rarefaction, run_pair
    n = (32, 16, 16)
    # the band of two cells that empties within the five steps, as at 16 cells
    ref, got, dts, gdt, cells, st = run_pair(rarefaction(n, axis, width=0.07 * 16 / n[axis]), n, 5)
    assert cells[-1] > 0, "the case must exercise the protected update"
    for a, b in zip(got[:2], ref[:2]):
        assert np.array_equal(a, b), np.max(np.abs(a - b))
    assert gdt == dts and got[3] == ref[3]


def test_fp64_driven_32():
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


def test_fp32_noncubic_within_1e5():
    n = (64, 32, 24)
    ic = problems.smooth_wave_box(n, npass=1)
    o = oracle_run(ic, n, "roe", steps=10, nthreads=8)
    g = gpu_run(ic, n, "roe", steps=10, precision=32, dts=o["dts"])
    for name in ("q", "b", "p"):
        err = rel_l1(g[name], o[name])
        assert np.all(err <= 1e-5), (name, err)


def test_batch_of_mixed_shapes_equals_each_box_alone():
    # passive counts 0..3, the four reconstructions, one protected box
    from isothermal_mhd_b200 import Batch, Box
    from isothermal_mhd_b200.batch import make_config
    from test_gpu_protect import rarefaction
    cases = [((32, 16, 24), "roe", "plm", 2, False), ((64, 8, 40), "hlld", "ppm", 0, False),
             ((16, 16, 16), "roe", "plm", 1, False), ((32, 24, 20), "hlle", "plm-prim", 3, False),
             ((48, 16, 16), "hlld", "plm", 1, False), ((32, 16, 16), "roe", "plm", 0, True)]
    steps = 4
    ics = []
    for n, r, rc, npass, prot in cases:
        if prot:
            ics.append(rarefaction(n, 0))
        else:
            q, b, _ = problems.smooth_wave_box(n, npass=1)
            p = np.random.default_rng(n[0] + n[2]).uniform(0.0, 1.0, (npass,) + q.shape[1:])
            ics.append((q, b, p))
    cfgs = [make_config(n, precision=64, riemann=r, npass=npass, cour=0.4, recon=rc, protect=prot)
            for n, r, rc, npass, prot in cases]
    with Batch(cfgs) as bt:
        for i, (q, b, p) in enumerate(ics):
            bt.upload(i, q, b, p if p.shape[0] else None)
            bt.schedule(i, steps)
        bt.run(steps)
        got = [bt.download(i) for i in range(len(cases))]
    for (n, r, rc, npass, prot), (q, b, p), (qb, bb, pb) in zip(cases, ics, got):
        with Box(n, precision=64, riemann=r, recon=rc, npass=npass, cour=0.4, protect=prot) as box:
            box.upload(q, b, p if npass else None)
            dt = 1e-15
            for _ in range(steps):
                dt = box.step(dt)
            qa, ba, pa = box.download()
        assert np.array_equal(qb, qa) and np.array_equal(bb, ba), (n, r, rc)
        if npass:
            assert np.array_equal(pb, pa), (n, r, rc, "passives")
