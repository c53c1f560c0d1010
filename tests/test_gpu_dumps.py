"""Output and restart files of a device box (imhd_write_* / imhd_read_restart)
against the downloaded state and the reference's layouts (io_mod.f90)."""
import numpy as np
import pytest

from isothermal_mhd_b200 import Box, dumps, problems

pytestmark = pytest.mark.gpu

N = (12, 10, 8)


def make_box(precision, npass=2):
    box = Box(N, precision=precision, riemann="roe", npass=npass, cour=0.4)
    q, b, p = problems.smooth_wave_box(N, npass=npass)
    box.upload(q, b, p)
    box.step(1e-3)
    box.step(1e-3)
    return box


@pytest.mark.parametrize("precision", [64, 32])
@pytest.mark.parametrize("double_prec", [True, False])
def test_xyzcube_and_state_dump_match_download(tmp_path, precision, double_prec):
    with make_box(precision) as box:
        q, b, p = box.download()
        dumps.write_xyzcube(box, tmp_path / "cube.dat", double_prec)
        dumps.write_state_dump(box, tmp_path / "state.dat", double_prec)
    dt = np.float64 if double_prec else np.float32
    cube = dumps.read_cells(tmp_path / "cube.dat", N, 8, double_prec)
    np.testing.assert_array_equal(cube[:7], q.astype(dt))
    np.testing.assert_array_equal(cube[7], p[0].astype(dt))       # first passive only
    st = dumps.read_cells(tmp_path / "state.dat", N, 9, double_prec)
    np.testing.assert_array_equal(st[7:], p.astype(dt))


def test_cuts_match_download(tmp_path):
    with make_box(64) as box:
        q, b, p = box.download()
        dumps.write_cuts(box, str(tmp_path), 3, double_prec=True)
    nx, ny, nz = N
    im, jm, km = nx // 2 - 1, ny // 2 - 1, nz // 2 - 1
    v = q[1:4] / q[0]
    def expect(sl):
        return np.stack([q[0][sl], v[0][sl], v[1][sl], v[2][sl], q[4][sl], q[5][sl], q[6][sl]], axis=-1)
    xc = dumps.read_cut(tmp_path / "xcut_ROE_rank=000_dump=3.dat", True)
    np.testing.assert_allclose(xc, expect((km, jm, slice(None))), rtol=1e-15, atol=0)
    zc = dumps.read_cut(tmp_path / "zcut_rank=000_dump=3.dat", True)
    np.testing.assert_allclose(zc, expect((slice(None), jm, im)), rtol=1e-15, atol=0)
    plane = dumps.read_cut(tmp_path / "xyplane_rank=000_dump=3.dat", True)
    np.testing.assert_allclose(plane, expect((km,)).reshape(-1, 7), rtol=1e-15, atol=0)
    xy = dumps.read_cut(tmp_path / "xydiagcut_rank=000_dump=3.dat", True)
    d = [(j, j) for j in range(min(nx, ny))]
    s = 1 / np.sqrt(2.0)
    rows = []
    for j, i in d:
        vx, vy, vz = v[0][km, j, i], v[1][km, j, i], v[2][km, j, i]
        bx, by, bz = q[4][km, j, i], q[5][km, j, i], q[6][km, j, i]
        rows.append([q[0][km, j, i], s * (vy + vx), s * (vy - vx), vz, s * (by + bx), s * (by - bx), bz])
    np.testing.assert_allclose(xy, np.array(rows), rtol=1e-14, atol=1e-16)


@pytest.mark.parametrize("precision", [64, 32])
def test_restart_round_trip_and_layout(tmp_path, precision):
    path = tmp_path / "restart_mhd_rank=000.dat"
    with make_box(precision) as box:
        q, b, p = box.download()
        dumps.write_restart(box, path, 0.125, nb=6, dump_count=4, seeds=(11, 22, 33))
    r = dumps.parse_restart(path, N, 2, nb=6)
    assert r["t"] == 0.125 and r["dump_count"] == 4 and r["seeds"] == (11, 22, 33)
    np.testing.assert_array_equal(r["q"], problems.pad(q, 6))
    np.testing.assert_array_equal(r["bface"], problems.pad(b, 6))
    np.testing.assert_array_equal(r["qpass"], problems.pad(p, 4))
    with Box(N, precision=precision, riemann="roe", npass=2, cour=0.4) as fresh:
        t, dc, seeds = dumps.read_restart(fresh, path, nb=6)
        q2, b2, p2 = fresh.download()
    assert (t, dc, seeds) == (0.125, 4, (11, 22, 33))
    np.testing.assert_array_equal(q2, q)
    np.testing.assert_array_equal(b2, b)
    np.testing.assert_array_equal(p2, p)


def test_restart_of_another_shape_is_refused(tmp_path):
    path = tmp_path / "r.dat"
    with make_box(64) as box:
        dumps.write_restart(box, path, 1.0)
    with Box((12, 10, 10), precision=64, riemann="roe", npass=2) as other:
        with pytest.raises(Exception, match="record sizes"):
            dumps.read_restart(other, path)
