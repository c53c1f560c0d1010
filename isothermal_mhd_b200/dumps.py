"""The reference's output and restart files (io_mod.f90) for a device box,
and numpy readers for them.

Writers run through the C ABI (imhd_write_* / imhd_read_restart; the cell
records are packed on the device).  The readers here are plain numpy and
need no GPU: ``read_cells`` for the xyzcube / state-dump stream files,
``read_cut`` for the cut files, ``read_records`` / ``write_records`` for
Fortran sequential unformatted files with gfortran's record markers
(including its split of records longer than 2^31 - 9 bytes into
sub-records).
"""
from __future__ import annotations

import ctypes
import os
import struct

import numpy as np

from ._lib import check, lib

CUT_X, CUT_Y, CUT_Z, CUT_XYDIAG, CUT_YZDIAG, CUT_XYPLANE = 1, 2, 4, 8, 16, 32
MAX_SUBRECORD = 2147483639


def _dt(double_prec):
    return np.float64 if double_prec else np.float32


# ------------------------------------------------------------------ writers
def write_xyzcube(box, path, double_prec=False):
    """xyzcube stream dump (io_mod.f90:249-277): per cell q(1..7) and the
    first passive scalar."""
    check(lib().imhd_write_xyzcube(box._h, os.fsencode(path), 1 if double_prec else 0))


def write_state_dump(box, path, double_prec=False):
    """Per-rank block of the parallel dump (io_mod.f90:378-432): per cell
    q(1..7) and every passive scalar."""
    check(lib().imhd_write_state_dump(box._h, os.fsencode(path), 1 if double_prec else 0))


def write_cuts(box, directory, dump, flags=CUT_X | CUT_Y | CUT_Z | CUT_XYDIAG | CUT_YZDIAG | CUT_XYPLANE,
               double_prec=False):
    """Cut files of io_mod.f90:62-240 into `directory`."""
    check(lib().imhd_write_cuts(box._h, os.fsencode(directory), int(dump), int(flags), int(box.cfg.riemann),
                                1 if double_prec else 0))


def write_restart(box, path, t_sim, nb=6, dump_count=0, seeds=(1234, 5678, 9123)):
    """restart_mhd file (io_mod.f90:440-473)."""
    s1, s2, s3 = (int(s) for s in seeds)
    check(lib().imhd_write_restart(box._h, os.fsencode(path), float(t_sim), int(nb), int(dump_count), s1, s2, s3))


def read_restart(box, path, nb=6):
    """Load a restart file into the box; returns (t_sim, dump_count, seeds)."""
    t = ctypes.c_double()
    dc, s1, s2, s3 = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    check(lib().imhd_read_restart(box._h, os.fsencode(path), int(nb), ctypes.byref(t), ctypes.byref(dc),
                                  ctypes.byref(s1), ctypes.byref(s2), ctypes.byref(s3)))
    return t.value, dc.value, (s1.value, s2.value, s3.value)


# ------------------------------------------------------------------ readers
def read_cells(path, n, nvar, double_prec=False):
    """Cell-record stream file -> array (nvar, nz, ny, nx)."""
    nx, ny, nz = (n, n, n) if np.isscalar(n) else tuple(n)
    a = np.fromfile(path, dtype=_dt(double_prec))
    return np.ascontiguousarray(a.reshape(nz, ny, nx, nvar).transpose(3, 0, 1, 2))


def read_cut(path, double_prec=False):
    """Cut file -> array (ncell, 7): rho, v (or rotated), B."""
    return np.fromfile(path, dtype=_dt(double_prec)).reshape(-1, 7)


def write_records(path, records, max_sub=MAX_SUBRECORD):
    """Fortran sequential unformatted file of the given byte strings, with
    gfortran's markers: a record longer than max_sub bytes is split into
    sub-records; a head marker is negative when another sub-record follows,
    a tail marker negative when one precedes."""
    with open(path, "wb") as f:
        for rec in records:
            rec = bytes(rec)
            pos, first = 0, True
            while True:
                n = min(len(rec) - pos, max_sub)
                more = pos + n < len(rec)
                f.write(struct.pack("<i", -n if more else n))
                f.write(rec[pos:pos + n])
                f.write(struct.pack("<i", n if first else -n))
                pos += n
                first = False
                if not more:
                    break


def read_records(path):
    """List of the records (bytes) of a Fortran sequential unformatted file."""
    out = []
    with open(path, "rb") as f:
        while True:
            h = f.read(4)
            if not h:
                break
            parts = []
            while True:
                (m,) = struct.unpack("<i", h)
                n = abs(m)
                parts.append(f.read(n))
                (tm,) = struct.unpack("<i", f.read(4))
                if abs(tm) != n:
                    raise ValueError("inconsistent record markers in %s" % path)
                if m >= 0:
                    break
                h = f.read(4)
            out.append(b"".join(parts))
    return out


def parse_restart(path, n, npass, nb=6):
    """Restart file -> dict(t, q (7, P..), bface (3, P..), qpass, dump_count,
    seeds), arrays padded with ghost width nb (nb - 2 for qpass), Fortran
    order (i fastest)."""
    nx, ny, nz = (n, n, n) if np.isscalar(n) else tuple(n)
    recs = read_records(path)
    shp = (nz + 2 * nb, ny + 2 * nb, nx + 2 * nb)
    nbp = nb - 2
    shp_p = (nz + 2 * nbp, ny + 2 * nbp, nx + 2 * nbp)
    r = iter(recs)
    out = {"t": struct.unpack("<d", next(r))[0]}
    out["q"] = np.frombuffer(next(r), dtype=np.float64).reshape((7,) + shp)
    out["bface"] = np.frombuffer(next(r), dtype=np.float64).reshape((3,) + shp)
    out["qpass"] = np.frombuffer(next(r), dtype=np.float64).reshape((npass,) + shp_p) if npass else None
    out["dump_count"] = struct.unpack("<i", next(r))[0]
    out["seeds"] = tuple(struct.unpack("<i", next(r))[0] for _ in range(3))
    return out
