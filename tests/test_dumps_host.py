"""Fortran sequential unformatted records as gfortran writes them (restart
files, io_mod.f90:440-517): markers, sub-record split, round trip."""
import struct

import numpy as np

from isothermal_mhd_b200 import dumps


def test_record_layout_matches_gfortran_markers(tmp_path):
    p = tmp_path / "r.dat"
    dumps.write_records(p, [struct.pack("<d", 1.5), struct.pack("<i", 7)])
    raw = p.read_bytes()
    assert raw == (struct.pack("<i", 8) + struct.pack("<d", 1.5) + struct.pack("<i", 8) +
                   struct.pack("<i", 4) + struct.pack("<i", 7) + struct.pack("<i", 4))


def test_split_records_have_signed_markers_and_round_trip(tmp_path):
    p = tmp_path / "r.dat"
    big = bytes(range(256)) * 3 + b"xyz"            # 771 bytes, split at 300
    small = b"abcd"
    dumps.write_records(p, [big, small], max_sub=300)
    raw = p.read_bytes()
    m = [struct.unpack("<i", raw[o:o + 4])[0] for o in (0, 304, 308, 612, 616)]
    # sub-record 1: head -300 (more follow), tail +300 (first)
    assert m[0] == -300 and m[1] == 300
    # sub-record 2: head -300, tail -300
    assert m[2] == -300 and m[3] == -300
    # last: head +171, tail -171
    assert m[4] == 171
    assert struct.unpack("<i", raw[620 + 171:624 + 171])[0] == -171
    assert dumps.read_records(p) == [big, small]


def test_cell_and_cut_readers(tmp_path):
    a = np.arange(3 * 4 * 5 * 8, dtype=np.float32)
    p = tmp_path / "c.dat"
    a.tofile(p)
    cells = dumps.read_cells(p, (5, 4, 3), 8)
    assert cells.shape == (8, 3, 4, 5)
    assert cells[2, 1, 3, 4] == a.reshape(3, 4, 5, 8)[1, 3, 4, 2]
    c = np.arange(21, dtype=np.float64)
    c.tofile(tmp_path / "cut.dat")
    cut = dumps.read_cut(tmp_path / "cut.dat", double_prec=True)
    assert cut.shape == (3, 7) and cut[2, 0] == 14.0
