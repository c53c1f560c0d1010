"""The C ABI library loads and exports every entry point include/imhd.h
declares (no device calls: runs without a GPU)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "imhd.h")


def declared():
    names = []
    for line in open(HEADER):
        m = re.match(r"^\s*(?:const\s+)?(?:int|void|long long|const char\*|char)\s*\*?\s*(imhd_\w+)\s*\(", line)
        if m:
            names.append(m.group(1))
    return names


def test_header_declares_the_boundary():
    names = declared()
    for must in ("imhd_create", "imhd_upload", "imhd_step", "imhd_download", "imhd_set_force",
                 "imhd_diagnostics", "imhd_destroy"):
        assert must in names


def test_library_exports_every_declared_symbol():
    from isothermal_mhd_b200 import _lib
    L = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared() if not hasattr(L, n)]
    assert not missing, missing
    assert set(declared()) == set(_lib.EXPORTS)


def test_config_errors_are_reported_without_a_device():
    from isothermal_mhd_b200 import ImhdError, _lib
    cfg = _lib.ImhdConfig()
    _lib.lib().imhd_default_config(ctypes.byref(cfg))
    assert cfg.nx == 64 and cfg.ng == 6 and cfg.ng_pass == 4 and cfg.cour == 0.35
    h = ctypes.c_void_p()
    for field, bad in (("nx", 2), ("precision", 16), ("riemann", 7), ("npass", 9), ("recon", 5)):
        c = _lib.ImhdConfig()
        _lib.lib().imhd_default_config(ctypes.byref(c))
        setattr(c, field, bad)
        rc = _lib.lib().imhd_create(ctypes.byref(c), ctypes.byref(h))
        assert rc == 1, (field, rc)
        assert _lib.lib().imhd_last_error()
    with pytest.raises(ImhdError):
        _lib.check(1)
