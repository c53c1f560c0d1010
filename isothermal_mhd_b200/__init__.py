"""B200-native isothermal-MHD time step (van Leer + CT, Roe / HLLD / HLLE,
passive scalars, turbulence kick, CFL reduction) behind the C ABI of
include/imhd.h.

The compute path is libimhd.so (hand-written CUDA for sm_100a, built in-tree
by ``python -m isothermal_mhd_b200.build``).  Importing this package does not
require a GPU; creating a :class:`Box` does.
"""
from .box import Box, RIEMANN  # noqa: F401
from . import problems, forcing, driver, batch  # noqa: F401
from .batch import Batch  # noqa: F401
from ._lib import ImhdError, LIB_PATH, lib  # noqa: F401

__all__ = ["Box", "Batch", "RIEMANN", "problems", "forcing", "driver", "batch", "ImhdError", "LIB_PATH", "lib"]
