"""pfsim — B200-native particle solver behind threejs-particle-fluids' API.

The CUDA path lives in libpfsim.so (C ABI: include/pfsim.h); this package is
the host-side mirror of the reference's TypeScript surface on top of it.
"""

from ._native import PfError, lib  # noqa: F401
from .hashgrid import GridOptions, HashGridSnapshot, sort  # noqa: F401

__all__ = ["PfError", "lib", "GridOptions", "HashGridSnapshot", "sort"]
