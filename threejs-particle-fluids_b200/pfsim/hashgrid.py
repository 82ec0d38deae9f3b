"""Neighbour-grid counting sort (the reference's HashGrid rebuild) on the GPU.

Mirrors ``HashGrid`` / ``HashGridSnapshot`` of threejs-particle-fluids
(src/core/hashGrid/HashGrid.ts:29-64, 219-249): a grid descriptor with
``cellSize``, ``hashTableSize`` and ``hashOrigin`` and a rebuild that returns
``cellIndex``, ``counts``, ``cellStart``, ``cellEnd`` and ``sortedIndices``.
The sort is stable: each cell lists its particles in ascending index order.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _native as N


def _next_pow2(n: int) -> int:
    p = 1
    while p < n:
        p <<= 1
    return p


MAX_CELLS_SINGLE_LEVEL_SCAN = 1024 * 1024  # the reference's cap (sort.ts:28)


@dataclass(frozen=True)
class GridOptions:
    """A hash-grid key function.

    ``kind='morton'`` is the reference bucket function; ``kind='linear'`` is a
    bounded linear cell index with ``dims`` cells per axis (coordinates
    clamped into the grid).
    """

    cell_size: float
    kind: str = "morton"
    hash_origin: tuple[float, float, float] = (0.0, 0.0, 0.0)
    hash_table_size: int | None = None
    dims: tuple[int, int, int] | None = None

    def desc(self, capacity: int = 0) -> N.GridDesc:
        if not (np.isfinite(self.cell_size) and self.cell_size > 0):
            raise N.PfError(N.PF_ERR_INVALID, f"HashGrid: cellSize must be a positive finite number, got {self.cell_size}")
        d = N.GridDesc()
        d.cell_size = float(self.cell_size)
        d.origin[:] = [float(v) for v in self.hash_origin]
        if self.kind == "linear":
            if self.dims is None:
                raise N.PfError(N.PF_ERR_INVALID, "HashGrid: a linear grid needs dims")
            d.key_kind = N.PF_KEY_LINEAR
            d.dims[:] = [int(v) for v in self.dims]
        elif self.kind == "morton":
            d.key_kind = N.PF_KEY_MORTON
            size = self.hash_table_size
            if size is None:
                # HashGrid.ts:122-124 (without the single-level-scan cap, which
                # the look-back scan does not have).
                size = _next_pow2(2 * max(capacity, 1))
            d.table_size = int(size)
        else:
            raise N.PfError(N.PF_ERR_INVALID, f"HashGrid: unknown key kind {self.kind!r}")
        return d


@dataclass
class HashGridSnapshot:
    """The grid read back to the host (HashGrid.ts:55-64)."""

    capacity: int
    cells: int
    cell_index: np.ndarray
    counts: np.ndarray
    cell_start: np.ndarray
    sorted_indices: np.ndarray
    overflow: bool

    @property
    def cell_end(self) -> np.ndarray:
        return self.cell_start + self.counts


def sort(positions: np.ndarray, grid: GridOptions) -> HashGridSnapshot:
    """Sort host positions (n x 4 float32) by cell on the GPU; returns the snapshot."""
    pos = np.ascontiguousarray(positions, dtype=np.float32)
    if pos.ndim != 2 or pos.shape[1] != 4:
        raise N.PfError(N.PF_ERR_INVALID, "HashGrid: positions must be an (n, 4) float32 array")
    n = pos.shape[0]
    d = grid.desc(n)
    L = N.lib()
    cells = int(L.pf_grid_cells(C.byref(d)))
    if cells == 0:
        raise N.PfError(N.PF_ERR_INVALID, "HashGrid: invalid grid descriptor")
    perm = np.empty(n, np.uint32)
    keys = np.empty(n, np.uint32)
    start = np.empty(cells, np.uint32)
    count = np.empty(cells, np.uint32)
    ovf = np.zeros(1, np.uint32)
    N.check(
        L.pf_sort_host(
            N.ptr(pos),
            n,
            C.byref(d),
            N.ptr(perm, C.c_uint32),
            N.ptr(start, C.c_uint32),
            N.ptr(count, C.c_uint32),
            N.ptr(keys, C.c_uint32),
            N.ptr(ovf, C.c_uint32),
        )
    )
    return HashGridSnapshot(n, cells, keys, count, start, perm, bool(ovf[0]))
