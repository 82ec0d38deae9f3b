"""pf_sort_noalloc: the grid sort for callers that cannot allocate GPU memory.

Some hosts hand all device memory to their own pool allocator, and some frame
loops must not stall on an allocation once they run; pf_sort grows a scratch
workspace with cudaMalloc, pf_sort_noalloc uses a fixed block compiled into
the library instead. These tests call it through the C ABI on caller-owned
device buffers and compare its results with pf_sort's on the same input, bit
for bit (the sort is integer work), on two calls in a row so the second call
runs on the block the first one left behind. This file is collected last so a
run that stops at the first failure has run every other test first.
"""

import ctypes as C

import numpy as np
import pytest

from pfsim import _native as N
from pfsim import hashgrid as H
from pfsim import workloads as W

pytestmark = pytest.mark.gpu

MAX_PARTICLES = 1 << 20


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _run(entry, pos, n, desc, cells):
    import torch

    perm = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    start = torch.full((cells,), -1, dtype=torch.int32, device="cuda")
    count = torch.full((cells,), -1, dtype=torch.int32, device="cuda")
    keys = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    ovf = torch.full((1,), 7, dtype=torch.int32, device="cuda")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    N.check(entry(_ptr(pos), n, C.byref(desc), _ptr(perm), _ptr(start), _ptr(count), _ptr(keys), _ptr(ovf), stream))
    torch.cuda.synchronize()
    return [t.cpu().numpy() for t in (perm, start, count, keys, ovf)]


@pytest.mark.parametrize("dist", ["uniform", "blobs"])
def test_noalloc_matches_pf_sort_twice(pfsim, dist):
    import torch

    L = N.lib()
    n = MAX_PARTICLES
    host = W.sort_uniform(n, 71) if dist == "uniform" else W.sort_blobs(n, 72)
    pos = torch.from_numpy(host).cuda()
    grid = H.GridOptions(cell_size=W.SORT_CELL, kind="linear", dims=W.SORT_GRID_DIMS)
    desc = grid.desc(n)
    cells = int(L.pf_grid_cells(C.byref(desc)))
    want = _run(L.pf_sort, pos, n, desc, cells)
    for _ in range(2):
        got = _run(L.pf_sort_noalloc, pos, n, desc, cells)
        for a, b in zip(got, want):
            assert np.array_equal(a, b)


def test_noalloc_small_then_morton(pfsim):
    """A small linear sort after a large one, then Morton keys: the block keeps
    the previous call's contents, so each call must clear what it needs."""
    import torch

    L = N.lib()
    r = np.random.default_rng(5)
    for grid, n in ((H.GridOptions(cell_size=W.SORT_CELL, kind="linear", dims=W.SORT_GRID_DIMS), 1000),
                    (H.GridOptions(cell_size=0.05, kind="morton"), 200_000)):
        host = np.zeros((n, 4), np.float32)
        host[:, :3] = r.uniform(-2.0, 2.0, (n, 3))
        pos = torch.from_numpy(host).cuda()
        desc = grid.desc(n)
        cells = int(L.pf_grid_cells(C.byref(desc)))
        want = _run(L.pf_sort, pos, n, desc, cells)
        got = _run(L.pf_sort_noalloc, pos, n, desc, cells)
        for a, b in zip(got, want):
            assert np.array_equal(a, b)


def test_noalloc_rejects_sizes_beyond_its_block(pfsim):
    """Sizes past the fixed block are refused on the host with a clear error."""
    L = N.lib()
    grid = H.GridOptions(cell_size=W.SORT_CELL, kind="linear", dims=W.SORT_GRID_DIMS)
    desc = grid.desc(MAX_PARTICLES + 1)
    rc = L.pf_sort_noalloc(C.c_void_p(16), MAX_PARTICLES + 1, C.byref(desc), C.c_void_p(16), C.c_void_p(16),
                           C.c_void_p(16), None, None, None)
    assert rc == N.PF_ERR_INVALID
    assert "at most 1048576 particles" in L.pf_last_error().decode()
    big = H.GridOptions(cell_size=0.001, kind="linear", dims=(256, 256, 256)).desc(10)
    rc = L.pf_sort_noalloc(C.c_void_p(16), 10, C.byref(big), C.c_void_p(16), C.c_void_p(16), C.c_void_p(16),
                           None, None, None)
    assert rc == N.PF_ERR_INVALID
    assert "cells" in L.pf_last_error().decode()
