"""pf_sort_noalloc: the grid sort for callers that cannot allocate GPU memory.

Some hosts hand all device memory to their own pool allocator, and some frame
loops must not stall on an allocation once they run; pf_sort grows a scratch
workspace with cudaMalloc, pf_sort_noalloc uses a fixed block compiled into
the library instead. These tests call it through the C ABI on caller-owned
device buffers and compare its results with the oracle's stable counting sort
and with pf_sort's on the same input, bit for bit (the sort is integer work),
on two calls in a row so the second call runs on the block the first one left
behind. They also check that calls after the first allocate no device memory
and that the block's device error word reads back clear. This file is
collected last so a run that stops at the first failure has run every other
test first.
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


def _buffers(n, cells):
    import torch

    return dict(
        perm=torch.full((max(n, 1),), -1, dtype=torch.int32, device="cuda"),
        start=torch.full((cells,), -1, dtype=torch.int32, device="cuda"),
        count=torch.full((cells,), -1, dtype=torch.int32, device="cuda"),
        keys=torch.full((max(n, 1),), -1, dtype=torch.int32, device="cuda"),
        ovf=torch.full((1,), 7, dtype=torch.int32, device="cuda"),
    )


def _call(entry, pos, n, desc, b, stream):
    N.check(entry(_ptr(pos), n, C.byref(desc), _ptr(b["perm"]), _ptr(b["start"]), _ptr(b["count"]),
                  _ptr(b["keys"]), _ptr(b["ovf"]), stream))


def _host(b, n):
    import torch

    torch.cuda.synchronize()
    out = [t.cpu().numpy().view(np.uint32) for t in (b["perm"], b["start"], b["count"], b["keys"], b["ovf"])]
    out[0] = out[0][:n]
    out[3] = out[3][:n]
    return out


def _run(entry, pos, n, desc, cells):
    import torch

    b = _buffers(n, cells)
    _call(entry, pos, n, desc, b, C.c_void_p(torch.cuda.current_stream().cuda_stream))
    return _host(b, n)


def _assert_oracle(got, ref):
    perm, start, count, keys, ovf = got
    assert np.array_equal(perm, ref["perm"])
    assert np.array_equal(start, ref["start"])
    assert np.array_equal(count, ref["count"])
    assert np.array_equal(keys, ref["keys"])
    assert int(ovf[0]) == int(ref["overflow"][0])


@pytest.mark.parametrize("dist", ["uniform", "blobs"])
def test_noalloc_matches_oracle_and_pf_sort_twice(oracle, pfsim, dist):
    import torch

    L = N.lib()
    n = MAX_PARTICLES
    host = W.sort_uniform(n, 71) if dist == "uniform" else W.sort_blobs(n, 72)
    pos = torch.from_numpy(host).cuda()
    grid = H.GridOptions(cell_size=W.SORT_CELL, kind="linear", dims=W.SORT_GRID_DIMS)
    desc = grid.desc(n)
    cells = int(L.pf_grid_cells(C.byref(desc)))
    ref = oracle.sort(host, desc)
    want = _run(L.pf_sort, pos, n, desc, cells)
    _assert_oracle(want, ref)
    for _ in range(2):
        got = _run(L.pf_sort_noalloc, pos, n, desc, cells)
        _assert_oracle(got, ref)
        for a, b in zip(got, want):
            assert np.array_equal(a, b)


def test_noalloc_small_then_morton(oracle, pfsim):
    """A small linear sort after a large one, then Morton keys: the block keeps
    the previous call's contents, so each call must clear what it needs."""
    import torch

    L = N.lib()
    r = np.random.default_rng(5)
    for grid, n in ((H.GridOptions(cell_size=W.SORT_CELL, kind="linear", dims=W.SORT_GRID_DIMS), 1000),
                    (H.GridOptions(cell_size=0.05, kind="morton"), 200_000),
                    (H.GridOptions(cell_size=0.05, kind="morton", hash_table_size=64), 5_000)):
        host = np.zeros((n, 4), np.float32)
        host[:, :3] = r.uniform(-2.0, 2.0, (n, 3))
        pos = torch.from_numpy(host).cuda()
        desc = grid.desc(n)
        cells = int(L.pf_grid_cells(C.byref(desc)))
        ref = oracle.sort(host, desc)
        got = _run(L.pf_sort_noalloc, pos, n, desc, cells)
        _assert_oracle(got, ref)
        for a, b in zip(got, _run(L.pf_sort, pos, n, desc, cells)):
            assert np.array_equal(a, b)


def test_noalloc_allocates_nothing_after_setup(pfsim):
    """After the set-up call, calls of several sizes leave the device's free
    memory unchanged, and the block's error word reads back 0."""
    import torch

    L = N.lib()
    grid = H.GridOptions(cell_size=W.SORT_CELL, kind="linear", dims=W.SORT_GRID_DIMS)
    sizes = (MAX_PARTICLES, 1000, 300_000, 4097)
    inputs = []
    for n in sizes:
        desc = grid.desc(n)
        cells = int(L.pf_grid_cells(C.byref(desc)))
        inputs.append((n, desc, torch.from_numpy(W.sort_blobs(n, 900 + n)).cuda(), _buffers(n, cells)))
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    # set-up only (no start/count buffers), then one full call that loads
    # every kernel the later calls use
    N.check(L.pf_sort_noalloc(None, 0, C.byref(inputs[0][1]), None, None, None, None, None, stream))
    n0, d0, p0, b0 = inputs[0]
    _call(L.pf_sort_noalloc, p0, n0, d0, b0, stream)
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    for n, desc, pos, b in inputs + inputs:
        _call(L.pf_sort_noalloc, pos, n, desc, b, stream)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free_before
    bits = C.c_uint32(0xFFFF)
    N.check(L.pf_sort_device_errors(stream, C.byref(bits)))
    assert bits.value == 0


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
    bad = H.GridOptions(cell_size=0.05, kind="morton", hash_table_size=1000).desc(10)
    bad.table_size = 1000
    rc = L.pf_sort_noalloc(C.c_void_p(16), 10, C.byref(bad), C.c_void_p(16), C.c_void_p(16), C.c_void_p(16),
                           None, None, None)
    assert rc == N.PF_ERR_INVALID
    assert "hashTableSize must be a positive power of two" in L.pf_last_error().decode()
