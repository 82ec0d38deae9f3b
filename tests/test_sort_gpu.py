"""Parity of the CUDA stable counting sort (pf_sort through the C ABI) with
the oracle: permutation, cell start and count bit-exact.

Covers the 128^3 linear-key workload in both distributions, the reference's
Morton bucket keys, and the edge cases the reference's grid tests exercise
(empty input, a single cell holding everything, out-of-range cells).
"""

import numpy as np
import pytest

from pfsim import _native as N
from pfsim import hashgrid as H
from pfsim import workloads as W

pytestmark = pytest.mark.gpu


def linear_grid():
    return H.GridOptions(cell_size=W.SORT_CELL, kind="linear", dims=W.SORT_GRID_DIMS)


def oracle_sort(oracle, pos, grid: H.GridOptions):
    return oracle.sort(pos, grid.desc(pos.shape[0]))


def assert_same(gpu: H.HashGridSnapshot, ref: dict):
    assert np.array_equal(gpu.cell_index, ref["keys"])
    assert np.array_equal(gpu.counts, ref["count"])
    assert np.array_equal(gpu.cell_start, ref["start"])
    assert np.array_equal(gpu.sorted_indices, ref["perm"])
    assert gpu.overflow == bool(ref["overflow"][0])


@pytest.mark.parametrize("dist", ["uniform", "blobs"])
@pytest.mark.parametrize("n", [1_000, 100_000, 1_000_000, 4_000_000, 16_000_000])
def test_linear_sort_bit_exact(oracle, pfsim, dist, n):
    """The standalone sort workload at each of its sizes (1M, 4M, 16M) and in
    both distributions: keys, counts, cell starts and the permutation equal
    the oracle's stable counting sort bit for bit."""
    pos = W.sort_uniform(n, 100 + n) if dist == "uniform" else W.sort_blobs(n, 200 + n)
    g = linear_grid()
    assert_same(H.sort(pos, g), oracle_sort(oracle, pos, g))


@pytest.mark.parametrize("n", [64, 10_000, 300_000, 3_000_000])
def test_morton_sort_bit_exact(oracle, pfsim, n):
    """The reference's Morton buckets (one radix pass of 11 bits or fewer, or two)."""
    r = np.random.default_rng(n)
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = r.uniform(-3.0, 3.0, (n, 3))
    g = H.GridOptions(cell_size=0.05, kind="morton")
    assert_same(H.sort(pos, g), oracle_sort(oracle, pos, g))


def test_empty_input(pfsim):
    pos = np.zeros((0, 4), np.float32)
    snap = H.sort(pos, linear_grid())
    assert snap.sorted_indices.size == 0
    assert int(snap.counts.sum()) == 0
    assert int(snap.cell_start.max()) == 0


@pytest.mark.parametrize("n", [17, 4_096, 4_097, 70_000])
def test_all_in_one_cell(oracle, pfsim, n):
    """Every particle in one cell: the thread, CTA and radix fix-up tiers."""
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = 0.5
    g = linear_grid()
    snap = H.sort(pos, g)
    assert np.array_equal(snap.sorted_indices, np.arange(n, dtype=np.uint32))
    assert_same(snap, oracle_sort(oracle, pos, g))


def test_skewed_cells(oracle, pfsim):
    """A few hot cells of 10..20k particles among sparse ones."""
    r = np.random.default_rng(7)
    n = 200_000
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = r.random((n, 3))
    hot = r.integers(0, n, 60_000)
    pos[hot, :3] = (r.integers(0, 5, (hot.size, 1)) * 0.1 + 0.05).astype(np.float32)
    g = linear_grid()
    assert_same(H.sort(pos, g), oracle_sort(oracle, pos, g))


def test_out_of_range_clamps_and_flags(oracle, pfsim):
    pos = W.sort_uniform(10_000, 5)
    pos[::97, 0] = 1.7
    pos[::89, 1] = -0.4
    g = linear_grid()
    snap = H.sort(pos, g)
    assert snap.overflow
    assert_same(snap, oracle_sort(oracle, pos, g))


def test_repeat_is_deterministic(pfsim):
    pos = W.sort_blobs(500_000, 9)
    a = H.sort(pos, linear_grid())
    b = H.sort(pos, linear_grid())
    assert np.array_equal(a.sorted_indices, b.sorted_indices)


@pytest.mark.parametrize("dist", ["uniform", "blobs"])
def test_16m_properties(pfsim, dist):
    """Full size: properties that need no oracle (stable sort of the keys)."""
    n = 16_000_000
    pos = W.sort_uniform(n, 31) if dist == "uniform" else W.sort_blobs(n, 32)
    snap = H.sort(pos, linear_grid())
    keys = snap.cell_index
    cnt = np.bincount(keys, minlength=128**3)
    assert np.array_equal(snap.counts, cnt)
    assert np.array_equal(snap.cell_start, (np.cumsum(cnt) - cnt).astype(np.uint32))
    perm = snap.sorted_indices.astype(np.int64)
    sk = keys[perm]
    assert np.all(sk[1:] >= sk[:-1])
    same = sk[1:] == sk[:-1]
    assert np.all(perm[1:][same] > perm[:-1][same])
    assert np.array_equal(np.sort(perm), np.arange(n))


@pytest.mark.parametrize("cells", [(1, 1, 1), (2, 1, 1), (40, 40, 1), (64, 64, 64), (2048, 2048, 64)])
def test_radix_plans(oracle, pfsim, cells):
    """Grids whose keys need no, one, two and three radix passes (1 cell,
    1 bit, 11 bits, 18 bits, 28 bits), with ragged last tiles."""
    r = np.random.default_rng(sum(cells))
    n = 123_457
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = r.random((n, 3)) * np.array(cells, np.float32) * 0.01
    g = H.GridOptions(cell_size=0.01, kind="linear", dims=cells)
    assert_same(H.sort(pos, g), oracle_sort(oracle, pos, g))


def test_sizes_shrink_and_grow(oracle, pfsim):
    """Successive sorts of different sizes on one workspace: each pass leaves
    the look-back words of the next call clear."""
    g = linear_grid()
    for n in (300_000, 5_000, 2_000_000, 4_097, 1_000_000):
        pos = W.sort_blobs(n, 400 + n)
        assert_same(H.sort(pos, g), oracle_sort(oracle, pos, g))


@pytest.mark.parametrize("n", [4_097, 300_001])
def test_unaligned_caller_buffers(oracle, pfsim, n):
    """pf_sort on caller buffers that are 4-byte but not 16-byte aligned (the
    keys buffer is also the first radix pass's input, which is then copied
    element by element instead of 16 bytes at a time): the same results as
    the oracle."""
    import ctypes as C

    import torch

    pos_h = W.sort_blobs(n, 500 + n)
    g = linear_grid()
    desc = g.desc(n)
    cells = int(N.lib().pf_grid_cells(C.byref(desc)))
    pos = torch.from_numpy(pos_h).cuda()
    # each buffer one element into a larger allocation
    perm = torch.full((n + 1,), -1, dtype=torch.int32, device="cuda")
    keys = torch.full((n + 1,), -1, dtype=torch.int32, device="cuda")
    start = torch.full((cells + 1,), -1, dtype=torch.int32, device="cuda")
    count = torch.full((cells + 1,), -1, dtype=torch.int32, device="cuda")
    ovf = torch.zeros(2, dtype=torch.int32, device="cuda")

    def at1(t):
        return C.c_void_p(t.data_ptr() + 4)

    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    N.check(N.lib().pf_sort(C.c_void_p(pos.data_ptr()), n, C.byref(desc), at1(perm), at1(start), at1(count),
                            at1(keys), at1(ovf), stream))
    torch.cuda.synchronize()
    ref = oracle_sort(oracle, pos_h, g)
    u32 = lambda t: t.cpu().numpy().view(np.uint32)[1:]  # noqa: E731
    assert np.array_equal(u32(keys), ref["keys"])
    assert np.array_equal(u32(perm), ref["perm"])
    assert np.array_equal(u32(start), ref["start"])
    assert np.array_equal(u32(count), ref["count"])
    assert int(u32(ovf)[0]) == int(ref["overflow"][0])
    for t in (perm, keys, start, count):
        assert int(t[0]) == -1  # nothing written before the buffers
