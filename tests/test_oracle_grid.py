"""The oracle's neighbour grid against the reference's own known-answer tests.

CPU only. Each test restates a hash-grid test of the reference suite
(tests/analytical/hashgrid/*.gpu.test.ts) with the same inputs, tolerances
and ground truth, and runs it on the C++ oracle. Passing these pins the
oracle before it is used to check the CUDA path.
"""

import numpy as np
import pytest

from pfsim import _native as N
from pfsim import workloads as W

MORTON_BIAS = 512


def part1by2_cpu(n: int) -> int:
    # morton-encoding.gpu.test.ts:23-30
    m = n & 0x000003FF
    m = (m | (m << 16)) & 0xFF0000FF
    m = (m | (m << 8)) & 0x0300F00F
    m = (m | (m << 4)) & 0x030C30C3
    m = (m | (m << 2)) & 0x09249249
    return m & 0xFFFFFFFF


def morton_cpu(cx: int, cy: int, cz: int) -> int:
    # morton-encoding.gpu.test.ts:32-37
    ux = (cx + MORTON_BIAS) & 0xFFFFFFFF
    uy = (cy + MORTON_BIAS) & 0xFFFFFFFF
    uz = (cz + MORTON_BIAS) & 0xFFFFFFFF
    return (part1by2_cpu(ux) | (part1by2_cpu(uy) << 1) | (part1by2_cpu(uz) << 2)) & 0xFFFFFFFF


MORTON_CELLS = [
    (0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 1, 1), (-1, 0, 0), (0, -1, 0), (0, 0, -1),
    (-1, -1, -1), (10, 20, 30), (-10, -20, -30), (MORTON_BIAS - 1, 0, 0), (-MORTON_BIAS, 0, 0),
    (MORTON_BIAS - 1, MORTON_BIAS - 1, MORTON_BIAS - 1),
]


def morton_desc(cell, table, origin=(0.0, 0.0, 0.0)):
    d = N.GridDesc()
    d.key_kind = N.PF_KEY_MORTON
    d.cell_size = cell
    d.origin[:] = origin
    d.table_size = table
    return d


def linear_desc(cell, dims, origin=(0.0, 0.0, 0.0)):
    d = N.GridDesc()
    d.key_kind = N.PF_KEY_LINEAR
    d.cell_size = cell
    d.origin[:] = origin
    d.dims[:] = dims
    return d


def default_table(capacity: int) -> int:
    # HashGrid.ts:122-124
    p = 1
    while p < 2 * capacity:
        p <<= 1
    return min(p, 1 << 20)


def test_morton_known_answers(oracle):
    """morton-encoding.gpu.test.ts:41-98: 14 hand-verified cells."""
    L = oracle.lib()
    for c in MORTON_CELLS:
        assert L.or_morton(*c) == morton_cpu(*c)
    cell = 0.1
    pos = np.zeros((len(MORTON_CELLS), 4), np.float32)
    pos[:, :3] = (np.array(MORTON_CELLS, np.float64) + 0.5) * cell
    table = 1 << 18
    out = oracle.sort(pos, morton_desc(cell, table))
    expected = [morton_cpu(*c) & (table - 1) for c in MORTON_CELLS]
    assert out["keys"].tolist() == expected
    assert out["overflow"][0] == 0


def test_morton_overflow_flag(oracle):
    """morton-encoding.gpu.test.ts:100-127: one cell past the Morton range."""
    pos = np.zeros((1, 4), np.float32)
    pos[0, 0] = (MORTON_BIAS + 0.5) * 0.1
    out = oracle.sort(pos, morton_desc(0.1, default_table(1)))
    assert out["overflow"][0] == 1


def brute_counts(points: np.ndarray, h2: float, idx) -> np.ndarray:
    res = []
    for p in idx:
        d = points - points[p]
        d2 = (d * d).sum(axis=1)
        d2[p] = np.inf
        res.append(int((d2 < h2).sum()))
    return np.array(res)


def walk_counts(oracle, pos32: np.ndarray, desc, out, h2: float, idx) -> np.ndarray:
    res = []
    for p in idx:
        cand = oracle.walk(pos32[p, :3], desc, out["perm"], out["start"], out["count"])
        cand = cand[cand != p]
        d = pos32[cand, :3] - pos32[p, :3]
        d2 = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
        res.append(int((d2 < np.float32(h2)).sum()))
    return np.array(res)


def test_lattice_invariants_and_neighbor_counts(oracle):
    """hashgrid-lattice.gpu.test.ts:21-125: 4^3 lattice, spacing 0.05, h 0.08."""
    lat, s, h = 4, 0.05, 0.08
    pts = np.array([(i * s, j * s, k * s) for k in range(lat) for j in range(lat) for i in range(lat)])
    n = pts.shape[0]
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = pts
    desc = morton_desc(h, default_table(n))
    out = oracle.sort(pos, desc)
    assert int(out["count"].sum()) == n
    prefix = np.concatenate([[0], np.cumsum(out["count"])[:-1]]).astype(np.uint32)
    assert np.array_equal(out["start"], prefix)
    assert sorted(out["perm"].tolist()) == list(range(n))
    assert (out["keys"] < desc.table_size).all()
    got = walk_counts(oracle, pos, desc, out, h * h, range(n))
    want = brute_counts(pts, h * h, range(n))
    assert np.array_equal(got, want)


def lcg(seed: int):
    # hashgrid-random-stress.gpu.test.ts:21-27
    state = (seed & 0xFFFFFFFF) or 1

    def nxt():
        nonlocal state
        state = (state * 1664525 + 1013904223) & 0xFFFFFFFF
        return state / 0x100000000

    return nxt


def test_random_stress_sampled_counts(oracle):
    """hashgrid-random-stress.gpu.test.ts:29-109: 100k points, h 0.05, 100 samples."""
    n, h, margin = 100_000, 0.05, 0.01
    rand = lcg(0xC0FFEE)
    pts = np.array([[margin + rand() * (1 - 2 * margin) for _ in range(3)] for _ in range(n)])
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = pts
    desc = morton_desc(h, default_table(n))
    out = oracle.sort(pos, desc)
    srand = lcg(0xBEEFCAFE)
    idx = [int(srand() * n) for _ in range(100)]
    got = walk_counts(oracle, pos, desc, out, h * h, idx)
    want = brute_counts(pts, h * h, idx)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("dist", ["uniform", "blobs"])
def test_stable_linear_sort_matches_numpy(oracle, dist):
    """The oracle's counting sort is the stable sort of the linear 128^3 keys."""
    n = 200_000
    pos = W.sort_uniform(n, 11) if dist == "uniform" else W.sort_blobs(n, 12)
    desc = linear_desc(W.SORT_CELL, W.SORT_GRID_DIMS)
    out = oracle.sort(pos, desc)
    c = np.clip(np.floor(pos[:, :3].astype(np.float32) / np.float32(W.SORT_CELL)), 0, 127).astype(np.int64)
    keys = (c[:, 0] + 128 * (c[:, 1] + 128 * c[:, 2])).astype(np.uint32)
    assert np.array_equal(out["keys"], keys)
    assert np.array_equal(out["perm"], np.argsort(keys, kind="stable").astype(np.uint32))
    cnt = np.bincount(keys, minlength=128**3)
    assert np.array_equal(out["count"], cnt)
    assert np.array_equal(out["start"], (np.cumsum(cnt) - cnt).astype(np.uint32))
    assert out["overflow"][0] == 0
