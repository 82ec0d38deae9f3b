"""The solver's neighbour grid against the reference's unbounded hash.

The reference bins particles into Morton-hashed buckets over an unbounded
cell lattice (src/core/hashGrid/cellIndex.ts:113-170, HashGrid.ts:122-125):
a particle may be anywhere, and its overflow flag fires only for cells
512 or more cells from the hash origin. The solver uses a window of linear
cells over the same lattice that moves with the particles every substep.
These tests check, against the oracle (which walks the reference's Morton
buckets, query.ts:24-70), that

* lists built from the same positions are equal element for element while
  the particles roam far outside the window's first placement (auto bounds
  and free fall), with neither flag raised;
* the reference's grid flag fires where the reference's would;
* particles spread wider than a too-small window are clamped and flagged
  (grid_clamped) with every neighbour still found.
"""

import copy

import numpy as np
import pytest

from pfsim import _native as N
from pfsim import recipe as R
from pfsim import workloads as W

pytestmark = pytest.mark.gpu

DT = 1.0 / 60.0


@pytest.fixture(scope="module")
def cuda():
    return R.NativeBackend()


def frozen(r, x, grid_min=(0.0, 0.0, 0.0), grid_max=(0.0, 0.0, 0.0)):
    """`r` rebuilt at positions x, at rest and without gravity, one substep
    of one iteration: its first list is built from exactly x."""
    q = copy.deepcopy(r)
    q.uploads = [R.Upload(0, np.ascontiguousarray(x[:, :3], np.float32))]
    q.loop.gravity = (0.0, 0.0, 0.0)
    q.loop.substeps = 1
    q.loop.iterations = 1
    q.loop.grid_min, q.loop.grid_max = tuple(grid_min), tuple(grid_max)
    return q


def lists(scene):
    return scene.readback(N.PF_FIELD_NEIGHBOR_COUNT), scene.readback(N.PF_FIELD_NEIGHBORS)


def assert_same_lists(oracle, cuda, r):
    a, b = cuda.build(r), oracle.OracleBackend().build(r)
    a.step(DT)
    b.step(DT)
    (ca, la), (cb, lb) = lists(a), lists(b)
    assert np.array_equal(ca, cb)
    assert np.array_equal(la, lb)
    return a.overflow(), b.overflow()


def test_auto_bounds_dam_break_lists_and_flags(oracle, cuda):
    """A dam break built without grid bounds: 100 frames with no flag, and
    the lists of its state every 20 frames equal to the oracle's walk."""
    r = W.dam_break(5000, seed=21)
    r.loop.grid_min = r.loop.grid_max = (0.0, 0.0, 0.0)
    a = cuda.build(r)
    for frame in range(1, 101):
        a.step(DT)
        if frame % 20 == 0:
            ov = a.overflow()
            assert not ov["grid"] and not ov["grid_clamped"] and not ov["neighbors"], (frame, ov)
            oa, ob = assert_same_lists(oracle, cuda, frozen(r, a.readback(N.PF_FIELD_POSITIONS)))
            assert not oa["grid"] and not ob["grid"]


def test_auto_bounds_equal_explicit_bounds(cuda):
    """Auto bounds and the container's bounds give the same lists, so the same
    bits, over 30 frames."""
    r = W.dam_break(5000, seed=22)
    q = copy.deepcopy(r)
    q.loop.grid_min = q.loop.grid_max = (0.0, 0.0, 0.0)
    a, b = cuda.build(r), cuda.build(q)
    for _ in range(30):
        a.step(DT)
        b.step(DT)
    assert np.array_equal(a.readback(N.PF_FIELD_POSITIONS), b.readback(N.PF_FIELD_POSITIONS))


def test_auto_bounds_step_time_matches_explicit_bounds(cuda):
    """A 100k-particle dam break steps as fast with auto bounds (a window
    placed on the particles and moved with them) as with the container's
    bounds: the median device time of a step over 40 frames each, the two
    scenes stepped alternately, within 10 %."""
    r = W.dam_break(100_000, seed=24)
    q = copy.deepcopy(r)
    q.loop.grid_min = q.loop.grid_max = (0.0, 0.0, 0.0)
    a, b = cuda.build(r), cuda.build(q)
    for _ in range(5):
        a.step(DT)
        b.step(DT)
    ta, tb = [], []
    for _ in range(40):
        a.step(DT)
        ta.append(a.last_step_ms())
        b.step(DT)
        tb.append(b.last_step_ms())
    ma, mb = float(np.median(ta)), float(np.median(tb))
    print(f"explicit bounds {ma:.3f} ms, auto bounds {mb:.3f} ms per step")
    assert not b.overflow()["grid_clamped"]
    assert mb <= 1.10 * ma, (ma, mb)


def test_window_grows_instead_of_clamping(cuda, monkeypatch):
    """A dam break whose explicit window holds only the fluid block, which
    the fluid outgrows within frames (and whose splash leaves through the
    open top), widens its window between steps instead of clamping: no
    clamp flag over 60 frames, and the same bits as the same scene in a
    window far larger than the fluid ever spreads (the lists, and so the
    results, do not depend on the window). Both run the slot path: the
    autotuner could otherwise pick the warp-tile path for one window size
    and not the other, and the two paths agree within tolerance, not bit
    for bit."""
    monkeypatch.setenv("PFSIM_NBR_PATH", "0")
    r = W.dam_break(20000, seed=25)
    h = r.materials[0][1].smoothing_radius
    small, big = copy.deepcopy(r), copy.deepcopy(r)
    small.loop.grid_min = (-0.5 - 2 * h, -2 * h, -0.3 - 2 * h)
    small.loop.grid_max = (-0.1 + 2 * h, 0.5 + 2 * h, 0.3 + 2 * h)
    big.loop.grid_min = (-0.5 - 2 * h, -2 * h, -0.3 - 2 * h)
    big.loop.grid_max = (0.5 + 2 * h, 12.0, 0.3 + 2 * h)
    a, b = cuda.build(small), cuda.build(big)
    for _ in range(60):
        a.step(DT)
        b.step(DT)
    assert not a.overflow()["grid_clamped"] and not b.overflow()["grid_clamped"]
    assert np.array_equal(a.readback(N.PF_FIELD_POSITIONS), b.readback(N.PF_FIELD_POSITIONS))
    assert np.array_equal(a.readback(N.PF_FIELD_VELOCITIES), b.readback(N.PF_FIELD_VELOCITIES))


def free_fall_blob(n=3000, seed=23, offset=(0.0, 0.0, 0.0)):
    """A fluid block with no walls, falling: it leaves any fixed window."""
    r = W.dam_break(n, seed=seed, offset=offset)
    r.prims = []
    h = r.materials[0][1].smoothing_radius
    lo = np.array([-0.5, 0.0, -0.3]) + np.asarray(offset)
    hi = np.array([-0.1, 0.5, 0.3]) + np.asarray(offset)
    # a window the size of the block plus four cells each side
    r.loop.grid_min, r.loop.grid_max = tuple(lo - 4 * h), tuple(hi + 4 * h)
    return r


def test_window_follows_a_falling_block(oracle, cuda):
    """60 frames of free fall (about 4.9 m below the window's first placement):
    no clamp, and the lists of the fallen state, built with the first
    window's bounds, equal the oracle's."""
    r = free_fall_blob()
    a = cuda.build(r)
    for _ in range(60):
        a.step(DT)
    x = a.readback(N.PF_FIELD_POSITIONS)
    assert x[:, 1].max() < -4.0
    ov = a.overflow()
    assert not ov["grid_clamped"] and not ov["grid"], ov
    oa, ob = assert_same_lists(oracle, cuda, frozen(r, x, r.loop.grid_min, r.loop.grid_max))
    assert not oa["grid_clamped"] and not oa["grid"] and not ob["grid"]


def test_reference_grid_flag_far_from_origin(oracle, cuda):
    """A block 600 cells from the hash origin: the reference's flag fires on
    both paths, the window does not clamp, and the lists still agree."""
    h = free_fall_blob().materials[0][1].smoothing_radius
    r = free_fall_blob(offset=(600.0 * h, 0.0, 0.0))
    x = np.asarray(r.uploads[0].pos, np.float32)
    oa, ob = assert_same_lists(oracle, cuda, frozen(r, x, r.loop.grid_min, r.loop.grid_max))
    assert ob["grid"] and oa["grid"]
    assert not oa["grid_clamped"]


def test_too_small_window_clamps_and_keeps_every_neighbour(oracle, cuda):
    """A window narrower than the block: particles outside it are clamped
    into its border cells and flagged; each particle's neighbour set (not
    their order) is still the oracle's."""
    r = free_fall_blob(seed=24)
    pos = np.asarray(r.uploads[0].pos, np.float32)[:, :3]
    c = pos.mean(0)
    x = np.concatenate([pos, np.zeros((r.capacity, 1), np.float32)], 1)
    q = frozen(r, x, c - 0.01, c + 0.01)
    a, b = cuda.build(q), oracle.OracleBackend().build(q)
    a.step(DT)
    b.step(DT)
    assert a.overflow()["grid_clamped"] and not a.overflow()["grid"]
    assert not b.overflow()["grid"]
    (ca, la), (cb, lb) = lists(a), lists(b)
    assert np.array_equal(ca, cb)
    for i in range(0, r.capacity, 7):
        assert set(la[i, :ca[i]].tolist()) == set(lb[i, :cb[i]].tolist())


def test_wide_warps_keep_32_bit_entries(oracle, cuda):
    """A fluid slab two cells thick and 130 cells wide: a z-layer holds about
    135,000 particles, so a warp's 27-cell rows reach further than 65,536
    slots and its list falls back to whole 32-bit slots. The lists still
    equal the oracle's, element for element."""
    s = 0.01
    h = 2.0 * s
    pts = W.fill_box(np.array([0.0, 0.0, 0.0]), np.array([130 * h, 130 * h, 2 * h]), s)
    pts = pts + W.rng(25).uniform(-0.05 * s, 0.05 * s, pts.shape)
    mass = 1000.0 * s**3
    rho0 = W.lattice_rest_density(s, h, mass)
    fluid = R.FluidOpts(range=(0, pts.shape[0]), rest_density=rho0, particle_spacing=(mass / rho0) ** (1 / 3),
                        smoothing_radius=h, compliance=1e-4, viscosity=0.01)
    r = R.Recipe(capacity=pts.shape[0], radius=s / 2, uploads=[R.Upload(0, pts.astype(np.float32))],
                 materials=[("fluid", fluid)], loop=R.LoopOpts(substeps=1, iterations=1, gravity=(0.0, 0.0, 0.0)))
    assert pts.shape[0] > 260_000
    assert_same_lists(oracle, cuda, r)
