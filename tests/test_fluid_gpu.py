"""PBF fluid substep on the CUDA path against the oracle.

Tolerances: positions after one step (one frame of substeps) within 1e-5 of
the container extent (1 m here); neighbour lists, which are integer work,
element for element; long runs by statistics because the dynamics are
chaotic.
"""

import numpy as np
import pytest

from pfsim import _native as N
from pfsim import recipe as R
from pfsim import workloads as W

pytestmark = pytest.mark.gpu

DT = 1.0 / 60.0
EXTENT = 1.0  # container extent of the dam break (x span), metres
POS_TOL = 1e-5 * EXTENT


@pytest.fixture(scope="module")
def cuda():
    return R.NativeBackend()


def test_neighbor_lists_bit_exact(oracle, cuda, nbr_path):
    """Lists built from identical positions hold the same particles in the
    same order (walk order dz, dy, dx; ascending index in a cell)."""
    r = W.dam_break(5000, seed=1, gravity=(0.0, 0.0, 0.0), substeps=1, iterations=1)
    a, b = cuda.build(r), oracle.OracleBackend().build(r)
    a.step(DT)
    b.step(DT)
    na, nb = a.readback(N.PF_FIELD_NEIGHBOR_COUNT), b.readback(N.PF_FIELD_NEIGHBOR_COUNT)
    assert np.array_equal(na, nb)
    la, lb = a.readback(N.PF_FIELD_NEIGHBORS), b.readback(N.PF_FIELD_NEIGHBORS)
    assert np.array_equal(la, lb)
    da, db = a.readback(N.PF_FIELD_DENSITY), b.readback(N.PF_FIELD_DENSITY)
    np.testing.assert_allclose(da, db, rtol=1e-5, atol=5e-3)
    lam_a, lam_b = a.readback(N.PF_FIELD_LAMBDA), b.readback(N.PF_FIELD_LAMBDA)
    np.testing.assert_allclose(lam_a, lam_b, rtol=1e-4, atol=1e-9)


@pytest.mark.parametrize("seed", [0, 7])
def test_one_frame_positions_within_tolerance(oracle, cuda, seed, nbr_path):
    r = W.dam_break(5000, seed=seed)
    a, b = cuda.build(r), oracle.OracleBackend().build(r)
    a.step(DT)
    b.step(DT)
    xa, xb = a.readback(N.PF_FIELD_POSITIONS), b.readback(N.PF_FIELD_POSITIONS)
    assert np.abs(xa - xb).max() <= POS_TOL
    va, vb = a.readback(N.PF_FIELD_VELOCITIES), b.readback(N.PF_FIELD_VELOCITIES)
    assert np.abs(va - vb).max() <= POS_TOL / (DT / r.loop.substeps)
    assert not any(a.overflow().values())


def test_one_frame_against_fp64_rerun(oracle, cuda):
    r = W.dam_break(5000, seed=3)
    a = cuda.build(r)
    b = oracle.OracleBackend(precision=64).build(r)
    a.step(DT)
    b.step(DT)
    xa = a.readback(N.PF_FIELD_POSITIONS).astype(np.float64)
    xb = b.readback(N.PF_FIELD_POSITIONS, as_f64=True)
    assert np.abs(xa - xb).max() <= POS_TOL


def stats(scene, rho0):
    x = scene.readback(N.PF_FIELD_POSITIONS)[:, :3].astype(np.float64)
    v = scene.readback(N.PF_FIELD_VELOCITIES)[:, :3].astype(np.float64)
    d = scene.readback(N.PF_FIELD_DENSITY).astype(np.float64)
    err = np.maximum(d / rho0 - 1.0, 0.0)
    return {"com": x.mean(0), "ke": 0.5 * (v * v).sum(1).mean(), "mean_err": err.mean(), "max_err": err.max()}


def test_long_run_statistics(oracle, cuda):
    """100 frames: centre of mass, kinetic energy and density error agree."""
    r = W.dam_break(5000, seed=5)
    rho0 = r.materials[0][1].rest_density
    a, b = cuda.build(r), oracle.OracleBackend().build(r)
    for _ in range(100):
        a.step(DT)
        b.step(DT)
    sa, sb = stats(a, rho0), stats(b, rho0)
    assert np.abs(sa["com"] - sb["com"]).max() < 0.01
    assert abs(sa["ke"] - sb["ke"]) <= 0.15 * max(sb["ke"], 1e-6)
    assert abs(sa["mean_err"] - sb["mean_err"]) < 0.01
    assert sa["max_err"] < 0.5
    x = a.readback(N.PF_FIELD_POSITIONS)
    assert np.isfinite(x).all()
    assert x[:, 1].min() > -1e-3  # the floor holds


def test_repeat_is_bit_identical(cuda):
    r = W.dam_break(5000, seed=2)
    a, b = cuda.build(r), cuda.build(r)
    for _ in range(10):
        a.step(DT)
        b.step(DT)
    assert np.array_equal(a.readback(N.PF_FIELD_POSITIONS), b.readback(N.PF_FIELD_POSITIONS))


@pytest.mark.parametrize("use_graph", [False, True])
def test_batched_equals_plain(cuda, use_graph):
    """A scene stepped alone and inside a batch of uneven scenes agrees bit for bit."""
    recipes = [W.dam_break(3000, seed=11), W.dam_break(8000, seed=12, scale=1.5, offset=(3.0, 0.0, 0.0)),
               W.dam_break(1200, seed=13, scale=0.7)]
    plain = [cuda.build(r) for r in recipes]
    batch = R.Batch([cuda.build(r) for r in recipes], use_graph=use_graph)
    for _ in range(5):
        for s in plain:
            s.step(DT)
        batch.step(DT)
    for i, s in enumerate(plain):
        assert np.array_equal(s.readback(N.PF_FIELD_POSITIONS), batch.readback(i, N.PF_FIELD_POSITIONS))
        assert np.array_equal(s.readback(N.PF_FIELD_VELOCITIES), batch.readback(i, N.PF_FIELD_VELOCITIES))


def test_async_batch_reads_equal_sync_reads(cuda):
    """pf_batch_read_positions_async, one read per step into two pinned
    buffers in turn while the next steps run, delivers every step's positions
    bit for bit as the synchronous read of a twin batch does."""
    import ctypes as C

    import torch

    recipes = [W.dam_break(3000, seed=14), W.dam_break(6000, seed=15, scale=1.3, offset=(3.0, 0.0, 0.0))]
    a = R.Batch([cuda.build(r) for r in recipes])
    b = R.Batch([cuda.build(r) for r in recipes])
    total = sum(r.capacity for r in recipes)
    L = N.lib()
    want = []
    for _ in range(5):
        a.step(DT)
        buf = np.empty(total * 4, np.float32)
        N.check(L.pf_batch_read_positions(a.h, buf.ctypes.data_as(C.POINTER(C.c_float)), buf.nbytes))
        want.append(buf)
    pinned = [torch.empty(total * 4, dtype=torch.float32).pin_memory() for _ in range(5)]
    for k in range(5):
        b.step(DT)
        N.check(L.pf_batch_read_positions_async(b.h, C.cast(C.c_void_p(pinned[k].data_ptr()), C.POINTER(C.c_float)),
                                                pinned[k].numel() * 4))
    N.check(L.pf_batch_wait_reads(b.h))
    for k in range(5):
        assert np.array_equal(pinned[k].numpy(), want[k]), k
    a.close()
    b.close()


def _tuning(batch):
    import ctypes as C

    v = [C.c_uint32() for _ in range(5)]
    N.check(N.lib().pf_batch_tuning(batch.h, *[C.byref(x) for x in v]))
    return [x.value for x in v]  # path, block, unroll (density pass), group, entry bits


def test_tuning_cache_file(cuda, tmp_path, monkeypatch):
    """PFSIM_TUNE_CACHE: a world that times its candidates appends one line
    keyed by GPU, configuration and particle count; a world of the same
    configuration takes the last matching line's choices and times nothing
    (a planted line with other slot-path choices is what pf_batch_tuning then
    reports, and nothing is appended); a world of another particle count
    appends its own line. The planted choices (512-thread blocks, fetch depth
    2, 32-bit entries) step to the same bits as the fixed default ones."""
    monkeypatch.delenv("PFSIM_NBR_PATH", raising=False)
    cache = tmp_path / "tune.txt"
    monkeypatch.setenv("PFSIM_TUNE_CACHE", str(cache))

    def recipes(n0=3000):
        return [W.dam_break(n0, seed=21), W.dam_break(5000, seed=22, scale=1.2, offset=(3.0, 0.0, 0.0))]

    a = R.Batch([cuda.build(r) for r in recipes()])
    a.step(DT)
    lines = cache.read_text().splitlines()
    assert len(lines) == 1
    f = lines[0].split()
    assert f[0] == "pfsim-tune-1" and len(f) == 17
    assert int(f[4]) >= sum(r.capacity for r in recipes())  # slots, scenes padded to whole chunks
    assert _tuning(a)[:4] == [int(f[5]), int(f[7]), int(f[11]), int(f[14])]
    a.close()

    planted = f[:5] + ["0"] + ["512"] * 4 + ["2"] * 4 + ["0", "0", "1"]
    cache.write_text(lines[0] + "\nnot a tuning line\n" + " ".join(planted) + "\n")
    b = R.Batch([cuda.build(r) for r in recipes()])
    b.step(DT)
    assert _tuning(b) == [0, 512, 2, 0, 32]
    assert len(cache.read_text().splitlines()) == 3

    monkeypatch.setenv("PFSIM_NBR_PATH", "0")  # slot path, 256-thread blocks, depth 4, 16-bit entries
    c = R.Batch([cuda.build(r) for r in recipes()])
    c.step(DT)
    assert _tuning(c) == [0, 256, 4, 0, 16]
    for _ in range(4):
        b.step(DT)
        c.step(DT)
    for i in range(2):
        assert np.array_equal(b.readback(i, N.PF_FIELD_POSITIONS), c.readback(i, N.PF_FIELD_POSITIONS))
        assert np.array_equal(b.readback(i, N.PF_FIELD_VELOCITIES), c.readback(i, N.PF_FIELD_VELOCITIES))
    b.close()
    c.close()

    monkeypatch.delenv("PFSIM_NBR_PATH")
    d = R.Batch([cuda.build(r) for r in recipes(4000)])
    d.step(DT)
    d.close()
    lines = cache.read_text().splitlines()
    assert len(lines) == 4 and int(lines[3].split()[4]) > int(f[4])


def test_worlds_reuse_pooled_device_memory(cuda):
    """A destroyed world's device memory stays in the library's pool, the
    next world of the same size takes it from there (the device's free
    memory does not move), and pf_trim_device_memory hands it back; the
    second world steps to the same bits as the first."""
    import torch

    L = N.lib()
    N.check(L.pf_trim_device_memory())
    free0 = torch.cuda.mem_get_info()[0]
    r = W.dam_break(200_000, seed=31)
    a = cuda.build(r)
    a.step(DT)
    xa = a.readback(N.PF_FIELD_POSITIONS)
    free1 = torch.cuda.mem_get_info()[0]
    held = free0 - free1
    assert held > 0
    a.close()
    free2 = torch.cuda.mem_get_info()[0]
    assert free2 - free1 < 0.25 * held  # kept by the pool
    b = cuda.build(r)
    b.step(DT)
    free3 = torch.cuda.mem_get_info()[0]
    assert abs(free3 - free2) < 0.25 * held  # taken from the pool
    assert np.array_equal(b.readback(N.PF_FIELD_POSITIONS), xa)
    b.close()
    N.check(L.pf_trim_device_memory())
    free4 = torch.cuda.mem_get_info()[0]
    assert free4 - free1 > 0.75 * held  # handed back


@pytest.mark.parametrize("seed", [4, 9])
def test_vorticity_confinement_one_frame(oracle, cuda, seed):
    """FluidSystem with vorticity (velocity.ts:36-120): curl in the XSPH walk,
    eta over fluid neighbours, eps (N x omega) dt added with the XSPH change."""
    r = W.dam_break(5000, seed=seed)
    r.materials[0][1].vorticity = 0.02
    a, b = cuda.build(r), oracle.OracleBackend().build(r)
    for _ in range(2):
        a.step(DT)
        b.step(DT)
    xa, xb = a.readback(N.PF_FIELD_POSITIONS), b.readback(N.PF_FIELD_POSITIONS)
    assert np.abs(xa - xb).max() <= POS_TOL
    va, vb = a.readback(N.PF_FIELD_VELOCITIES), b.readback(N.PF_FIELD_VELOCITIES)
    assert np.abs(va - vb).max() <= POS_TOL / (DT / r.loop.substeps)


def test_two_fluids_in_one_scene(oracle):
    """Two fluids on one particle system (halves of a dam break, rest
    densities 1 and 1.3 of the lattice's): each fluid's position correction
    reads its own multipliers only (the reference keeps one lambda buffer
    per FluidSystem), against the oracle after one frame."""
    import copy

    from pfsim import _native as N
    from pfsim import recipe as R
    from pfsim import workloads as W

    r = copy.deepcopy(W.dam_break(6000, seed=12))
    f = r.materials[0][1]
    n = r.capacity
    h = n // 2
    a = R.FluidOpts(**{**f.__dict__, "range": (0, h)})
    b = R.FluidOpts(**{**f.__dict__, "range": (h, n - h), "rest_density": f.rest_density * 1.3})
    r.materials = [("fluid", a), ("fluid", b)]
    g = R.NativeBackend().build(r)
    o = oracle.OracleBackend(precision=32).build(r)
    for _ in range(2):
        g.step(1.0 / 60.0)
        o.step(1.0 / 60.0)
    dev = float(np.abs(g.readback(N.PF_FIELD_POSITIONS).astype(np.float64)
                       - o.readback(N.PF_FIELD_POSITIONS).astype(np.float64)).max())
    assert dev <= 1e-5, dev


def test_mass_write_leaves_the_one_mass_path(oracle, cuda):
    """A single-fluid scene of one mass takes the one-mass path (the position
    pass gathers (x*, lambda) and applies the slot itself). Writing unequal
    inverse masses moves it to the general path from the next step on, in a
    plain scene and inside a batch stepped by a captured graph: the two agree
    bit for bit, and positions stay within the tolerance of the oracle given
    the same write. The masses change by 10 %: with every other particle's
    mass doubled the step is ill-conditioned (the oracle's own FP32 and FP64
    runs then differ by centimetres after one frame), so such a write is no
    parity case at 1e-5."""
    r = W.dam_break(4000, seed=21)
    a = cuda.build(r)
    o = oracle.OracleBackend(precision=32).build(r)
    batch = R.Batch([cuda.build(r), cuda.build(W.dam_break(2000, seed=22))], use_graph=True)
    a.step(DT)
    o.step(DT)
    batch.step(DT)
    w = a.readback(N.PF_FIELD_INV_MASS)
    w[::2] *= np.float32(0.9)
    a.write(N.PF_FIELD_INV_MASS, w)
    o.write(N.PF_FIELD_INV_MASS, w)
    batch.write(0, N.PF_FIELD_INV_MASS, w)
    a.step(DT)
    o.step(DT)
    batch.step(DT)
    xa = a.readback(N.PF_FIELD_POSITIONS)
    assert np.array_equal(xa, batch.readback(0, N.PF_FIELD_POSITIONS))
    assert np.array_equal(a.readback(N.PF_FIELD_LAMBDA), batch.readback(0, N.PF_FIELD_LAMBDA))
    assert np.array_equal(a.readback(N.PF_FIELD_INV_MASS), w)
    assert np.abs(xa - o.readback(N.PF_FIELD_POSITIONS)).max() <= POS_TOL
    assert np.array_equal(a.readback(N.PF_FIELD_DENSITY), batch.readback(0, N.PF_FIELD_DENSITY))
