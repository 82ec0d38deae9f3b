"""Parity on the measured workloads at their full sizes.

* The mixed scene (50,000 particles: 30,000 fluid in a lattice block and 20
  shape-matching soft bodies of about 1,000 particles with 27-member
  clusters, a sphere collider moving on a circle; 3 substeps, 4
  iterations): one frame within 1e-5 of the 1 m container extent against the
  FP32 oracle, and 300 frames compared by statistics (mean and max density
  error, kinetic energy, centre of mass), since the dynamics are chaotic.
* The batch stream the bench steps (256 scenes, 5k-200k particles, 70 %
  dam breaks in containers scaled 0.5-2, 30 % cloth sheets of 64^2-256^2):
  one batched frame of all 256 scenes, with the largest fluid, the smallest
  fluid, a 256 x 256 cloth and the largest container compared with the
  oracle, each within 1e-5 of its own container extent.

The oracle runs on every host core here (its threads split particles, and
its sums are per particle, so the thread count changes no result).
"""

import os

import numpy as np
import pytest

from pfsim import _native as N
from pfsim import recipe as R
from pfsim import workloads as W

pytestmark = pytest.mark.gpu

DT = 1.0 / 60.0
THREADS = os.cpu_count() or 1
BENCH_SEED = 1000  # the batch workload's scene stream on rank 0


@pytest.fixture(scope="module")
def cuda():
    return R.NativeBackend()


def dev(a, b):
    return float(np.abs(a.astype(np.float64) - b.astype(np.float64)).max())


def test_mixed_scene_full_one_frame(oracle, cuda):
    r = W.mixed_scene(seed=31)
    assert r.capacity >= 48_000 and len(r.materials[0][1].bodies) == 20
    a, b = cuda.build(r), oracle.OracleBackend(threads=THREADS).build(r)
    a.step(DT)
    b.step(DT)
    assert dev(a.readback(N.PF_FIELD_POSITIONS), b.readback(N.PF_FIELD_POSITIONS)) <= 1e-5
    assert not any(a.overflow().values())


def mixed_stats(scene, r):
    fluid = r.materials[1][1]
    s0, n = fluid.range
    x = scene.readback(N.PF_FIELD_POSITIONS)[:, :3].astype(np.float64)
    v = scene.readback(N.PF_FIELD_VELOCITIES)[:, :3].astype(np.float64)
    d = scene.readback(N.PF_FIELD_DENSITY)[s0:s0 + n].astype(np.float64)
    err = np.maximum(d / fluid.rest_density - 1.0, 0.0)
    return {"com": x.mean(0), "ke": 0.5 * (v * v).sum(1).mean(), "mean_err": err.mean(), "max_err": err.max()}


def test_mixed_scene_full_300_frames_statistics(oracle, cuda):
    r = W.mixed_scene(seed=32)
    a, b = cuda.build(r), oracle.OracleBackend(threads=THREADS).build(r)
    for _ in range(300):
        a.step(DT)
        b.step(DT)
    sa, sb = mixed_stats(a, r), mixed_stats(b, r)
    assert np.isfinite(a.readback(N.PF_FIELD_POSITIONS)).all()
    # five seconds of sloshing fluid among 20 soft bodies and a moving sphere
    # are chaotic: the two runs agree in their statistics, not their states
    # (the centre of mass within 5 % of the 1 m container, the kinetic energy
    # within 30 %, the mean density error within 0.01)
    assert np.abs(sa["com"] - sb["com"]).max() < 0.05, (sa, sb)
    assert abs(sa["ke"] - sb["ke"]) <= 0.3 * max(sb["ke"], 1e-4), (sa, sb)
    assert abs(sa["mean_err"] - sb["mean_err"]) < 0.01, (sa, sb)
    # the largest compression is one particle squeezed between bodies: the
    # same order of magnitude on both
    assert sa["max_err"] <= max(2.0 * sb["max_err"], 0.5), (sa, sb)
    assert not a.overflow()["grid_clamped"]


def test_batch_stream_sampled_scenes(oracle, cuda):
    recipes = W.batch_stream(256, seed=BENCH_SEED)
    info = [(i, r.capacity, r.materials[0][0], r.name) for i, r in enumerate(recipes)]
    fluids = [t for t in info if t[2] == "fluid"]
    pick = {
        max(fluids, key=lambda t: t[1])[0],
        min(fluids, key=lambda t: t[1])[0],
        next(t[0] for t in info if t[3] == "cloth_256x256"),
    }
    # the largest container: the dam breaks' walls span scale x 1 m in x
    def extent(r):
        lo = min(p.data1[0] for p in r.prims if p.kind == 0)
        hi = max(p.data1[0] for p in r.prims if p.kind == 0)
        return hi - lo
    pick.add(max(range(len(recipes)), key=lambda i: extent(recipes[i])))
    batch = R.Batch([cuda.build(r) for r in recipes], use_graph=True)
    try:
        batch.step(DT)
        for i in sorted(pick):
            ref = oracle.OracleBackend(threads=THREADS).build(recipes[i])
            ref.step(DT)
            tol = 1e-5 * extent(recipes[i])
            got = batch.readback(i, N.PF_FIELD_POSITIONS)
            assert dev(got, ref.readback(N.PF_FIELD_POSITIONS)) <= tol, (recipes[i].name, i)
            assert not any(batch.overflow(i).values()), (recipes[i].name, batch.overflow(i))
    finally:
        batch.close()
