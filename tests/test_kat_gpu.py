"""The reference's analytical known-answer tests on the CUDA path (through the
C ABI), with the oracle's result beside each one."""

import numpy as np
import pytest

import kat_scenes as K
from pfsim import _native as N
from pfsim import recipe as R

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cuda():
    return R.NativeBackend()


@pytest.fixture(scope="module")
def cpu(oracle):
    return oracle.OracleBackend(precision=32)


def test_free_fall(cuda, cpu):
    a, b = cuda.build(K.free_fall()), cpu.build(K.free_fall())
    for _ in range(60):
        a.step(K.DT)
        b.step(K.DT)
    y = float(a.readback(N.PF_FIELD_POSITIONS)[0, 1])
    assert y < 0
    assert abs(y - K.free_fall_reference(60)) < 1e-4
    # 60 steps of |y| ~ 5 m: a few f32 ulps of contraction difference
    assert abs(y - float(b.readback(N.PF_FIELD_POSITIONS)[0, 1])) < 1e-5


def test_xpbd_rigid_limit(cuda, cpu):
    a, b = cuda.build(K.distance_pair(0.0, 4, 4)), cpu.build(K.distance_pair(0.0, 4, 4))
    ta, tb = K.run_trace(a, 1000, every=25), K.run_trace(b, 1000, every=25)
    drift = 0.0
    for (p, _), (q, _) in zip(ta, tb):
        drift = max(drift, abs(float(np.linalg.norm(p[1, :3].astype(np.float64) - p[0, :3])) - 1.0))
    assert drift < 1e-4
    assert float(np.abs(ta[0][0] - tb[0][0]).max()) < 1e-5


def test_xpbd_soft_limit(cuda):
    a = cuda.build(K.distance_pair(1e12, 1, 2))
    b = cuda.build(K.distance_pair(1e12, 1, 2, constrained=False))
    ta, tb = K.run_trace(a, 120, every=20), K.run_trace(b, 120, every=20)
    dev = max(float(np.abs(pa[1, :3] - pb[1, :3]).max()) for (pa, _), (pb, _) in zip(ta, tb))
    assert dev < 1e-6


def test_density_matches_brute_force(cuda, cpu):
    a = cuda.build(K.density_lattice())
    a.step(K.DT)
    rho = a.readback(N.PF_FIELD_DENSITY).astype(np.float64)
    ref = K.density_brute_force()
    d = np.abs(rho - ref)
    assert d.max() < 5e-3
    assert (d / np.maximum(ref, 1.0)).max() < 1e-5
    b = cpu.build(K.density_lattice())
    b.step(K.DT)
    np.testing.assert_allclose(rho, b.readback(N.PF_FIELD_DENSITY), rtol=1e-5, atol=5e-3)


def test_plane_rest(cuda):
    s = cuda.build(K.plane_rest())
    tr = K.run_trace(s, 60)
    ys = [float(p[0, 1]) for p, _ in tr]
    r = 0.05
    assert r - 1e-4 < ys[-1] < r + 5e-3
    assert abs(float(tr[-1][1][0, 1])) < 0.1
    assert min(ys) > r - 1e-4


def test_sdf_rotated_scaled_projection(cuda, cpu):
    rec, center, radius = K.sdf_rotated_scaled()
    a, b = cuda.build(rec), cpu.build(rec)
    a.step(K.DT)
    b.step(K.DT)
    pa = a.readback(N.PF_FIELD_POSITIONS)
    d = np.linalg.norm(pa[:, :3].astype(np.float64) - center, axis=1)
    assert (d < radius - 5e-3).sum() == 0
    # 1e-5 of the extent: the scaled sphere spans 2 m
    assert float(np.abs(pa - b.readback(N.PF_FIELD_POSITIONS)).max()) < 2e-5


def test_bending_holds_rest_angle(cuda, cpu):
    rec, g = K.folded_quad(np.pi / 2)
    a, b = cuda.build(rec), cpu.build(rec)
    a0 = K.signed_dihedral(g.positions)
    for _ in range(60):
        a.step(K.DT)
        b.step(K.DT)
    pa = a.readback(N.PF_FIELD_POSITIONS)
    assert abs(np.degrees(K.signed_dihedral(pa) - a0)) < 2.0
    assert float(np.abs(pa - b.readback(N.PF_FIELD_POSITIONS)).max()) < 1e-5
