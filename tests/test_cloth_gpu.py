"""Cloth tethers, drag and lift and velocity smoothing on the CUDA path:
the reference's cloth known-answer tests (the scenes of test_cloth_oracle.py)
and parity with the oracle, positions within 1e-5 of the container extent;
batched scenes bit-identical to their plain steps; runtime parameter
changes and whole-field writes through the C ABI."""

import math

import numpy as np
import pytest

import kat_scenes as K
from pfsim import _native as N
from pfsim import recipe as R
from pfsim import shapes
from pfsim import workloads as W

pytestmark = pytest.mark.gpu

DT = 1.0 / 60.0
TOL = 1e-5  # metres: 1e-5 of the 1 m container extent


@pytest.fixture(scope="module")
def cuda():
    return R.NativeBackend()


def _graph(pos, idx, pinned, density=0.2):
    return shapes.create_cloth_graph(pos, idx, density, pinned=pinned)


def _dev(a, b, field=N.PF_FIELD_POSITIONS):
    return float(np.abs(a.readback(field).astype(np.float64) - b.readback(field).astype(np.float64)).max())


def test_tether_unilateral(cuda):
    """tether-unilateral.gpu.test.ts:68-175 (see test_cloth_oracle.py)."""
    pos, idx, top = K.grid_sheet(12)
    g = _graph(pos, idx, top)
    init = g.positions.copy()
    init[g.inv_mass != 0, 1] *= 0.5
    r, (tp, ta, tr) = K.cloth_system(g, 4, 2, gravity=(0.0, 0.0, 0.0), stretch=1e10, bend=1e10, positions=init)
    s = cuda.build(r)
    K.run_damped(s, 60, 0.95)
    p = s.readback(N.PF_FIELD_POSITIONS)[:, :3].astype(np.float64)
    assert np.isfinite(p).all()
    assert (np.linalg.norm(p[tp] - g.positions[ta], axis=1) - tr).max() < 1e-3


def test_tether_moving_pins(cuda):
    """tether-moving-pins.gpu.test.ts:23-74: pins moved through pf_write
    (positions and predicted positions) before the first step."""
    pos, idx = shapes.plane_geometry(1.0, 1.0, 7, 7)
    g = _graph(pos, idx, range(8))
    r, (tp, ta, tr) = K.cloth_system(g, 4, 2, gravity=(0.0, 0.0, 0.0), stretch=1e10, bend=1e10, drag=0.0,
                                     lift=0.0, radius=0.02)
    s = cuda.build(r)
    pinned = g.inv_mass == 0
    for field in (N.PF_FIELD_POSITIONS, N.PF_FIELD_PREDICTED):
        a = s.readback(field)
        a[pinned, 0] += 1.5
        s.write(field, a)
    for _ in range(5):
        s.step(DT)
    p = s.readback(N.PF_FIELD_POSITIONS)[:, :3].astype(np.float64)
    anchors = g.positions[ta] + np.array([1.5, 0.0, 0.0])
    assert (np.linalg.norm(p[tp] - anchors, axis=1) - tr).max() < 1e-3


def test_tether_stretch(cuda):
    """tether-stretch.gpu.test.ts:146-195 (see test_cloth_oracle.py)."""
    pos, idx, top = K.grid_sheet(32)
    g = _graph(pos, idx, top)
    out = {}
    for comp in (0.0, 1e10):
        r, _ = K.cloth_system(g, 8, 4, gravity=(0.0, -981.0, 0.0), bend=1.0, tether_compliance=comp)
        s = cuda.build(r)
        K.run_damped(s, 120, 0.9)
        p = s.readback(N.PF_FIELD_POSITIONS)[:, :3].astype(np.float64)
        ok = bool(np.isfinite(p).all())
        d = np.linalg.norm(p[g.pairs[:, 0]] - p[g.pairs[:, 1]], axis=1) if ok else None
        out[comp] = (ok, float(np.abs((d - g.rest_lengths) / g.rest_lengths).max()) if ok else math.inf)
    assert out[0.0][0] and out[0.0][1] < 0.05
    assert (not out[1e10][0]) or out[1e10][1] > 0.2


def test_wind_deflection(cuda, oracle):
    """wind-deflection.gpu.test.ts:215-260 (see test_cloth_oracle.py), and
    the same 240 damped frames on the oracle end within 1e-4 m."""
    pos, idx, top = K.grid_sheet(16, x0=-0.5)
    g = _graph(pos, idx, top)
    r, _ = K.cloth_system(g, 8, 4, bend=1.0, wind=(0.0, 0.0, 1.0))
    s = cuda.build(r)
    K.run_damped(s, 240, 0.9)
    p = s.readback(N.PF_FIELD_POSITIONS)
    assert np.isfinite(p).all()
    ang, dy, dz = K.wind_deflection_angle(p, g.inv_mass, top)
    want = K.wind_deflection_analytic(0.2, K.G, 1.0, 0.6125, 0.3)
    assert abs(math.degrees(ang) - math.degrees(want)) / math.degrees(want) < 0.1
    assert dz > 0.01 and dy < 0
    o = oracle.OracleBackend(precision=32).build(r)
    K.run_damped(o, 240, 0.9)
    assert _dev(s, o) < 1e-4


def _full_cloth(side, seed, **kw):
    args = dict(bend_compliance=1e-5, tethers=True, stretch_tolerance=0.06, wind=(0.8, 0.0, 1.5), drag=0.18,
                lift=0.02, damping=0.1)
    args.update(kw)
    return W.cloth_sheet(side, seed=seed, **args)


@pytest.mark.parametrize("side", [32, 64])
def test_full_cloth_matches_oracle(oracle, cuda, side):
    """Stretch, bending and tether colours, drag and lift, and velocity
    smoothing (the façade's cloth settings, Simulation.ts:703-718) against
    the oracle over three frames."""
    r = _full_cloth(side, side + 3)
    a, b = cuda.build(r), oracle.OracleBackend(precision=32).build(r)
    for _ in range(3):
        a.step(DT)
        b.step(DT)
    assert _dev(a, b) <= TOL
    assert _dev(a, b, N.PF_FIELD_VELOCITIES) <= TOL / DT


def test_cloth_params_setters(oracle, cuda):
    """ClothSystem wind / drag / lift / damping / bendCompliance setters
    (pf_cloth_set_params) between frames, on both backends."""
    r = _full_cloth(48, 11)
    a, b = cuda.build(r), oracle.OracleBackend(precision=32).build(r)
    sets = [R.cloth_params((0.0, 0.0, -3.0), 0.6, 0.4, 0.3, 1e-4), R.cloth_params((2.0, 0.5, 0.0), 0.0, 0.0, 0.0, 1e-6)]
    for f in range(6):
        if f in (2, 4):
            p = sets[(f - 2) // 2]
            a.set_cloth_params(0, p)
            b.set_cloth_params(0, p)
        a.step(DT)
        b.step(DT)
    assert _dev(a, b) <= 2 * TOL
    got = R.cloth_params()
    N.check(N.lib().pf_cloth_get_params(a.h, 0, got))
    assert tuple(got.wind) == (2.0, 0.5, 0.0) and got.drag == 0.0 and got.bend_compliance == np.float32(1e-6)
    with pytest.raises(N.PfError):
        a.set_cloth_params(0, R.cloth_params(drag=-1.0))
    with pytest.raises(N.PfError):
        a.set_cloth_params(0, R.cloth_params(damping=1.5))


def test_damping_needs_the_pass(cuda):
    """damping can change later only when it was given at creation
    (ClothSystemOptions.damping: the pass is only built then)."""
    s = cuda.build(_full_cloth(16, 1, damping=None))
    s.set_cloth_params(0, R.cloth_params((0.8, 0.0, 1.5), 0.18, 0.02, 0.0, 1e-5))
    with pytest.raises(N.PfError):
        s.set_cloth_params(0, R.cloth_params(damping=0.2))


def test_full_cloth_batch_matches_plain(cuda):
    """Full cloths batched with a fluid (cloth colours on the second stream,
    drag and lift and smoothing on the main one) equal their plain steps,
    also after a parameter change on scene 2 through the batch."""
    recipes = [_full_cloth(48, 2), W.dam_break(4000, seed=3), _full_cloth(32, 4, damping=None, wind=(0.0, 0.0, 0.5))]
    plain = [cuda.build(r) for r in recipes]
    batch = R.Batch([cuda.build(r) for r in recipes], use_graph=True)
    p = R.cloth_params((1.0, 0.0, -1.0), 0.3, 0.1, 0.0, 2e-5)
    for f in range(4):
        if f == 2:
            plain[2].set_cloth_params(0, p)
            batch.set_cloth_params(2, 0, p)
        for s in plain:
            s.step(DT)
        batch.step(DT)
    for i, s in enumerate(plain):
        for field in (N.PF_FIELD_POSITIONS, N.PF_FIELD_VELOCITIES):
            assert np.array_equal(s.readback(field), batch.readback(i, field)), (i, field)


def _cloth_and_fluid(cloth_first: bool):
    """One scene holding a dam-break fluid and a hanging cloth with drag and
    lift, in either material order: the cloth's aerodynamics runs before or
    after the fluid's neighbour pass (loop.ts:230-239 keeps material order)."""
    c = _full_cloth(24, 5)
    f = W.dam_break(3000, seed=6)
    nc, nf = c.capacity, f.capacity
    cloth = c.materials[0][1]
    fluid = f.materials[0][1]
    co = cloth.offset if cloth_first else nf
    fo = nc if cloth_first else 0
    cloth = R.ClothOpts(**{**cloth.__dict__, "offset": co})
    fluid = R.FluidOpts(**{**fluid.__dict__, "range": (fo, nf)})
    ups = [R.Upload(fo + u.start, u.pos, u.vel, u.inv_mass) for u in f.uploads]
    mats = [("cloth", cloth), ("fluid", fluid)] if cloth_first else [("fluid", fluid), ("cloth", cloth)]
    return R.Recipe(capacity=nc + nf, radius=f.radius, uploads=ups, materials=mats, prims=f.prims, loop=f.loop,
                    name=f"cloth_fluid_{'cf' if cloth_first else 'fc'}")


@pytest.mark.parametrize("cloth_first", [True, False])
def test_cloth_and_fluid_order(oracle, cuda, cloth_first):
    r = _cloth_and_fluid(cloth_first)
    a, b = cuda.build(r), oracle.OracleBackend(precision=32).build(r)
    a.step(DT)
    b.step(DT)
    assert _dev(a, b) <= TOL


def test_write_and_readback_roundtrip(cuda):
    """pf_write then pf_readback returns what was written, through the
    sorted slot order (positions keep their inverse mass)."""
    s = cuda.build(W.dam_break(3000, seed=8))
    s.step(DT)
    v = s.readback(N.PF_FIELD_VELOCITIES)
    v[:, :3] = np.random.default_rng(0).normal(size=(len(v), 3)).astype(np.float32)
    s.write(N.PF_FIELD_VELOCITIES, v)
    assert np.array_equal(s.readback(N.PF_FIELD_VELOCITIES)[:, :3], v[:, :3])
    w = s.readback(N.PF_FIELD_INV_MASS)
    x = s.readback(N.PF_FIELD_POSITIONS)
    x[:, 1] += 0.01
    s.write(N.PF_FIELD_POSITIONS, x)
    assert np.array_equal(s.readback(N.PF_FIELD_POSITIONS), x)
    assert np.array_equal(s.readback(N.PF_FIELD_INV_MASS), w)
    with pytest.raises(N.PfError):
        s.write(N.PF_FIELD_INV_MASS, -np.ones(len(w), np.float32))
    s.step(DT)
    assert np.isfinite(s.readback(N.PF_FIELD_POSITIONS)).all()
