"""Cloth tethers, drag and lift on the CPU.

The native tether builder (pf_cloth_build_tethers, host code of libpfsim)
against the oracle's pure-Python restatement of buildTethers, bit for bit;
then the oracle against the reference's cloth known-answer tests
(tests/analytical/cloth/tether-*.gpu.test.ts, wind-deflection.gpu.test.ts),
with their scenes, frame loops and tolerances. The same scenes run on the
CUDA path in test_cloth_gpu.py.
"""

import math

import numpy as np
import pytest

import kat_scenes as K
from pfsim import _native as N
from pfsim import recipe as R
from pfsim import shapes


def _graph(pos, idx, pinned, density=0.2):
    return shapes.create_cloth_graph(pos, idx, density, pinned=pinned)


def _tether_cases():
    pos, idx, top = K.grid_sheet(12)
    yield "grid12-top", _graph(pos, idx, top), 4, 0.0
    pos, idx = shapes.plane_geometry(1.0, 1.0, 7, 7)
    yield "plane7-top", _graph(pos, idx, range(8)), 4, 0.0
    pos, idx = shapes.plane_geometry(1.0, 1.0, 10, 10)
    yield "plane10-two-corners", _graph(pos, idx, [0, 10]), 4, 0.0
    pos, idx = shapes.plane_geometry(1.0, 0.5, 12, 6)
    corners = [0, 12, 13 * 6, 13 * 7 - 1]
    for m in (1, 2, 4):
        yield f"plane12x6-corners-max{m}", _graph(pos, idx, corners), m, 0.06
    # islands of several pins each, and pins joined only through free particles
    yield "plane12x6-islands", _graph(pos, idx, [0, 1, 2, 5, 6, 40, 41, 54, 90]), 4, 0.1


def _random_graph(seed: int):
    """Random connected graph with small integer rest lengths (many equal
    geodesic distances, so the heap's order settles the anchors)."""
    r = np.random.default_rng(seed)
    n = 60
    pairs = [(i, int(r.integers(0, i))) for i in range(1, n)]
    while len(pairs) < 150:
        a, b = (int(x) for x in r.integers(0, n, 2))
        if a != b and (a, b) not in pairs and (b, a) not in pairs:
            pairs.append((a, b))
    rest = r.integers(1, 4, len(pairs)).astype(np.float64)
    inv = np.ones(n, np.float32)
    inv[r.choice(n, 9, replace=False)] = 0.0
    return inv, np.array(pairs, np.uint32), rest


def _same(a, b):
    for x, y in zip(a, b):
        assert x.dtype == y.dtype
        assert np.array_equal(x, y)


@pytest.mark.parametrize("case", list(_tether_cases()), ids=lambda c: c[0])
def test_tethers_native_matches_oracle(oracle, case):
    name, g, m, tol = case
    lib = shapes.build_tethers(g.inv_mass, g.pairs, g.rest_lengths, max_attachments=m, stretch_tolerance=tol)
    ref = oracle.build_tethers(g.inv_mass, g.pairs, g.rest_lengths, max_attachments=m, stretch_tolerance=tol)
    _same(lib, ref)
    assert len(lib[0]) > 0


@pytest.mark.parametrize("seed", range(6))
def test_tethers_random_graphs(oracle, seed):
    inv, pairs, rest = _random_graph(seed)
    for m in (1, 3):
        _same(shapes.build_tethers(inv, pairs, rest, max_attachments=m),
              oracle.build_tethers(inv, pairs, rest, max_attachments=m))


def test_tether_counts_and_edges():
    """tether-stretch.gpu.test.ts:170 (M x (M-1) tethers for a top-pinned
    sheet), tether-moving-pins.gpu.test.ts:68 (segments x (segments+1)),
    no pins -> no tethers (tetherBuild.ts:125), one tether per island."""
    pos, idx, top = K.grid_sheet(32)
    g = _graph(pos, idx, top)
    tp, ta, tr = shapes.build_tethers(g.inv_mass, g.pairs, g.rest_lengths)
    assert len(tp) == 32 * 31
    assert set(ta.tolist()) <= set(top)
    assert np.all(tr > 0)
    pos, idx = shapes.plane_geometry(1.0, 1.0, 7, 7)
    g = _graph(pos, idx, range(8))
    assert len(shapes.build_tethers(g.inv_mass, g.pairs, g.rest_lengths)[0]) == 7 * 8
    g = _graph(pos, idx, [])
    assert len(shapes.build_tethers(g.inv_mass, g.pairs, g.rest_lengths)[0]) == 0
    pos, idx = shapes.plane_geometry(1.0, 1.0, 10, 10)
    g = _graph(pos, idx, [0, 10])
    tp, ta, _ = shapes.build_tethers(g.inv_mass, g.pairs, g.rest_lengths)
    assert len(tp) == 2 * (121 - 2) and set(ta.tolist()) == {0, 10}
    # stretch tolerance scales every radius
    a = shapes.build_tethers(g.inv_mass, g.pairs, g.rest_lengths)[2]
    b = shapes.build_tethers(g.inv_mass, g.pairs, g.rest_lengths, stretch_tolerance=0.5)[2]
    assert np.allclose(b, a * 1.5, rtol=1e-6)
    with pytest.raises(N.PfError):
        shapes.build_tethers(g.inv_mass, g.pairs, g.rest_lengths, max_attachments=0)
    with pytest.raises(N.PfError):
        shapes.build_tethers(g.inv_mass, g.pairs, g.rest_lengths, stretch_tolerance=-1.0)


@pytest.fixture(scope="module")
def cpu(oracle):
    return oracle.OracleBackend(precision=32)


def test_aero_single_triangle(cpu):
    """aero.ts:248-283 on one free triangle in still air, zero gravity,
    moving along its normal: drag = -dragCoeff |v|^2 A v_hat, no lift
    (n x v = 0), a third on each vertex; one substep moves each predicted
    position by dt^2 w F/3 on top of x + v dt."""
    pos = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0]], np.float32)
    v = np.array([0.0, 0.0, 2.0])
    w = 0.5
    cloth = R.ClothOpts(offset=0, positions=pos, inv_mass=np.full(3, w, np.float32),
                        pairs=np.array([[0, 1], [1, 2], [2, 0]], np.uint32),
                        rest_lengths=np.array([1.0, math.sqrt(2.0), 1.0], np.float32), stretch_compliance=1e10,
                        triangles=np.array([[0, 1, 2]], np.uint32), wind=(0.0, 0.0, 0.0), drag=0.6125, lift=0.3)
    r = R.Recipe(capacity=3, radius=0.05, materials=[("cloth", cloth)],
                 loop=R.LoopOpts(substeps=1, iterations=0, gravity=(0.0, 0.0, 0.0)))
    s = cpu.build(r)
    s.write(N.PF_FIELD_VELOCITIES, np.tile(np.r_[v, 0.0], (3, 1)).astype(np.float32))
    s.step(K.DT)
    area = 0.5
    f_third = -0.6125 * 4.0 * area * np.array([0.0, 0.0, 1.0]) / 3.0
    expect = pos + v * K.DT + f_third * K.DT ** 2 * w
    got = s.readback(N.PF_FIELD_POSITIONS)[:, :3]
    assert np.allclose(got, expect, atol=2e-7), got - expect


def test_aero_lift_direction(cpu):
    """Lift = liftCoeff |v|^2 A ((n x v_hat) x v_hat): for a face at 45
    degrees to the flow, perpendicular to the flow in the (n, v) plane and
    of magnitude liftCoeff |v|^2 A cos(45 deg); drag along -v with
    magnitude dragCoeff |v|^2 A cos(45 deg)."""
    c = math.sqrt(0.5)
    pos = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, c, c]], np.float32)
    wind = (0.0, 0.0, -3.0)  # still cloth, relative flow +z
    cloth = R.ClothOpts(offset=0, positions=pos, inv_mass=np.ones(3, np.float32),
                        pairs=np.array([[0, 1], [1, 2], [2, 0]], np.uint32),
                        rest_lengths=np.array([1.0, math.sqrt(2.0), 1.0], np.float32), stretch_compliance=1e10,
                        triangles=np.array([[0, 1, 2]], np.uint32), wind=wind, drag=0.6, lift=0.4)
    r = R.Recipe(capacity=3, radius=0.05, materials=[("cloth", cloth)],
                 loop=R.LoopOpts(substeps=1, iterations=0, gravity=(0.0, 0.0, 0.0)))
    s = cpu.build(r)
    s.step(K.DT)
    p = pos.astype(np.float64)
    n = np.cross(p[1] - p[0], p[2] - p[0])
    area = 0.5 * np.linalg.norm(n)
    n /= np.linalg.norm(n)
    vrel = np.array([0.0, 0.0, 3.0])
    vh = vrel / 3.0
    nbar = n * (1.0 if n @ vrel >= 0 else -1.0)
    f = -vh * (0.6 * 9.0 * area * (nbar @ vh)) + np.cross(np.cross(nbar, vh), vh) * (0.4 * 9.0 * area)
    assert abs(np.linalg.norm(np.cross(np.cross(nbar, vh), vh)) - c) < 1e-12
    expect = p + f / 3.0 * K.DT ** 2
    got = s.readback(N.PF_FIELD_POSITIONS)[:, :3]
    assert np.allclose(got, expect, atol=2e-7)


def test_tether_unilateral(cpu):
    """tether-unilateral.gpu.test.ts:68-175: a top-pinned 12 x 12 sheet with
    its free rows pulled to half their depth, zero gravity, stretch and
    bending off (compliance 1e10), 60 frames at 4 x 2 with velocities damped
    by 0.95 each frame: no particle ends beyond its tether radius by 1e-3."""
    pos, idx, top = K.grid_sheet(12)
    g = _graph(pos, idx, top)
    init = g.positions.copy()
    free = g.inv_mass != 0
    init[free, 1] *= 0.5
    r, (tp, ta, tr) = K.cloth_system(g, 4, 2, gravity=(0.0, 0.0, 0.0), stretch=1e10, bend=1e10, positions=init)
    assert len(tp) == 12 * 11
    s = cpu.build(r)
    K.run_damped(s, 60, 0.95)
    p = s.readback(N.PF_FIELD_POSITIONS)[:, :3].astype(np.float64)
    assert np.isfinite(p).all()
    over = np.linalg.norm(p[tp] - g.positions[ta], axis=1) - tr
    assert over.max() < 1e-3


def test_tether_moving_pins(cpu):
    """tether-moving-pins.gpu.test.ts:23-74: PlaneGeometry(1, 1, 7, 7) pinned
    along its top row, zero gravity, stretch and bending off, drag and lift
    0; the pins (positions and predicted positions) move 1.5 m along +x
    before the first step; after 5 frames every free particle is within
    its tether radius (+1e-3) of its moved anchor."""
    pos, idx = shapes.plane_geometry(1.0, 1.0, 7, 7)
    g = _graph(pos, idx, range(8))
    r, (tp, ta, tr) = K.cloth_system(g, 4, 2, gravity=(0.0, 0.0, 0.0), stretch=1e10, bend=1e10, drag=0.0,
                                     lift=0.0, radius=0.02)
    assert len(tp) == 7 * 8
    s = cpu.build(r)
    pinned = g.inv_mass == 0
    for field in (N.PF_FIELD_POSITIONS, N.PF_FIELD_PREDICTED):
        a = s.readback(field)
        a[pinned, 0] += 1.5
        s.write(field, a)
    for _ in range(5):
        s.step(K.DT)
    p = s.readback(N.PF_FIELD_POSITIONS)[:, :3].astype(np.float64)
    anchors = g.positions[ta] + np.array([1.5, 0.0, 0.0])
    assert (np.linalg.norm(p[tp] - anchors, axis=1) - tr).max() < 1e-3


def _max_stretch(p, g):
    d = np.linalg.norm(p[g.pairs[:, 0]] - p[g.pairs[:, 1]], axis=1)
    return float(np.abs((d - g.rest_lengths) / g.rest_lengths).max())


def test_tether_stretch(cpu):
    """tether-stretch.gpu.test.ts:146-195: a top-pinned 32 x 32 sheet at
    100 g, 8 substeps x 4 iterations, bending compliance 1, 120 frames with
    velocities damped by 0.9: strict tethers keep every edge within 5 % of
    its rest length; with tether compliance 1e10 the sheet stretches by more
    than 20 % (or blows up)."""
    pos, idx, top = K.grid_sheet(32)
    g = _graph(pos, idx, top)
    out = {}
    for comp in (0.0, 1e10):
        r, (tp, _, _) = K.cloth_system(g, 8, 4, gravity=(0.0, -981.0, 0.0), bend=1.0, tether_compliance=comp)
        assert len(tp) == 32 * 31
        s = cpu.build(r)
        K.run_damped(s, 120, 0.9)
        p = s.readback(N.PF_FIELD_POSITIONS)[:, :3].astype(np.float64)
        out[comp] = (np.isfinite(p).all(), _max_stretch(p, g) if np.isfinite(p).all() else math.inf)
    assert out[0.0][0] and out[0.0][1] < 0.05
    assert (not out[1e10][0]) or out[1e10][1] > 0.2


def test_wind_deflection(cpu):
    """wind-deflection.gpu.test.ts:215-260: a 16 x 16 sheet (surface density
    0.2) hanging from its top row in a 1 m/s wind along +z, drag 0.6125,
    lift 0.3, stretch 1e-7, bending 1, strict tethers, 8 substeps x 4
    iterations, 240 frames with velocities damped by 0.9: the pivot-to-centre-
    of-mass angle is within 10 % of the pendulum estimate, the sheet moved
    downwind (> 1 cm) and still hangs."""
    pos, idx, top = K.grid_sheet(16, x0=-0.5)
    g = _graph(pos, idx, top)
    r, _ = K.cloth_system(g, 8, 4, bend=1.0, wind=(0.0, 0.0, 1.0))
    s = cpu.build(r)
    K.run_damped(s, 240, 0.9)
    p = s.readback(N.PF_FIELD_POSITIONS)
    assert np.isfinite(p).all()
    ang, dy, dz = K.wind_deflection_angle(p, g.inv_mass, top)
    want = K.wind_deflection_analytic(0.2, K.G, 1.0, 0.6125, 0.3)
    assert abs(math.degrees(ang) - math.degrees(want)) / math.degrees(want) < 0.1
    assert dz > 0.01 and dy < 0
