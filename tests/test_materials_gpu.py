"""Cloth, shape matching and primitive colliders on the CUDA path against the
oracle: positions after one step within 1e-5 of the container extent, a
scene alone and inside a batch bit-identical."""

import numpy as np
import pytest

from pfsim import _native as N
from pfsim import recipe as R
from pfsim import workloads as W

pytestmark = pytest.mark.gpu

DT = 1.0 / 60.0
TOL = 1e-5  # metres: 1e-5 of the 1 m container extent


@pytest.fixture(scope="module")
def cuda():
    return R.NativeBackend()


def one_frame(oracle, cuda, recipe, frames=1, precision=32):
    a = cuda.build(recipe)
    b = oracle.OracleBackend(precision=precision).build(recipe)
    for _ in range(frames):
        a.step(DT)
        b.step(DT)
    return a, b


def max_dev(a, b, field=N.PF_FIELD_POSITIONS):
    return float(np.abs(a.readback(field).astype(np.float64) - b.readback(field).astype(np.float64)).max())


@pytest.mark.parametrize("side", [64, 96])
def test_cloth_one_frame(oracle, cuda, side):
    a, b = one_frame(oracle, cuda, W.cloth_sheet(side, seed=side))
    assert max_dev(a, b) <= TOL
    # pinned top row stays put
    x0 = a.recipe.materials[0][1].positions[:side]
    np.testing.assert_array_equal(a.readback(N.PF_FIELD_POSITIONS)[:side, :3], x0)


def test_cloth_colouring_matches_oracle(oracle):
    """The host colouring is the reference's greedy colouring (same groups)."""
    from pfsim import shapes

    pos, idx = shapes.plane_geometry(1.0, 1.0, 20, 15)
    g = shapes.create_cloth_graph(pos, idx, 0.2, pinned=range(21))
    groups, k = oracle.color_constraints(g.pairs)
    deg = np.bincount(g.pairs.reshape(-1))
    assert deg.max() <= k <= 1 + 2 * (deg.max() - 1)


@pytest.mark.parametrize("mode", ["local", "global"])
def test_softbodies_one_frame(oracle, cuda, mode):
    r = W.softbody_pile(8_000, seed=4, per_body=500)
    r.materials[0][1].shape_matching = mode
    a, b = one_frame(oracle, cuda, r)
    assert max_dev(a, b) <= TOL
    if mode == "local":
        qa = a.readback(N.PF_FIELD_ROTATION)
        qb = b.readback(N.PF_FIELD_ROTATION)
        # q and -q are the same rotation
        d = np.minimum(np.abs(qa - qb).max(1), np.abs(qa + qb).max(1))
        assert d.max() < 1e-4


def test_mixed_scene_one_frame(oracle, cuda, nbr_path):
    """Fluid with dynamic soft-body boundaries (Akinci volumes and reaction),
    local shape matching and a swept sphere on a circle."""
    r = W.mixed_scene(n_budget=12_000, n_fluid=8_000, n_bodies=4, seed=1)
    a, b = one_frame(oracle, cuda, r)
    assert max_dev(a, b) <= TOL
    bv_a, bv_b = a.readback(N.PF_FIELD_BOUNDARY_VOLUME), b.readback(N.PF_FIELD_BOUNDARY_VOLUME)
    np.testing.assert_allclose(bv_a, bv_b, rtol=1e-5, atol=1e-12)


def test_mixed_scene_long_run_statistics(oracle, cuda):
    r = W.mixed_scene(n_budget=12_000, n_fluid=8_000, n_bodies=4, seed=2)
    a, b = one_frame(oracle, cuda, r, frames=30)
    xa, xb = a.readback(N.PF_FIELD_POSITIONS)[:, :3], b.readback(N.PF_FIELD_POSITIONS)[:, :3]
    assert np.isfinite(xa).all()
    assert np.abs(xa.mean(0) - xb.mean(0)).max() < 0.01


def test_box_capsule_and_inverted_colliders(oracle, cuda):
    r = W.dam_break(4000, seed=9)
    # replace the walls by an inverted (container) box, plus a capsule and a rotated box obstacle
    c = np.array([0.0, 0.4, 0.0])
    r.prims = [
        R.box(tuple(c), (0.5, 0.4, 0.3), invert=True),
        R.capsule((0.1, 0.1, -0.2), (0.1, 0.1, 0.2), 0.05),
        R.box((0.3, 0.1, 0.0), (0.05, 0.1, 0.05), rotation=(0.0, 0.3826834, 0.0, 0.9238795)),
    ]
    a, b = one_frame(oracle, cuda, r, frames=1)
    assert max_dev(a, b) <= TOL
    a2, b2 = one_frame(oracle, cuda, r, frames=20)
    x = a2.readback(N.PF_FIELD_POSITIONS)
    assert np.isfinite(x).all()
    assert np.abs(x[:, :3] - c).max() < 0.6  # the inverted box keeps the fluid in


def test_uneven_batch_matches_plain(cuda):
    recipes = [W.cloth_sheet(64, seed=1), W.dam_break(6000, seed=2, scale=1.3, offset=(5.0, 0, 0)),
               W.mixed_scene(n_budget=9_000, n_fluid=6_000, n_bodies=3, seed=3),
               W.softbody_pile(4_000, seed=4, per_body=400)]
    plain = [cuda.build(r) for r in recipes]
    batch = R.Batch([cuda.build(r) for r in recipes], use_graph=True)
    for _ in range(4):
        for s in plain:
            s.step(DT)
        batch.step(DT)
    for i, s in enumerate(plain):
        assert np.array_equal(s.readback(N.PF_FIELD_POSITIONS), batch.readback(i, N.PF_FIELD_POSITIONS)), i


def sdf_bowl_scene(seed=3):
    """A dam-break block poured into a baked hemispherical bowl (an inverted
    sphere SDF) instead of the floor plane."""
    r = W.dam_break(6000, seed=seed)
    r.prims = [p for p in r.prims if p.data0[1] != 1.0]  # drop the floor
    r.sdfs = [R.sphere_sdf((0.0, 0.55, 0.0), 0.75, res=48, invert=True, thickness=0.0)]
    return r


def test_sdf_collider_one_frame(oracle, cuda):
    a, b = one_frame(oracle, cuda, sdf_bowl_scene())
    assert max_dev(a, b) <= TOL


def test_sdf_collider_transform_update(oracle, cuda):
    """SDFCollider.setPosition between steps (pf_set_sdf_transform) on both sides."""
    import ctypes as C

    r = sdf_bowl_scene(seed=5)
    a = cuda.build(r)
    b = oracle.OracleBackend().build(r)
    a.step(DT)
    b.step(DT)
    pos = (C.c_float * 3)(0.01, 0.0, -0.005)  # a small shift of the bowl's frame
    rot = (C.c_float * 4)(0.0, 0.0, 0.0, 1.0)
    N.check(N.lib().pf_set_sdf_transform(a.h, 0, pos, rot, 1.0))
    oracle.lib().or_set_sdf_transform(b.h, 0, pos, rot, 1.0)
    a.step(DT)
    b.step(DT)
    assert max_dev(a, b) <= TOL


def test_cloth_side_stream_batch_matches_plain(cuda):
    """Cloth-only scenes batched with fluids run on the second stream of each
    substep; results stay bit-identical to the plain per-scene steps."""
    recipes = [W.cloth_sheet(64, seed=7), W.dam_break(6000, seed=8), W.cloth_sheet(48, seed=9),
               W.dam_break(3000, seed=10, scale=0.7)]
    plain = [cuda.build(r) for r in recipes]
    batch = R.Batch([cuda.build(r) for r in recipes], use_graph=True)
    for _ in range(4):
        for s in plain:
            s.step(DT)
        batch.step(DT)
    for i, s in enumerate(plain):
        assert np.array_equal(s.readback(N.PF_FIELD_POSITIONS), batch.readback(i, N.PF_FIELD_POSITIONS)), i
        assert np.array_equal(s.readback(N.PF_FIELD_VELOCITIES), batch.readback(i, N.PF_FIELD_VELOCITIES)), i


def test_surface_tension_and_adhesion_one_frame(oracle, cuda):
    """FluidSystem surfaceTension + adhesion (cohesion.ts, adhesion.ts) on the
    mixed scene, whose soft bodies are the fluid's dynamic boundaries:
    pairwise cohesion/curvature impulses and adhesion toward boundary
    particles through the velocity accumulator, before the pressure solve."""
    r = W.mixed_scene(n_budget=12_000, n_fluid=8_000, n_bodies=4, seed=21)
    r.motion = None
    fo = r.materials[1][1]
    fo.surface_tension, fo.adhesion, fo.vorticity = 0.1, 0.1, 0.02
    a, b = one_frame(oracle, cuda, r, frames=2)
    assert max_dev(a, b) <= TOL
    assert max_dev(a, b, N.PF_FIELD_DENSITY) <= 0.5  # kg/m^3, rho ~ 1000


@pytest.mark.parametrize("side", [32, 64])
def test_cloth_bending_one_frame(oracle, cuda, side):
    """Stretch and dihedral bending colours (bending.ts) against the oracle."""
    r = W.cloth_sheet(side, seed=side + 1, bend_compliance=1e-5)
    a, b = one_frame(oracle, cuda, r, frames=3)
    assert max_dev(a, b) <= TOL


def test_cloth_bending_batch_matches_plain(cuda):
    """Bending cloths batched with fluids (second stream) equal their plain steps."""
    recipes = [W.cloth_sheet(48, seed=2, bend_compliance=1e-5), W.dam_break(4000, seed=3),
               W.cloth_sheet(32, seed=4, bend_compliance=1e-4)]
    plain = [cuda.build(r) for r in recipes]
    batch = R.Batch([cuda.build(r) for r in recipes], use_graph=True)
    for _ in range(3):
        for s in plain:
            s.step(DT)
        batch.step(DT)
    for i, s in enumerate(plain):
        assert np.array_equal(s.readback(N.PF_FIELD_POSITIONS), batch.readback(i, N.PF_FIELD_POSITIONS)), i


@pytest.mark.parametrize("lanes", ["1", "2", "4", "8", "16", "32"])
def test_shape_matching_gather_lanes_same_bits(oracle, cuda, monkeypatch, lanes):
    """The shape-matching gather gives each cluster member a group of 4, 8, 16
    or 32 lanes (the world picks one from how many clusters hold its
    particles). The corrections are fixed-point ticks summed across the group,
    so every width steps to the same bits: two frames of a soft-body pile and
    of the mixed scene against the world's own choice, and the pile's first
    frame against the oracle."""
    recipes = [W.softbody_pile(8_000, seed=4, per_body=500), W.mixed_scene(n_budget=12_000, n_fluid=8_000, n_bodies=4, seed=1)]
    out = []
    for fixed in ("", lanes):
        if fixed:
            monkeypatch.setenv("PFSIM_MEMBER_LANES", fixed)
        scenes = [cuda.build(r) for r in recipes]
        frames = []
        for _ in range(2):
            for sc in scenes:
                sc.step(DT)
            frames.append([(sc.readback(N.PF_FIELD_POSITIONS), sc.readback(N.PF_FIELD_VELOCITIES)) for sc in scenes])
        out.append(frames)
    for f in range(2):
        for i in range(len(recipes)):
            assert np.array_equal(out[0][f][i][0], out[1][f][i][0]), (f, i)
            assert np.array_equal(out[0][f][i][1], out[1][f][i][1]), (f, i)
    ref = oracle.OracleBackend().build(recipes[0])
    ref.step(DT)
    assert np.abs(out[1][0][0][0] - ref.readback(N.PF_FIELD_POSITIONS)).max() <= TOL
