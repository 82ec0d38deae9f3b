"""Mesh -> particle setup: the voxeliser and the SDF baker.

The oracle (CPU, doubles) against the reference's known-answer tests
(tests/analytical/softbody/softbody-voxelize.test.ts,
tests/analytical/sdf/sdf-sphere-bake-accuracy.test.ts, sdf-validation.test.ts)
on the CPU; the GPU entry points (pf_voxelize_mesh, pf_voxelize_sdf,
pf_bake_sdf) bit for bit against the oracle, and their argument checks.
"""

import math

import numpy as np
import pytest

import kat_scenes as K


def _run_kats(vox, bake):
    """The reference's expectations, for a voxeliser and a baker with the
    pfsim.mesh signatures."""
    v, i = K.unit_cube_mesh()
    res = vox(v, i, 0.1)
    # softbody-voxelize.test.ts:64-73: 125 voxels, 98 surface, 27 interior
    assert abs(res.count - 125) <= 2 and abs(res.surface_count - 98) <= 2
    assert abs(res.count - res.surface_count - 27) <= 2
    # :75-88: surface particles first (a face neighbour missing), then interior
    deg = np.bincount(res.edges.reshape(-1), minlength=res.count)
    assert np.all(deg[: res.surface_count] < 6) and np.all(deg[res.surface_count:] == 6)
    # :90-113: interior centres inside +-0.3
    assert np.all(np.abs(res.positions[res.surface_count:]) < 0.3)
    # :115-146: surface inside the box, the eight corners present
    s = res.positions[: res.surface_count]
    assert np.all(np.abs(s) <= 0.5)
    assert int(np.sum(np.all(np.abs(np.abs(s) - 0.4) < 1e-5, axis=1))) == 8
    # :148-163: a 1 x 2 x 3 slab
    slab = vox(*K.unit_cube_mesh((0.5, 1.0, 1.5)), 0.1)
    assert slab.count > 0 and 0 < slab.surface_count < slab.count

    # sdf-sphere-bake-accuracy.test.ts:34-96: 64^3 bake of a UV sphere
    # (r = 0.5, 32 x 32), 100 seeded points 3 voxels inside the grid within
    # half a voxel of |x| - 0.5
    sv, si = K.uv_sphere(0.5, 32, 32)
    data, org, vs, _ = bake(sv, si, 64, 0.1)
    rnd = K.lcg_js(0xBAAB)
    lo = org + 3 * vs
    hi = org + (64 - 3) * vs
    worst = 0.0
    for _ in range(100):
        p = [lo[a] + (hi[a] - lo[a]) * rnd() for a in range(3)]
        got = K.sample_field(data, org, (vs, vs, vs), p)
        worst = max(worst, abs(got - (math.hypot(*p) - 0.5)))
    assert worst < 0.5 * vs
    # sdf-validation.test.ts:36-52: default padding of two voxels
    d16, o16, v16, _ = bake(*K.uv_sphere(0.5, 16, 16), 16, None)
    assert abs(v16 * 16 - (1.0 + 4 * v16)) < 5e-7
    edge = np.ones_like(d16, bool)
    edge[1:-1, 1:-1, 1:-1] = False
    assert float(d16[edge].min()) > 1.4 * v16
    # :54-60: meridians on the grid diagonals do not trip the watertight check
    bake(sv, si, 32, 0.0)
    return res


def test_oracle_kats(oracle):
    from pfsim import mesh as M

    def vox(v, i, r):
        return oracle.voxelize_mesh(v, i, r)

    def bake(v, i, res, pad):
        out = oracle.bake_sdf(v, i, res, pad)
        assert out[3] <= 0.01 * res ** 3
        return out

    _run_kats(vox, bake)
    # a 2^3 field of -1 with dilation 0.01 fills (softbody-voxelize.test.ts:171-181)
    f = oracle.voxelize_sdf(np.full(8, -1.0, np.float32), (2, 2, 2), (0, 0, 0), (0.1, 0.1, 0.1), 0.05, 0.01)
    assert f.count > 0
    assert isinstance(f, M.Voxels)


@pytest.mark.gpu
def test_gpu_kats():
    from pfsim import mesh as M

    _run_kats(M.voxelize_mesh, lambda v, i, res, pad: M.bake_sdf(v, i, res, pad))


def _same_voxels(a, b):
    assert a.surface_count == b.surface_count
    assert np.array_equal(a.positions, b.positions)
    assert np.array_equal(a.edges, b.edges)


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["cube", "sphere", "torus", "torus_largest"])
def test_voxelize_mesh_matches_oracle(oracle, case):
    from pfsim import mesh as M

    if case == "cube":
        v, i, r, big = *K.unit_cube_mesh((0.5, 0.37, 0.61)), 0.03, False
    elif case == "sphere":
        v, i, r, big = *K.uv_sphere(0.5, 24, 40), 0.021, False
    else:
        v, i, r, big = *K.torus(0.4, 0.12, 48, 24), 0.017, case == "torus_largest"
    _same_voxels(M.voxelize_mesh(v, i, r, big), oracle.voxelize_mesh(v, i, r, big))


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["sphere16", "sphere32", "torus", "cube"])
def test_bake_matches_oracle(oracle, case):
    from pfsim import mesh as M

    if case.startswith("sphere"):
        n = int(case[6:])
        v, i, res, pad = *K.uv_sphere(0.5, n, n), 2 * n, None
    elif case == "torus":
        v, i, res, pad = *K.torus(0.4, 0.12, 32, 16), 40, 0.05
    else:
        v, i, res, pad = *K.unit_cube_mesh((0.3, 0.2, 0.45)), 24, 0.1
    a = M.bake_sdf(v, i, res, pad)
    b = oracle.bake_sdf(v, i, res, pad)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) and a[2] == b[2] and a[3] == b[3]


@pytest.mark.gpu
def test_voxelize_sdf_matches_oracle(oracle):
    """voxelize(SDFData) of a baked torus field, with dilation and the
    largest piece."""
    from pfsim import mesh as M

    data, org, vs, _ = M.bake_sdf(*K.torus(0.4, 0.12, 32, 16), 40, 0.05)
    args = (data, (40, 40, 40), org, (vs, vs, vs), 0.016)
    for dil, big in ((0.0, False), (0.01, True), (-0.02, False)):
        _same_voxels(M.voxelize_sdf(*args, dil, big), oracle.voxelize_sdf(*args, dil, big))


@pytest.mark.gpu
def test_argument_checks():
    """softbody-voxelize.test.ts:165-200, bake.ts:142-172 and mesh.ts:45-56."""
    from pfsim import _native as N
    from pfsim import mesh as M

    v, i = K.unit_cube_mesh()
    for r in (0.0, -0.1, float("nan")):
        with pytest.raises(N.PfError, match="particleRadius"):
            M.voxelize_mesh(v, i, r)
    with pytest.raises(N.PfError, match="indices length"):
        M.voxelize_mesh(np.zeros(3, np.float32), np.array([0, 1], np.uint32), 0.1)
    with pytest.raises(N.PfError, match="out of range"):
        M.voxelize_mesh(v, np.array([0, 1, 9], np.uint32), 0.1)
    with pytest.raises(N.PfError, match="dilation"):
        M.voxelize_sdf(np.full(8, -1.0, np.float32), (2, 2, 2), (0, 0, 0), (0.1, 0.1, 0.1), 0.05, float("nan"))
    with pytest.raises(N.PfError, match="resolution"):
        M.bake_sdf(v, i, 3)
    with pytest.raises(N.PfError, match="zero triangles"):
        M.bake_sdf(v, np.zeros(0, np.uint32), 8)
    # a box with one face missing is not watertight
    with pytest.raises(N.PfError, match="non-watertight"):
        M.bake_sdf(v, i[:-6], 16)
