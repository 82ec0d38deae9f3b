"""The oracle against the reference's analytical known-answer tests (CPU).

Each test restates one reference test's scene, expected value and tolerance
(tests/analytical/...), runs it on the oracle, and so pins the oracle's
integrator, PBF density, XPBD distance constraint, collider contact, greedy
colouring, polar decomposition and global shape matching to the reference's
own expectations. The same scenes, but for the shape-matching ones, run on
the CUDA path in test_kat_gpu.py; the CUDA path's shape matching is held to
this oracle scene by scene.
"""

import numpy as np
import pytest

import kat_scenes as K
from pfsim import _native as N


@pytest.fixture(scope="module")
def cpu(oracle):
    return oracle.OracleBackend(precision=32)


def test_free_fall(cpu):
    """integrate-free-fall.gpu.test.ts:34-44: y after 60 steps within 1e-4 of
    the semi-implicit Euler reference."""
    s = cpu.build(K.free_fall())
    for _ in range(60):
        s.step(K.DT)
    y = float(s.readback(N.PF_FIELD_POSITIONS)[0, 1])
    assert y < 0
    assert abs(y - K.free_fall_reference(60)) < 1e-4


def test_xpbd_rigid_limit(cpu):
    """xpbd-limits.gpu.test.ts:44-77 and 140-146: alpha = 0, 4 substeps x 4
    iterations, |len - L0| < 1e-4 sampled every 25 of 1000 frames."""
    s = cpu.build(K.distance_pair(0.0, 4, 4))
    drift = 0.0
    for p, _ in K.run_trace(s, 1000, every=25):
        drift = max(drift, abs(float(np.linalg.norm(p[1, :3].astype(np.float64) - p[0, :3])) - 1.0))
    assert drift < 1e-4


def test_xpbd_soft_limit(cpu):
    """xpbd-limits.gpu.test.ts:80-131 and 149-156: alpha = 1e12 matches the
    unconstrained particle within 1e-6 over 120 frames (1 substep, 2 iterations)."""
    a = cpu.build(K.distance_pair(1e12, 1, 2))
    b = cpu.build(K.distance_pair(1e12, 1, 2, constrained=False))
    ta, tb = K.run_trace(a, 120, every=20), K.run_trace(b, 120, every=20)
    dev = max(float(np.abs(pa[1, :3] - pb[1, :3]).max()) for (pa, _), (pb, _) in zip(ta, tb))
    assert dev < 1e-6


def test_density_matches_brute_force(cpu):
    """density-pair-list-cpu-parity.gpu.test.ts:120-146: |d rho| < 5e-3 and
    |d rho| / max(rho, 1) < 1e-5 on the 5^3 lattice."""
    s = cpu.build(K.density_lattice())
    s.step(K.DT)
    rho = s.readback(N.PF_FIELD_DENSITY).astype(np.float64)
    ref = K.density_brute_force()
    d = np.abs(rho - ref)
    assert d.max() < 5e-3
    assert (d / np.maximum(ref, 1.0)).max() < 1e-5


def test_plane_rest(cpu):
    """collider-plane-rest.gpu.test.ts:36-75: settles at y = r, never below
    r - 1e-4, |vy| < 0.1 after 60 frames."""
    s = cpu.build(K.plane_rest())
    tr = K.run_trace(s, 60)
    ys = [float(p[0, 1]) for p, _ in tr]
    r = 0.05
    assert r - 1e-4 < ys[-1] < r + 5e-3
    assert abs(float(tr[-1][1][0, 1])) < 0.1
    assert min(ys) > r - 1e-4


@pytest.mark.parametrize("name,a,expected,tol", K.polar_cases(), ids=[c[0] for c in K.polar_cases()])
def test_polar_decomposition(oracle, name, a, expected, tol):
    """softbody-polar-decomp.gpu.test.ts:119-200 (FP32 oracle)."""
    r = oracle.polar(a).astype(np.float64)
    assert np.abs(r - expected).max() < tol
    if name == "rot-shear":
        assert np.abs(r @ r.T - np.eye(3)).max() < 1e-4
        assert abs(np.linalg.det(r) - 1.0) < 1e-4


def _no_conflict(pairs, groups, k):
    for g in range(k):
        sel = pairs[groups == g].reshape(-1)
        assert np.unique(sel).size == sel.size, f"group {g} shares a particle"


def test_colouring_empty(oracle):
    g, k = oracle.color_constraints(np.zeros((0, 2), np.uint32))
    assert k == 0 and g.size == 0


def test_colouring_chain(oracle):
    p = K.chain_pairs(10)
    g, k = oracle.color_constraints(p)
    assert k <= 2
    _no_conflict(p, g, k)


def test_colouring_star(oracle):
    p = K.star_pairs(8)
    g, k = oracle.color_constraints(p)
    assert k == 8
    _no_conflict(p, g, k)


def test_colouring_random(oracle):
    """xpbd-group-partition.test.ts:92-143: numGroups <= max(1, 2 maxDegree)."""
    for p in K.random_graphs():
        g, k = oracle.color_constraints(p)
        _no_conflict(p, g, k)
        deg = np.bincount(p.reshape(-1)).max()
        assert k <= max(1, 2 * deg)


def test_sdf_gradient_magnitude(oracle):
    """sdf-gradient-sanity.test.ts:20-64: |grad phi| in [0.8, 1.2] at 1000
    random points two voxels inside the grid's faces."""
    g = K.sdf_sphere_grid()
    res = g.data.shape[0]
    vs = g.voxel_size[0]
    lo = np.array(g.origin) + 2 * vs
    hi = np.array(g.origin) + (res - 2) * vs
    rand = K.lcg_js(0xDADA)
    pts = np.array([[lo[a] + (hi[a] - lo[a]) * rand() for a in range(3)] for _ in range(1000)])
    _, grad = oracle.sdf_sample(g, pts)
    mag = np.linalg.norm(grad.astype(np.float64), axis=1)
    assert mag.min() > 0.8 and mag.max() < 1.2


def test_sdf_rotated_scaled_projection(cpu):
    """sdf-rotated-scaled.gpu.test.ts:110-137: after one step no particle is
    closer than R - 5e-3 to the scaled sphere's centre."""
    rec, center, radius = K.sdf_rotated_scaled()
    s = cpu.build(rec)
    s.step(K.DT)
    d = np.linalg.norm(s.readback(N.PF_FIELD_POSITIONS)[:, :3].astype(np.float64) - center, axis=1)
    assert (d < radius - 5e-3).sum() == 0
    assert d.min() > radius - 5e-3


def test_bending_holds_rest_angle(cpu):
    """bending-rest.gpu.test.ts:250-265: a fold at 90 degrees with its edge
    pinned keeps its angle within 2 degrees over 60 frames."""
    rec, g = K.folded_quad(np.pi / 2)
    s = cpu.build(rec)
    a0 = K.signed_dihedral(g.positions)
    for _ in range(60):
        s.step(K.DT)
    p = s.readback(N.PF_FIELD_POSITIONS)
    assert np.isfinite(p).all()
    assert abs(np.degrees(K.signed_dihedral(p) - a0)) < 2.0


def test_bending_drives_toward_rest(cpu):
    """A 30-degree fold whose rest angle is flat moves toward flat (the
    reference's bending-rest test damps velocities between frames, which
    this API does not expose; here the angle must shrink within 30 frames)."""
    rec, g = K.folded_quad(np.pi / 6)
    rec.materials[0][1].bending_rest = np.zeros(1, np.float32)
    s = cpu.build(rec)
    a0 = abs(K.signed_dihedral(g.positions))
    smallest = a0
    for _ in range(30):
        s.step(K.DT)
        smallest = min(smallest, abs(K.signed_dihedral(s.readback(N.PF_FIELD_POSITIONS))))
    assert smallest < 0.5 * a0


def _shape_match(cpu, start, compliance=1e-12, iterations=1, inv_mass=1.0):
    rest = K.unit_cube_rest()
    s = cpu.build(K.shape_match_body(rest, start, compliance, iterations, inv_mass))
    s.step(K.SM_DT)
    return rest, s.readback(N.PF_FIELD_POSITIONS)[:, :3].astype(np.float64)


def _max_dist(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - np.asarray(b, np.float64), axis=1).max())


def test_shape_match_rest_is_still(cpu):
    """softbody-pass3-apply.gpu.test.ts:188-196: at rest, dx = 0 (< 1e-5)."""
    rest = K.unit_cube_rest()
    _, x = _shape_match(cpu, rest)
    assert _max_dist(x, rest) < 1e-5


def test_shape_match_rigid_translation_and_rotation(cpu):
    """softbody-pass3-apply.gpu.test.ts:198-229 (and pass2-rotation's rotated
    cases): a rigidly translated body, and one rotated by pi/4 about z, stay
    where they are (< 1e-4): the fitted frame is the rigid motion."""
    rest = K.unit_cube_rest()
    moved = rest + np.array([3.0, -1.0, 2.0], np.float32)
    _, x = _shape_match(cpu, moved)
    assert _max_dist(x, moved) < 1e-4
    rotated = (rest.astype(np.float64) @ K.rot_z(np.pi / 4).T).astype(np.float32)
    _, x = _shape_match(cpu, rotated)
    assert _max_dist(x, rotated) < 1e-4


def test_shape_match_perturbed_particle(cpu):
    """softbody-pass3-apply.gpu.test.ts:231-307: one corner moved by 0.5 in x.
    At compliance 1e-12 one iteration takes every particle to its goal under
    the frame fitted to the perturbed positions (< 1e-4); at compliance 1e-2
    (alpha / dt^2 = 576) the corner moves by under 0.05; ten iterations at
    1e-12 end at a fixed point of the fit (< 1e-5)."""
    rest = K.unit_cube_rest()
    start = rest.copy()
    start[0, 0] += 0.5
    _, x = _shape_match(cpu, start, 1e-12, 1)
    assert _max_dist(x, K.shape_match_goal(rest, start)) < 1e-4
    _, x = _shape_match(cpu, start, 1e-2, 1)
    assert abs(x[0, 0] - start[0, 0]) < 0.05
    _, x = _shape_match(cpu, start, 1e-12, 10)
    assert _max_dist(x, K.shape_match_goal(rest, x)) < 1e-5


def test_shape_match_kinematic_body(cpu):
    """softbody-pass3-apply.gpu.test.ts:309-322: particles of inverse mass 0
    are never corrected (< 1e-5), even at compliance 1e-12."""
    rest = K.unit_cube_rest()
    moved = rest + np.array([1.0, 0.0, 0.0], np.float32)
    _, x = _shape_match(cpu, moved, inv_mass=0.0)
    assert _max_dist(x, moved) < 1e-5


def test_shape_match_weights_by_mass(cpu):
    """softbody-center-of-mass.gpu.test.ts case (d) through the correction of
    softbody-pass3-apply.gpu.test.ts:231-259: with unequal masses the frame
    is fitted with mass weights (SoftbodySystem.ts:366-372), so one iteration
    at compliance 1e-12 takes the perturbed cube to the goal of the weighted
    fit (< 1e-4), and not to that of the unweighted one."""
    rest = K.unit_cube_rest()
    start = rest.copy()
    start[0, 0] += 0.5
    inv_mass = np.array([1.0, 0.5, 2.0, 1.0, 1.0, 0.25, 1.0, 1.0], np.float32)
    _, x = _shape_match(cpu, start, 1e-12, 1, inv_mass)
    weighted = K.shape_match_goal(rest, start, K.shape_match_weights(inv_mass))
    assert _max_dist(x, weighted) < 1e-4
    assert _max_dist(x, K.shape_match_goal(rest, start)) > 1e-2


def test_collider_non_penetration(cpu):
    """collider-non-penetration.gpu.test.ts:46-126: over 120 frames of 1/60 s
    no particle ends a frame with phi < -r - 5e-3 against any of the three
    colliders (the container pulls two particles into itself on the first
    substep, then all three settle on the plane inside it)."""
    s = cpu.build(K.non_penetration())
    worst = np.inf
    for _ in range(120):
        s.step(K.DT)
        worst = min(worst, float(K.non_penetration_phis(s.readback(N.PF_FIELD_POSITIONS)).min()))
    assert worst > -0.05 - 5e-3
    # and the particles did end inside the box, on the plane
    x = s.readback(N.PF_FIELD_POSITIONS)[:, :3]
    assert np.all(np.abs(x[:, 0] - 1.0) < 0.3) and np.all(np.abs(x[:, 1] - 0.05) < 0.01)


def test_rotated_box_non_penetration(cpu):
    """collider-rotated-box-non-penetration.gpu.test.ts:52-150: over 120
    frames no particle ends a frame with phi < -r - 5e-3 against the two
    tilted slabs and the rotated container (the rotated SDF and its gradient
    rotated back to world space)."""
    s = cpu.build(K.rotated_boxes())
    worst = np.inf
    for _ in range(120):
        s.step(K.DT)
        worst = min(worst, float(K.rotated_box_phis(s.readback(N.PF_FIELD_POSITIONS)).min()))
    assert worst > -0.05 - 5e-3


def test_sphere_bowl_rest(cpu):
    """collider-sphere-bowl-rest.gpu.test.ts:90-131: after 300 frames (5 s)
    every particle is inside the bowl (|x| < R - r + 5e-3), the pile has
    settled (every speed < 0.5 m/s) and no overflow flag is set."""
    s = cpu.build(K.sphere_bowl())
    for _ in range(300):
        s.step(K.DT)
    x = s.readback(N.PF_FIELD_POSITIONS)[:, :3].astype(np.float64)
    v = s.readback(N.PF_FIELD_VELOCITIES)[:, :3].astype(np.float64)
    assert np.linalg.norm(x, axis=1).max() < 1.0 - 0.05 + 5e-3
    assert np.linalg.norm(v, axis=1).max() < 0.5
    assert not any(s.overflow().values())


@pytest.mark.parametrize("alpha", [1e-2, 1e-4, 1e-6])
def test_xpbd_spring_frequency(cpu, alpha):
    """xpbd-frequency.gpu.test.ts:40-176: a pinned particle and a free one of
    mass 1 on a distance constraint of compliance alpha oscillate with period
    2 pi sqrt(alpha) within 2 %, at 20 frames per period over 10 periods, 4
    substeps and 2 iterations (8 at alpha <= 1e-5)."""
    period = 2.0 * np.pi * np.sqrt(alpha)
    frame_dt = period / 20.0
    iterations = 8 if alpha <= 1e-5 else 2
    s = cpu.build(K.spring_pair(alpha, 4, iterations))
    measured = K.spring_period(s, frame_dt, 200)
    assert abs(measured - period) / period < 0.02


def test_integrator_energy_drift(cpu):
    """integrate-energy-drift.gpu.test.ts:26-77: over 300 steps of 1/60 s the
    mean energy of 1000 free particles drifts down by semi-implicit Euler's
    1/2 g^2 dt^2 per step (-4.01 J/kg), within 0.5."""
    rec, pos, vel = K.energy_drift_cloud()
    s = cpu.build(rec)
    e0 = K.mean_energy(pos, vel)
    for _ in range(300):
        s.step(K.DT)
    e1 = K.mean_energy(s.readback(N.PF_FIELD_POSITIONS), s.readback(N.PF_FIELD_VELOCITIES))
    expected = -0.5 * K.G * K.G * K.DT * K.DT * 300
    assert e1 - e0 < 0
    assert abs((e1 - e0) - expected) < 0.5


def test_fluid_stays_in_sealed_tank(cpu):
    """mass-conservation.gpu.test.ts:79-130: after 600 frames (10 s) of the
    768-particle tank no position is NaN and none has escaped: inside the
    walls (+-0.15) and above the floor with 2r of slack, below y = 10."""
    s = cpu.build(K.sealed_tank())
    for _ in range(600):
        s.step(K.DT)
    x = s.readback(N.PF_FIELD_POSITIONS)[:, :3].astype(np.float64)
    assert np.isfinite(x).all()
    tol = 2 * 0.0125
    assert np.all(np.abs(x[:, 0]) <= 0.15 + tol) and np.all(np.abs(x[:, 2]) <= 0.15 + tol)
    assert np.all(x[:, 1] >= -tol) and np.all(x[:, 1] <= 10.0)


def test_box_container_holds_particles(cpu):
    """collider-box-container.gpu.test.ts:74-121: after 120 frames every
    particle is inside the inverted box less its radius (overrun < 2e-3),
    the pile has settled (every speed < 0.5 m/s) and no overflow flag is
    set."""
    s = cpu.build(K.box_container())
    for _ in range(120):
        s.step(K.DT)
    x = s.readback(N.PF_FIELD_POSITIONS)[:, :3].astype(np.float64)
    v = s.readback(N.PF_FIELD_VELOCITIES)[:, :3].astype(np.float64)
    overrun = np.maximum((np.abs(x) - (0.5 - 0.02)).max(1), 0.0)
    assert overrun.max() < 2e-3
    assert np.linalg.norm(v, axis=1).max() < 0.5
    assert not any(s.overflow().values())


def test_hydrostatic_column(cpu):
    """hydrostatic-column.gpu.test.ts:43-262: the 768-particle column of the
    sealed tank settles for 300 frames (5 s); its density excess over rest
    grows with depth. Over ten height bins, the middle eight's mean density
    excess against depth has a positive slope with r^2 > 0.5, and no density
    exceeds 1.1 rest density."""
    s = cpu.build(K.sealed_tank())
    for _ in range(300):
        s.step(K.DT)
    y = s.readback(N.PF_FIELD_POSITIONS)[:, 1].astype(np.float64)
    rho = s.readback(N.PF_FIELD_DENSITY).astype(np.float64)
    assert np.isfinite(y).all() and np.isfinite(rho).all()
    y0, y1 = y.min(), y.max()
    assert y1 - y0 > 0.025
    bins = 10
    idx = np.clip(np.floor((y - y0) / (y1 - y0) * bins).astype(int), 0, bins - 1)
    edges = y0 + (y1 - y0) * np.arange(bins + 1) / bins
    depth = y1 - 0.5 * (edges[:-1] + edges[1:])
    mid = [b for b in range(1, bins - 1) if np.any(idx == b)]
    assert len(mid) >= 6
    xs = depth[mid]
    ex = np.array([rho[idx == b].mean() for b in mid]) - 1000.0
    dx, dy = xs - xs.mean(), ex - ex.mean()
    sxx, sxy, syy = (dx * dx).sum(), (dx * dy).sum(), (dy * dy).sum()
    assert sxy / sxx > 0
    assert sxy * sxy / (sxx * syy) > 0.5
    assert rho.max() < 1100.0
