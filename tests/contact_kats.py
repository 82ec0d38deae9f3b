"""The reference's particle-contact known-answer tests
(tests/analytical/contact/*.gpu.test.ts), each a function that builds the
test's scene on a backend (the oracle or the CUDA path), runs the test's
frame loop and checks the test's own expectations and tolerances.
"""

from __future__ import annotations

import math

import numpy as np

import kat_scenes as K
from pfsim import _native as N
from pfsim import recipe as R


def headon(backend) -> dict:
    """contact-headon.gpu.test.ts:21-96: two particles of radius 0.5 at
    x = -/+0.75 approaching at 0.5 m/s, frictionless contacts, no gravity,
    4 substeps x 8 iterations, 120 frames: never closer than 2r - 1e-3, and
    momentum conserved within 1e-4."""
    r = 0.5
    rec = K.particles([(-0.75, 0, 0), (0.75, 0, 0)], r, 4, 8, gravity=(0, 0, 0),
                      vel=[(0.5, 0, 0), (-0.5, 0, 0)], inv_mass=[1, 1], contact=(16, 0.0, 0.0))
    s = backend.build(rec)
    dmin = math.inf
    for _ in range(120):
        s.step(K.DT)
        p = s.readback(N.PF_FIELD_POSITIONS)
        dmin = min(dmin, float(np.linalg.norm(p[0, :3].astype(np.float64) - p[1, :3])))
    v = s.readback(N.PF_FIELD_VELOCITIES)
    assert dmin > 2 * r - 1e-3, dmin
    assert abs(float(v[0, 0]) + float(v[1, 0])) < 1e-4
    return {"min_distance": dmin}


def emitter_subset(backend) -> dict:
    """contact-generate-emitters.gpu.test.ts:31-145: one substep of a
    200-particle column (group 1) on a pinned 60-particle slab (group 2),
    once with every particle emitting and once with the column a
    noSelfContacts range: the same non-empty pair set."""
    pos, w, g = K.column_on_slab()
    sets = []
    for quiet in ([], [(0, 200)]):
        rec = K.particles(pos, 0.025, 1, 1, inv_mass=w, group=g, contact=(260 * 8, 0.5, 0.4), quiet=quiet)
        s = backend.build(rec)
        s.step(K.DT)
        count, pairs = s.contacts()
        assert count == len(pairs)
        sets.append({(int(a), int(b)) for a, b in pairs})
    assert len(sets[0]) > 0 and sets[0] == sets[1]
    assert all(a < 200 <= b for a, b in sets[0])  # every pair is (column, slab)
    return {"pairs": sets[0]}


def overflow(backend) -> dict:
    """contact-overflow.gpu.test.ts:28-94: a 5 x 5 x 5 lattice at 2r x 1.01
    with maxContacts 16: the last substep's count exceeds 16 (and the
    overflow flag reports it); ten more frames leave every position finite."""
    r = 0.05
    rec = K.particles(K.lattice(5, 2 * r * 1.01, (0, 0.5, 0)), r, 2, 2, contact=(16, 0.4, 0.3))
    s = backend.build(rec)
    s.step(K.DT)
    count, pairs = s.contacts()
    assert count > 16 and len(pairs) <= 16
    assert s.overflow()["contacts"]
    for _ in range(10):
        s.step(K.DT)
    assert np.isfinite(s.readback(N.PF_FIELD_POSITIONS)).all()
    return {"count": count}


def single_on_floor(backend) -> dict:
    """contact-single-on-floor.gpu.test.ts:16-82: one particle (r = 0.05)
    dropped from 6r onto a plane (muS 0.6, muK 0.5) with contacts on, 4 x 4,
    60 frames: rests at y in (r - 1e-3, r + 5e-3) with |vy| < 0.1."""
    r = 0.05
    rec = K.particles([(0, 6 * r, 0)], r, 4, 4, inv_mass=[1], contact=(64, 0.6, 0.5),
                      prims=[R.plane((0, 1, 0), (0, 0, 0), 0.6, 0.5)])
    s = backend.build(rec)
    for _ in range(60):
        s.step(K.DT)
    y = float(s.readback(N.PF_FIELD_POSITIONS)[0, 1])
    vy = float(s.readback(N.PF_FIELD_VELOCITIES)[0, 1])
    assert r - 1e-3 < y < r + 5e-3, y
    assert abs(vy) < 0.1
    return {"y": y}


def small_cluster(backend) -> dict:
    """contact-small-cluster.gpu.test.ts:16-98: a 3 x 3 x 3 cluster at
    spacing 3r from y = 4r onto a plane (muS 0.5, muK 0.4), contacts
    (512, 0.5, 0.4), 4 x 4, 90 frames: lowest centre above r - 2e-3, every
    speed below 1 m/s."""
    r = 0.05
    rec = K.particles(K.lattice(3, 3 * r, (0, 4 * r, 0)), r, 4, 4, contact=(512, 0.5, 0.4),
                      prims=[R.plane((0, 1, 0), (0, 0, 0), 0.5, 0.4)])
    s = backend.build(rec)
    for _ in range(90):
        s.step(K.DT)
    p = s.readback(N.PF_FIELD_POSITIONS)
    v = s.readback(N.PF_FIELD_VELOCITIES)
    assert float(p[:, 1].min()) > r - 2e-3
    assert float(np.linalg.norm(v[:, :3], axis=1).max()) < 1.0
    return {"min_y": float(p[:, 1].min())}


def non_interpenetration(backend) -> dict:
    """contact-non-interpenetration.gpu.test.ts:21-116: a 3 x 3 x 3 cluster
    at 2r x 1.05 from y = 0.5 onto the floor (default friction), contacts
    (256, 0.4, 0.3), 4 x 4, 90 frames: after every frame no pair is closer
    than 2r - 2e-3."""
    r = 0.05
    rec = K.particles(K.lattice(3, 2 * r * 1.05, (0, 0.5, 0)), r, 4, 4, contact=(256, 0.4, 0.3),
                      prims=[R.plane((0, 1, 0), (0, 0, 0))])
    s = backend.build(rec)
    worst = -math.inf
    for _ in range(90):
        s.step(K.DT)
        worst = max(worst, K.pair_overlap(s.readback(N.PF_FIELD_POSITIONS), 2 * r))
    assert worst < 2e-3, worst
    return {"worst_overlap": worst}


def incline(backend, kinetic: bool) -> dict:
    """contact-two-ball-inclined.gpu.test.ts:26-139: two particles resting on
    a plane (muS 0.6, muK 0.5) under gravity tilted by atan(muS) -/+ 3 deg,
    contacts on: below the cone neither moves 1e-3 m in 5 s; above it both
    slide 1/2 a t^2 (a = g (sin t - muK cos t)) within 15 % in 2 s."""
    r, mus, muk = 0.05, 0.6, 0.5
    th = math.atan(mus) + (1 if kinetic else -1) * math.radians(3)
    seconds = 2.0 if kinetic else 5.0
    rec = K.particles([(-0.2, r, 0), (0.2, r, 0)], r, 4, 4, inv_mass=[1, 1], contact=(8, mus, muk),
                      gravity=(K.G * math.sin(th), -K.G * math.cos(th), 0.0),
                      prims=[R.plane((0, 1, 0), (0, 0, 0), mus, muk)])
    s = backend.build(rec)
    for _ in range(math.ceil(seconds / K.DT)):
        s.step(K.DT)
    x = s.readback(N.PF_FIELD_POSITIONS)[:, 0].astype(np.float64)
    d = x - np.array([-0.2, 0.2])
    if kinetic:
        want = 0.5 * K.G * (math.sin(th) - muk * math.cos(th)) * seconds ** 2
        assert np.all(d > 0.85 * want) and np.all(d < 1.15 * want), (d, want)
    else:
        assert float(np.abs(d).max()) < 1e-3
    return {"dx": d}


ALL = {
    "headon": headon,
    "emitter_subset": emitter_subset,
    "overflow": overflow,
    "single_on_floor": single_on_floor,
    "small_cluster": small_cluster,
    "non_interpenetration": non_interpenetration,
    "incline_static": lambda b: incline(b, False),
    "incline_kinetic": lambda b: incline(b, True),
}
