"""Particle contacts on the CUDA path: the reference's contact known-answer
tests (contact_kats.py), the pair sets against the oracle's, positions
against the oracle within 1e-5 of the container extent, a batched scene
bit-identical to its plain steps."""

import copy

import numpy as np
import pytest

import contact_kats as CK
import kat_scenes as K
from pfsim import _native as N
from pfsim import recipe as R
from pfsim import workloads as W

pytestmark = pytest.mark.gpu

DT = 1.0 / 60.0
TOL = 1e-5  # metres: 1e-5 of the 1 m container extent


@pytest.fixture(scope="module")
def cuda():
    return R.NativeBackend()


@pytest.mark.parametrize("name", list(CK.ALL))
def test_contact_kat(cuda, name):
    CK.ALL[name](cuda)


def _with_contact(r, mus=-1.0, muk=-1.0, max_contacts=0):
    r = copy.deepcopy(r)
    r.loop.contact = True
    r.loop.contact_mu_s, r.loop.contact_mu_k, r.loop.max_contacts = mus, muk, max_contacts
    return r


def _pair_set(scene):
    count, pairs = scene.contacts()
    return count, {(int(a), int(b)) for a, b in pairs}


def _scenes():
    yield "softbodies", _with_contact(W.softbody_pile(6000, seed=4, per_body=500))
    yield "mixed", _with_contact(W.mixed_scene(20000, 12000, 8, seed=5))
    yield "cloth", _with_contact(W.cloth_sheet(40, seed=6, bend_compliance=1e-5, tethers=True))
    pos, w, g = K.column_on_slab()
    yield "column", K.particles(pos, 0.025, 2, 3, inv_mass=w, group=g, contact=(2080, 0.5, 0.4))


@pytest.mark.parametrize("case", list(_scenes()), ids=lambda c: c[0])
def test_contacts_match_oracle(oracle, cuda, case):
    """The same pairs as the oracle after every frame; positions within the
    tolerance after the first frame, and within ten times it after three
    (the fluid and contact chains amplify the fast-math rounding)."""
    name, r = case
    a, b = cuda.build(r), oracle.OracleBackend(precision=32).build(r)
    for f in range(3):
        a.step(DT)
        b.step(DT)
        ca, pa = _pair_set(a)
        cb, pb = _pair_set(b)
        assert ca == cb and pa == pb, (name, f, ca, cb, len(pa ^ pb))
        dev = float(np.abs(a.readback(N.PF_FIELD_POSITIONS).astype(np.float64)
                           - b.readback(N.PF_FIELD_POSITIONS).astype(np.float64)).max())
        assert dev <= (TOL if f == 0 else 10 * TOL), (name, f, dev)
    assert not a.overflow()["contacts"]


def test_soft_bodies_get_collision_groups(oracle, cuda):
    """SoftbodySystem.build gives every body a collision group of its own
    (above the uploaded ones), so a body's particles make no pairs with each
    other; with selfCollision they do."""
    r = _with_contact(W.softbody_pile(3000, seed=7, per_body=500))
    s = cuda.build(r)
    s.step(DT)
    _, pairs = _pair_set(s)
    body = np.zeros(r.capacity, np.int64)
    for b, d in enumerate(r.materials[0][1].bodies):
        body[d.range[0]:d.range[0] + d.range[1]] = b
    assert all(body[i] != body[j] for i, j in pairs)
    r2 = copy.deepcopy(r)
    r2.materials[0][1].self_collision = True
    s2 = cuda.build(r2)
    s2.step(DT)
    _, pairs2 = _pair_set(s2)
    assert any(body[i] == body[j] for i, j in pairs2)
    o = oracle.OracleBackend(precision=32).build(r2)
    o.step(DT)
    assert _pair_set(o)[1] == pairs2


def test_contacts_batch_matches_plain(cuda):
    """Contact scenes batched with a fluid and a cloth equal their plain steps."""
    recipes = [_with_contact(W.softbody_pile(4000, seed=8, per_body=400)), W.dam_break(4000, seed=9),
               _with_contact(W.cloth_sheet(32, seed=10)), _with_contact(W.mixed_scene(12000, 8000, 4, seed=11))]
    plain = [cuda.build(r) for r in recipes]
    batch = R.Batch([cuda.build(r) for r in recipes], use_graph=True)
    for _ in range(3):
        for s in plain:
            s.step(DT)
        batch.step(DT)
    for i, s in enumerate(plain):
        for field in (N.PF_FIELD_POSITIONS, N.PF_FIELD_VELOCITIES):
            assert np.array_equal(s.readback(field), batch.readback(i, field)), (i, field)


def test_contact_budget_is_the_first_pairs(cuda):
    """Past maxContacts the first pairs in slot order are solved and the
    rest are counted: the stored pairs are a subset of the pairs found with
    a large budget, and the overflow flag is raised."""
    r = K.particles(K.lattice(5, 0.101, (0, 0.5, 0)), 0.05, 1, 2, contact=(40, 0.4, 0.3))
    big = copy.deepcopy(r)
    big.loop.max_contacts = 10000
    a, b = cuda.build(r), cuda.build(big)
    a.step(DT)
    b.step(DT)
    ca, pa = _pair_set(a)
    cb, pb = _pair_set(b)
    assert ca == cb == len(pb) and len(pa) == 40 and pa <= pb
    assert a.overflow()["contacts"] and not b.overflow()["contacts"]
