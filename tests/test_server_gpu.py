"""Serving (continuous batching) on the CUDA path: every request's result is
the same alone and in the mix, admission respects the HBM budget, and a
request that arrives while others run joins them without waiting for them.
"""

import numpy as np
import pytest

from pfsim import _native as N
from pfsim import recipe as R
from pfsim import workloads as W

pytestmark = pytest.mark.gpu

DT = 1.0 / 60.0
FIELDS = (N.PF_FIELD_POSITIONS, N.PF_FIELD_VELOCITIES)


def mix():
    """Small scenes of every material, with arrival ticks and lifetimes."""
    scenes = [
        (W.dam_break(3000, seed=11), 0, 9),
        (W.cloth_sheet(32, seed=12), 0, 14),
        (W.softbody_pile(3000, seed=13, per_body=300), 2, 7),
        (W.dam_break(6000, seed=14, scale=0.8), 3, 12),
        (W.mixed_scene(6000, n_fluid=3000, n_bodies=4, seed=15), 5, 6),
        (W.cloth_sheet(48, seed=16), 6, 5),
        (W.dam_break(2000, seed=17, scale=1.3), 8, 4),
    ]
    for r, _, _ in scenes:
        r.motion = None  # served scenes keep their primitives where they are
    return scenes


def alone(recipe, steps):
    s = R.NativeBackend().build(recipe)
    for _ in range(steps):
        s.step(DT)
    return [s.readback(f) for f in FIELDS]


def serve(scenes, **opts):
    srv = R.Server(**opts)
    tickets = {}
    tick = 0
    while True:
        for i, (r, arrive, life) in enumerate(scenes):
            if arrive == tick:
                tickets[i] = srv.submit(r, life)
        srv.tick(DT)
        tick += 1
        if len(tickets) == len(scenes) and all(srv.state(t)[0] == N.PF_REQ_DONE for t in tickets.values()):
            break
        if srv.stats()["live"] == 0:
            srv.drain()  # nothing to step: wait for the build in flight
        assert tick < 2000, "server did not finish"
    return srv, tickets


@pytest.fixture(scope="module")
def reference():
    return [alone(r, life) for r, _, life in mix()]


@pytest.mark.parametrize("opts", [
    dict(max_cohorts=2, async_build=True),
    dict(max_cohorts=1, async_build=False),
    dict(max_cohorts=8, async_build=True, use_graph=False),
    dict(plain=True, async_build=False),
], ids=["cohorts2-async", "cohorts1-sync", "cohorts8-nograph", "plain"])
def test_alone_equals_in_mix(reference, opts):
    scenes = mix()
    srv, tickets = serve(scenes, **opts)
    for i, (r, _, life) in enumerate(scenes):
        st, done = srv.state(tickets[i])
        assert st == N.PF_REQ_DONE and done == life
        for f, want in zip(FIELDS, reference[i]):
            got = srv.readback(tickets[i], f)
            np.testing.assert_array_equal(got, want, err_msg=f"scene {i} ({r.name}) field {f}")
    st = srv.stats()
    assert st["finished"] == len(scenes) and st["live"] == 0 and st["state_bytes"] == 0


def test_budget_admission():
    """Budget for two of the scenes: never more live than fit; all finish in
    FIFO order of admission."""
    scenes = [(W.dam_break(4000, seed=30 + i), 0, 6) for i in range(5)]
    est = R.Server.estimate_bytes(scenes[0][0])
    budget = int(2.2 * est)
    srv = R.Server(budget_bytes=budget, max_cohorts=4, async_build=False)
    tickets = [srv.submit(r, life) for r, _, life in scenes]
    admitted_at = {}
    for tick in range(200):
        srv.tick(DT)
        st = srv.stats()
        assert st["state_bytes"] <= budget
        assert st["live"] <= 2
        for t in tickets:
            if t not in admitted_at and srv.state(t)[0] != N.PF_REQ_QUEUED:
                admitted_at[t] = tick
        if st["finished"] == len(scenes):
            break
    assert srv.stats()["finished"] == len(scenes)
    order = sorted(tickets, key=lambda t: admitted_at[t])
    assert order == tickets


def test_over_budget_request_is_refused():
    r = W.dam_break(3000, seed=40)
    srv = R.Server(budget_bytes=R.Server.estimate_bytes(r) // 2)
    with pytest.raises(N.PfError):
        srv.submit(r, 3)


def test_late_arrival_joins_running_scenes():
    """A request submitted while a long one runs joins it (both live at once,
    the long one never paused), and the long one's result is unchanged."""
    long_r = W.dam_break(5000, seed=50)
    short_r = W.cloth_sheet(32, seed=51)
    life = 400
    want = alone(long_r, life)
    srv = R.Server(max_cohorts=4, async_build=True)
    t_long = srv.submit(long_r, life)
    srv.tick(DT)  # admission starts the long one's cohort build
    srv.drain()
    assert srv.state(t_long)[0] == N.PF_REQ_LIVE
    t_short = None
    joined = False
    for tick in range(4 * life):
        if tick == 5:
            t_short = srv.submit(short_r, 10)
        srv.tick(DT)
        if t_short is not None and srv.state(t_short)[0] == N.PF_REQ_LIVE:
            joined = joined or srv.state(t_long)[0] == N.PF_REQ_LIVE
        if srv.state(t_long)[0] == N.PF_REQ_DONE and t_short and srv.state(t_short)[0] == N.PF_REQ_DONE:
            break
    assert joined, "the late request never ran alongside the long one"
    assert srv.state(t_long) == (N.PF_REQ_DONE, life)
    for f, w in zip(FIELDS, want):
        np.testing.assert_array_equal(srv.readback(t_long, f), w)
