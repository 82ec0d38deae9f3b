"""FrameStepper and the façade's frame-paced step() on the host (no GPU).

Restates the reference's FrameStepper cases (tests/analytical/core/
core-validation.test.ts:21-58) and the clock rules of Simulation.step
(src/simulation/Simulation.ts:542-584): 60 fixed steps per second of wall
clock, at most 4 per call, the clock restarted after a pause of over 250 ms,
and a call made while another step runs covering that frame.
"""

import threading

import pytest

from pfsim import _native as N
from pfsim.api import FrameStepper, Simulation


def pump(stepper, elapsed_ms):
    runs = []
    res = stepper.pump(1000 + elapsed_ms, lambda dt: runs.append(dt))
    return {**res, "runs": len(runs)}


@pytest.mark.parametrize("fixed_dt", [0.01, 1 / 90, 1 / 60, 1 / 30])
def test_truncated_frame_runs_the_full_cap(fixed_dt):
    s = FrameStepper(fixed_dt, max_steps_per_frame=4)
    s.pump(1000, lambda dt: None)
    r = pump(s, 1000)
    assert (r["steps"], r["runs"], r["truncated"], r["remainder_seconds"]) == (4, 4, True, 0.0)


def test_elapsed_equal_to_the_cap_is_not_truncated():
    s = FrameStepper(0.01, max_steps_per_frame=4)
    s.pump(1000, lambda dt: None)
    r = pump(s, 40)
    assert r["steps"] == 4 and not r["truncated"] and r["remainder_seconds"] < 1e-9


def test_remainder_carries_between_frames():
    s = FrameStepper(0.01)
    s.pump(1000, lambda dt: None)
    first = pump(s, 15)
    assert first["steps"] == 1
    assert first["remainder_seconds"] == pytest.approx(0.005, abs=1e-9)
    assert s.pump(1020, lambda dt: None)["steps"] == 1


def test_first_pump_starts_the_clock_and_reset_forgets():
    s = FrameStepper(0.01)
    assert s.pump(5000, lambda dt: None)["steps"] == 0
    s.reset()
    assert s.pump(9000, lambda dt: None)["steps"] == 0
    assert pump(s, 8030)["steps"] == 3


@pytest.mark.parametrize("bad", [0.0, -1.0, float("nan"), float("inf")])
def test_rejects_bad_fixed_dt(bad):
    with pytest.raises(N.PfError, match="FrameStepper: fixedDt must be positive"):
        FrameStepper(bad)


def test_rejects_bad_cap():
    with pytest.raises(N.PfError, match="maxStepsPerFrame must be a positive integer"):
        FrameStepper(0.01, max_steps_per_frame=0)


class FakeLoop:
    def __init__(self, gate=None):
        self.dts = []
        self.gate = gate

    def step(self, dt):
        if self.gate is not None:
            self.gate.wait(5)
        self.dts.append(dt)


def paced(now):
    sim = Simulation(particles=100)
    sim.loop = FakeLoop()
    sim._cloth_systems = []
    sim._clock = lambda: now[0]
    return sim


def test_step_without_dt_keeps_pace_with_the_clock():
    now = [1000.0]
    sim = paced(now)
    sim.step()  # starts the clock
    assert sim.loop.dts == []
    now[0] += 50.0  # three 1/60 s steps
    sim.step()
    assert sim.loop.dts == [pytest.approx(1 / 60)] * 3
    now[0] += 200.0  # twelve steps' worth: capped at 4, the rest dropped
    sim.step()
    assert len(sim.loop.dts) == 7
    now[0] += 400.0  # a pause: the clock restarts instead of catching up
    sim.step()
    assert len(sim.loop.dts) == 7
    now[0] += 1000.0 / 60.0
    sim.step()
    assert len(sim.loop.dts) == 8


def test_step_with_dt_advances_exactly_dt():
    sim = paced([0.0])
    sim.step(0.005)
    assert sim.loop.dts == [0.005]


def test_concurrent_step_shares_the_running_one():
    gate = threading.Event()
    sim = paced([0.0])
    sim.loop = FakeLoop(gate)
    t = threading.Thread(target=sim.step, args=(0.01,))
    t.start()
    while sim._stepping is None:
        pass
    waiter = threading.Thread(target=sim.step, args=(0.01,))
    waiter.start()
    waiter.join(0.3)  # the waiter finds the running step and waits on it
    assert waiter.is_alive()
    gate.set()
    t.join(5)
    waiter.join(5)
    assert sim.loop.dts == [0.01]
