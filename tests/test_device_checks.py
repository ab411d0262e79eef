"""The engine's device-side checks, made to trip on purpose without faulting
or hanging the GPU (bh_debug_set_limits).

The reference has no such checks: its walk silently drops stack pushes
(barnes_hut.wgsl:100-105) and its sort has no bounded wait.  Here every wait
is bounded and every stack push is checked; a tripped check sets the
handle's device error word, the next synchronising call returns
BH_ERR_DEVICE_CHECK with a message, and the handle stays usable.

  look-back  the second tile of the first sort pass waits on a predecessor
             status that never reads as published; its spin cap is lowered
             so the wait runs out in milliseconds.  The step's build and walk
             then skip their work, so the bodies do not move.
  stacks     the walk stacks are capped at two entries, so the first node a
             warp opens after the root overflows them.
After each trip the limits are restored and the handle's next results are
compared bit for bit with a fresh handle's on the same state.
"""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GROUP = dict(walk="group", softening="plummer", plummerEps=1e-3, bhTheta=0.5,
             mortonDomain="bbox", leafSize=8)
N = 20000  # > one sort tile (6144 keys), so the first pass has a tile 1


def _sim(bh, **cfg):
    sim = bh.Simulation(bh.Config(**cfg))
    sim.setNumBodies(N)
    sim.setScenario("colliding-disks", 3)
    return sim


def _fresh_step(bh, cfg, state, steps=1):
    ref = bh.Simulation(bh.Config(**cfg))
    ref.setNumBodies(N)
    ref.upload(*state)
    ref.step(steps)
    out = ref.download()
    ref.close()
    return out


@pytest.mark.parametrize("graphs", [True, False])
def test_lookback_wait_runs_out_and_the_handle_recovers(bh, graphs):
    lib = bh.load()
    cfg = dict(GROUP, useGraphs=graphs)
    sim = _sim(bh, **cfg)
    state = sim.download()
    sim.debugSetLimits(flags=bh.BH_DEBUG_LOOKBACK_UNPUBLISHED, lookback_spin_cap=20000)
    t0 = time.perf_counter()
    sim.step(1)
    with pytest.raises(bh.BhError) as e:
        sim.sync()
    waited = time.perf_counter() - t0
    assert e.value.status == bh.BH_ERR_DEVICE_CHECK
    assert "look-back gave up" in str(e.value)
    assert waited < 10.0, waited  # bounded: the capped spin ends in milliseconds
    # the failed step's build and walk skipped their work: nothing moved
    after = sim.download()
    for a, b in zip(after, state):
        assert np.array_equal(a, b)
    # the word was cleared: the next synchronising call succeeds
    sim.sync()
    assert lib.bh_sync(sim._h) == 0
    # normal limits: the same step as a fresh handle's, bit for bit
    sim.debugSetLimits()
    sim.upload(*state)
    sim.step(2)
    got = sim.download()
    want = _fresh_step(bh, cfg, state, steps=2)
    for a, b in zip(got, want):
        assert np.array_equal(a, b)
    sim.close()


@pytest.mark.parametrize("walk", ["group", "exact"])
def test_walk_stack_overflow_is_reported_and_the_handle_recovers(bh, walk):
    cfg = dict(GROUP, walk=walk, leafSize=8 if walk == "group" else 1)
    sim = _sim(bh, **cfg)
    state = sim.download()
    sim.debugSetLimits(walk_stack_cap=2)
    with pytest.raises(bh.BhError) as e:
        sim.computeAccelerations()
    assert e.value.status == bh.BH_ERR_DEVICE_CHECK
    assert ("group-walk stack full" if walk == "group" else "walk stack full") in str(e.value)
    sim.debugSetLimits()
    acc = sim.computeAccelerations()
    ref = bh.Simulation(bh.Config(**cfg))
    ref.setNumBodies(N)
    ref.upload(*state)
    acc_ref = ref.computeAccelerations()
    ref.close()
    assert np.array_equal(acc, acc_ref)
    sim.close()


def test_debug_limits_reject_bad_arguments(bh):
    sim = _sim(bh, **GROUP)
    with pytest.raises(bh.BhError):
        sim.debugSetLimits(flags=1 << 7)
    with pytest.raises(bh.BhError):
        sim.debugSetLimits(walk_stack_cap=1)
    sim.close()
