"""The parity workload, run exactly: 16,384 equal-mass bodies uniform in the
unit disk with circular Keplerian velocities (seeded PCG32), 32-bit Morton
keys over the bounding box, theta 0.7, Plummer eps 1e-3, leapfrog dt 1e-4,
100 steps -- with the reference's own walk (walk="exact": the per-body
monopole DFS of barnes_hut.wgsl:48-111, leaf size 1) and with the group walk
(quadrupoles, leaf buckets of 8), both against the oracle on the same inputs.

Tolerances (FP32 engine against the oracle's FP32 restatement):
  first step   Morton codes, permutation, children, parents, boxes, lengths
               bit-exact; node mass |dm| <= 1e-5 |m|, COM |dc| <= 1e-5 (|c| + L);
               accelerations: median relative error <= 1e-5, at most 1% of
               bodies above 1e-3 (criterion flips at the theta boundary from
               rsqrt vs 1/sqrt rounding and FP64-aggregated node moments).
  FP64 error   every body's acceleration against the FP64 direct sum
               (bh_direct_forces_fp64); the median must equal the oracle's
               own median error within 2% (the same algorithm, so the same
               accuracy: exact walk ~5.0e-2, group walk ~1.3e-3 at theta 0.7).
  100 steps    |dv| <= 1e-4 max|v| and |dx| <= 1e-5 (max|x| + 1).  Over
               t = 100 dt = 0.01 (a small fraction of an orbit) a force
               difference delta (relative) moves a body by ~delta |a| t^2 / 2
               and changes its velocity by ~delta |a| t; criterion flips give
               delta ~ 1e-3 for a few bodies, i.e. |dv| ~ 1e-5 with |a|, |v| ~ 1,
               and close pairs (eps = 1e-3) amplify position differences by
               at most ~e^3.5 over the run.
"""
import dataclasses

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N = 16384
SEED = 1


def _setup(bh, walk):
    wl = bh.WORKLOADS["uniform-disk-16k"]
    assert wl["n"] == N and wl["steps"] == 100
    cfg = wl["config"]
    assert (cfg.bhTheta, cfg.plummerEps, cfg.deltaTime, cfg.integrator, cfg.mortonBits,
            cfg.mortonDomain) == (0.7, 1e-3, 1e-4, "leapfrog-kdk", 32, "bbox")
    cfg = dataclasses.replace(cfg, walk=walk, leafSize=1 if walk == "exact" else cfg.leafSize)
    sim = bh.Simulation(cfg)
    sim.setNumBodies(N)
    sim.setScenario(wl["scenario"], SEED)
    return sim, wl


def _rel(acc, ref):
    num = np.linalg.norm(acc.astype(np.float64) - ref, axis=1)
    den = np.linalg.norm(ref.astype(np.float64), axis=1)
    return num / np.maximum(den, 1e-6 * np.median(den) + 1e-30)


@pytest.mark.parametrize("walk", ["exact", "group"])
def test_config0_first_step_tree_and_forces(bh, orc, walk):
    sim, _ = _setup(bh, walk)
    mass, pos, vel = sim.download()
    acc = sim.computeAccelerations()
    t = sim.tree()
    p = orc.params_from_config(sim.config)
    st = orc.State(p, mass, pos, vel)
    acc_ref = st.accelerations()
    r = st.tree()
    assert (t["codes"].astype(np.uint64) == r["codes"]).all(), "Morton codes differ"
    assert (t["ids"] == r["ids"]).all(), "sorted permutation differs"
    assert (t["parent"] == r["parent"]).all(), "parent array differs"
    assert (t["children"][:, 0] == r["left"][: N - 1]).all(), "left children differ"
    assert (t["children"][:, 1] == r["right"][: N - 1]).all(), "right children differ"
    assert (t["aabb"] == r["aabb"][: N - 1]).all(), "AABBs differ"
    assert (t["node4"][: N - 1, 3] == r["length"][: N - 1]).all(), "lengths differ"
    m_gpu, m_ref = t["node4"][:, 2], r["mass"]
    assert np.all(np.abs(m_gpu - m_ref) <= 1e-5 * np.abs(m_ref) + 1e-30)
    scale = np.abs(r["com"]).max(1) + r["length"]
    assert np.all(np.abs(t["node4"][:, :2] - r["com"]).max(1) <= 1e-5 * scale + 1e-30)
    err = _rel(acc, acc_ref)
    assert np.median(err) <= 1e-5, np.median(err)
    assert (err > 1e-3).mean() <= 0.01, (err > 1e-3).mean()
    # FP64 direct sum over every body: the engine's and the oracle's errors
    fe = sim.forceError(acc, nsample=N)
    ref64 = orc.direct_sum_fp64(p, mass, pos, np.arange(N))
    e_orc = np.linalg.norm(acc_ref - ref64, axis=1) / np.linalg.norm(ref64, axis=1)
    print(f"config 0, {walk} walk: FP64 error median {fe['median']:.3e} p99 {fe['p99']:.3e} "
          f"(oracle {np.median(e_orc):.3e})")
    assert fe["sample"] == N
    assert abs(fe["median"] - np.median(e_orc)) <= 0.02 * np.median(e_orc)
    sim.close()


@pytest.mark.parametrize("walk", ["exact", "group"])
def test_config0_100_steps_match_oracle(bh, orc, walk):
    sim, wl = _setup(bh, walk)
    mass, pos, vel = sim.download()
    st = orc.State(orc.params_from_config(sim.config), mass, pos, vel)
    sim.step(wl["steps"])
    sim.sync()
    st.step(wl["steps"])
    _, p_gpu, v_gpu = sim.download()
    p_ref, v_ref = st.state()
    dv = np.abs(v_gpu - v_ref).max()
    dx = np.abs(p_gpu - p_ref).max()
    print(f"config 0, {walk} walk, 100 steps: max |dv| {dv:.3e} (max |v| {np.abs(v_ref).max():.3f}), "
          f"max |dx| {dx:.3e}")
    assert dv <= 1e-4 * np.abs(v_ref).max()
    assert dx <= 1e-5 * (np.abs(p_ref).max() + 1.0)
    # the bodies moved (the run is not a no-op)
    assert np.abs(p_gpu - pos).max() > 1e-3
    sim.close()
