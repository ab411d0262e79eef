"""Batched ensembles: many independent systems in one tree and one launch per
stage.  Every system must come out as if it had been simulated alone: the
oracle (one State per system, same parameters, bounding-box Morton domain)
gives the reference accelerations and steps.

Tolerances (FP32) match the single-system group-walk parity tests: median
relative acceleration error <= 1e-5, max <= 1e-3.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GROUP = dict(walk="group", softening="plummer", plummerEps=1e-3, bhTheta=0.5,
             mortonDomain="bbox", leafSize=8)


def acc_errors(acc, acc_ref):
    num = np.linalg.norm(acc.astype(np.float64) - acc_ref, axis=1)
    den = np.linalg.norm(acc_ref.astype(np.float64), axis=1)
    den = np.maximum(den, 1e-6 * np.median(den) + 1e-30)
    return num / den


def per_system(orc, ens, fn):
    mass, pos, vel = ens.download()
    off = ens.offsets
    p = orc.params_from_config(ens.config)
    return [fn(p, mass[off[k]:off[k + 1]], pos[off[k]:off[k + 1]], vel[off[k]:off[k + 1]])
            for k in range(len(off) - 1)]


@pytest.mark.parametrize("bpl", [1, 2, 4])
def test_ensemble_forces_match_oracle_per_system(bh, orc, bpl):
    sizes = [256, 300, 1000, 2500, 700, 5000, 257, 4096]
    ens = bh.Ensemble(sizes, bh.Config(**GROUP, bodiesPerLane=bpl))
    assert ens.numSystems() == len(sizes)
    assert list(ens.offsets) == list(np.concatenate([[0], np.cumsum(sizes)]))
    ens.setScenarios(None, seed=3)
    acc = ens.computeAccelerations()
    refs = per_system(orc, ens, lambda p, m, x, v: orc.State(p, m, x, v).accelerations())
    off = ens.offsets
    for k, ref in enumerate(refs):
        err = acc_errors(acc[off[k]:off[k + 1]], ref)
        assert np.median(err) <= 1e-5, (k, np.median(err))
        assert err.max() <= 1e-3, (k, err.max())
    ens.close()


def test_ensemble_systems_do_not_interact(bh, orc):
    # Two copies of the same system: identical accelerations, although their
    # bodies sit on top of each other in space.
    sizes = [3000, 3000]
    ens = bh.Ensemble(sizes, bh.Config(**GROUP))
    ens.setScenarios(["colliding-disks", "colliding-disks"], seed=5)
    mass, pos, vel = ens.download()
    mass[3000:], pos[3000:], vel[3000:] = mass[:3000], pos[:3000], vel[:3000]
    ens.upload(mass, pos, vel)
    acc = ens.computeAccelerations()
    assert np.array_equal(acc[:3000], acc[3000:])
    ens.close()


def test_ensemble_named_scenarios_and_errors(bh):
    ens = bh.Ensemble([400, 500], bh.Config(**GROUP))
    ens.setScenarios(["plummer-projection", "uniform-disk-kepler"], seed=1)
    with pytest.raises(bh.BhError):
        ens.setScenarios(["plummer-projection", "no-such-scenario"], seed=1)
    with pytest.raises(bh.BhError):
        ens.setNumBodies(10)
    with pytest.raises(bh.BhError):
        ens.setScenario("default")
    with pytest.raises(bh.BhError):
        ens.force_vjp(np.zeros((900, 2), np.float32))
    ens.close()
    with pytest.raises(bh.BhError):
        bh.Ensemble([100, 500], bh.Config(**GROUP))       # system below 256 bodies
    with pytest.raises(bh.BhError):
        bh.Ensemble([400, 500], bh.Config(**dict(GROUP, walk="exact")))


def test_ensemble_steps_match_oracle(bh, orc):
    sizes = [2000, 600, 3500]
    cfg = dict(GROUP, integrator="leapfrog-kdk", deltaTime=5e-5)
    ens = bh.Ensemble(sizes, bh.Config(**cfg))
    ens.setScenarios(None, seed=11)
    mass, pos0, vel0 = ens.download()
    off = ens.offsets
    p = orc.params_from_config(ens.config)
    states = [orc.State(p, mass[off[k]:off[k + 1]], pos0[off[k]:off[k + 1]],
                        vel0[off[k]:off[k + 1]]) for k in range(len(sizes))]
    ens.step(5)
    ens.sync()
    _, pos, vel = ens.download()
    for k, st in enumerate(states):
        st.step(5)
        rp, rv = st.state()
        sl = slice(off[k], off[k + 1])
        assert np.abs(vel[sl] - rv).max() <= 1e-4 * np.abs(rv).max(), k
        assert np.abs(pos[sl] - rp).max() <= 1e-5 * (np.abs(rp).max() + 1), k
    ens.close()


def test_ensemble_1024_systems_accuracy_vs_fp64(bh, orc):
    # The batched workload's distribution at reduced scale: 1,024 systems with
    # log-uniform sizes in [256, 4096], Plummer projections and uniform disks.
    sizes = bh.ensemble_sizes(1024, 7, 256, 4096)
    assert sizes.min() >= 256 and sizes.max() <= 4096
    ens = bh.Ensemble(sizes, bh.Config(**dict(GROUP, integrator="leapfrog-kdk", deltaTime=1e-4)))
    ens.setScenarios(None, seed=7)
    ens.step(3)
    acc = ens.computeAccelerations()
    mass, pos, _ = ens.download()
    off = ens.offsets
    p = orc.params_from_config(ens.config)
    rng = np.random.default_rng(0)
    errs = []
    for k in rng.choice(1024, 24, replace=False):
        sl = slice(off[k], off[k + 1])
        sample = rng.choice(off[k + 1] - off[k], 20, replace=False)
        ref = orc.direct_sum_fp64(p, mass[sl], pos[sl], sample)
        a = acc[sl][sample]
        errs.append(np.linalg.norm(a - ref, axis=1) / np.linalg.norm(ref, axis=1))
    assert np.median(np.concatenate(errs)) <= 1e-3
    assert ens.kernels_per_step() >= 5
    ens.close()


def test_ensemble_split_build_equals_fused_build(bh):
    """Large ensembles (the benchmark's 4.9e7 bodies) build their tree with
    the split build; forced on a small ensemble it gives the same tree and
    the same steps as the fused build, bit for bit."""
    sizes = [3000, 700, 5000, 12000]
    cfg = bh.Config(**dict(GROUP, integrator="symplectic-euler", deltaTime=1e-4))
    runs = []
    for flags in (0, bh.BH_DEBUG_SPLIT_BUILD):
        ens = bh.Ensemble(sizes, cfg)
        ens.setScenarios(None, seed=6)
        ens.debugSetLimits(flags=flags)
        ens.step(3)
        _, p, v = ens.download()
        t = ens.tree()
        runs.append((p, v, t["node4"], t["parent"]))
        ens.close()
    for x, y in zip(*runs):
        assert np.array_equal(x, y)
