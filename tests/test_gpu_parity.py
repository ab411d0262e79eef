"""GPU parity: the CUDA engine against the oracle on the same seeded inputs.

Bit-exact: Morton codes, the sorted permutation, left/right/parent arrays,
node AABBs and lengths.  Tolerances (FP32):
  node mass   |dm| <= 1e-5 |m|                    (FP64 top levels vs f32 reference)
  node COM    |dc| <= 1e-5 (|c| + length)
  acceleration (reference walk): median relative error <= 1e-5 and at most
    1% of bodies above 1e-3 (those are theta-boundary criterion flips caused
    by rsqrt vs 1/sqrt rounding; the count is reported).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SENT = 0xFFFFFFFF


def make_sim(bh, n, scenario="default", seed=1, **cfg):
    sim = bh.Simulation(bh.Config(**cfg))
    sim.setNumBodies(n)
    sim.setScenario(scenario, seed)
    return sim


def oracle_params(orc, sim):
    return orc.params_from_config(sim.config)


def compare_tree(orc, sim, check_values=True):
    n = sim.getNumBodies()
    mass, pos, vel = sim.download()
    acc = sim.computeAccelerations()
    t = sim.tree()
    st = orc.State(oracle_params(orc, sim), mass, pos, vel)
    acc_ref = st.accelerations()
    r = st.tree()
    assert (t["codes"].astype(np.uint64) == r["codes"]).all(), "Morton codes differ"
    assert (t["ids"] == r["ids"]).all(), "sorted permutation differs"
    assert (t["parent"] == r["parent"]).all(), "parent array differs"
    if n > 1:
        assert (t["children"][:, 0] == r["left"][: n - 1]).all(), "left children differ"
        assert (t["children"][:, 1] == r["right"][: n - 1]).all(), "right children differ"
        assert (t["aabb"] == r["aabb"][: n - 1]).all(), "AABBs differ"
        assert (t["node4"][: n - 1, 3] == r["length"][: n - 1]).all(), "lengths differ"
    if check_values:
        m_gpu, m_ref = t["node4"][:, 2], r["mass"]
        assert np.all(np.abs(m_gpu - m_ref) <= 1e-5 * np.abs(m_ref) + 1e-30)
        c_gpu, c_ref = t["node4"][:, :2], r["com"]
        scale = np.abs(c_ref).max(1) + r["length"]
        assert np.all(np.abs(c_gpu - c_ref).max(1) <= 1e-5 * scale + 1e-30)
    return acc, acc_ref


def node_body_counts(left, right, n):
    """Bodies under every node of the Karras numbering (internal nodes
    [0, n-2], leaves n-1+slot), from the child arrays, level by level."""
    nm1 = n - 1
    L, R = left.astype(np.int64), right.astype(np.int64)
    cnt = np.ones(2 * n - 1, np.int64)
    levels, fr = [], np.array([0])
    while fr.size:
        levels.append(fr)
        inner = fr[fr < nm1]
        fr = np.concatenate([L[inner], R[inner]])
    for lv in reversed(levels):
        inner = lv[lv < nm1]
        cnt[inner] = cnt[L[inner]] + cnt[R[inner]]
    return cnt


def acc_errors(acc, acc_ref):
    num = np.linalg.norm(acc.astype(np.float64) - acc_ref, axis=1)
    den = np.linalg.norm(acc_ref.astype(np.float64), axis=1)
    den = np.maximum(den, 1e-6 * np.median(den) + 1e-30)
    return num / den


@pytest.mark.parametrize("n", [1, 2, 3, 63, 64, 65, 1000, 4097, 20000])
def test_reference_mode_tree_and_forces(bh, orc, n):
    sim = make_sim(bh, n, "default", seed=n)
    acc, acc_ref = compare_tree(orc, sim)
    if n > 1:
        err = acc_errors(acc, acc_ref)
        assert np.median(err) <= 1e-5
        assert (err > 1e-3).mean() <= 0.01
    sim.close()


@pytest.mark.parametrize("scenario", ["two-clusters", "planetary-disk"])
def test_reference_scenarios(bh, orc, scenario):
    sim = make_sim(bh, 30000, scenario, seed=5)
    acc, acc_ref = compare_tree(orc, sim)
    err = acc_errors(acc, acc_ref)
    assert np.median(err) <= 1e-5
    assert (err > 1e-3).mean() <= 0.01
    sim.close()


@pytest.mark.parametrize("cfg", [
    dict(mortonDomain="bbox"),
    dict(mortonBits=64),
    dict(softening="plummer", plummerEps=1e-3, mortonDomain="bbox", bhTheta=0.5),
    dict(softening="plummer", plummerEps=1e-3, mortonBits=64, leafSize=8, bhTheta=0.5),
])
def test_extension_modes_tree_and_forces(bh, orc, cfg):
    sim = make_sim(bh, 20000, "colliding-disks", seed=3, **cfg)
    acc, acc_ref = compare_tree(orc, sim)
    err = acc_errors(acc, acc_ref)
    assert np.median(err) <= 1e-5
    assert (err > 1e-3).mean() <= 0.01
    sim.close()


def test_duplicates_gaussian_mixture_64bit(bh, orc):
    sim = make_sim(bh, 50000, "gaussian-mixture", seed=9, mortonBits=64, softening="plummer",
                   plummerEps=1e-4, bhTheta=0.5)
    acc, acc_ref = compare_tree(orc, sim)
    err = acc_errors(acc, acc_ref)
    assert np.median(err) <= 1e-5
    assert (err > 1e-3).mean() <= 0.01
    sim.close()


@pytest.mark.parametrize("integrator", ["symplectic-euler", "leapfrog-kdk"])
def test_steps_match_oracle(bh, orc, integrator):
    sim = make_sim(bh, 5000, "default", seed=2, integrator=integrator, mortonDomain="bbox")
    mass, pos, vel = sim.download()
    st = orc.State(oracle_params(orc, sim), mass, pos, vel)
    sim.step(3)
    sim.sync()
    st.step(3)
    _, p_gpu, v_gpu = sim.download()
    p_ref, v_ref = st.state()
    vscale = np.abs(v_ref).max()
    assert np.abs(v_gpu - v_ref).max() <= 1e-4 * vscale
    assert np.abs(p_gpu - p_ref).max() <= 1e-5 * (np.abs(p_ref).max() + 1)
    sim.close()


def test_large_tree_properties_800k(bh):
    # Full-size case: size-independent properties instead of an oracle run.
    sim = make_sim(bh, 800_000, "colliding-disks", seed=11, mortonDomain="bbox",
                   softening="plummer", bhTheta=0.5)
    mass, pos, vel = sim.download()
    sim.computeAccelerations()
    t = sim.tree()
    n = 800_000
    codes, ids = t["codes"], t["ids"]
    assert (np.diff(codes.astype(np.int64)) >= 0).all()
    assert np.array_equal(np.sort(ids), np.arange(n, dtype=np.uint32))
    # stable: equal codes keep ascending ids
    same = codes[1:] == codes[:-1]
    assert (ids[1:][same] > ids[:-1][same]).all()
    ch, par = t["children"], t["parent"]
    assert par[0] == SENT
    assert (par[ch[:, 0]] == np.arange(n - 1)).all() and (par[ch[:, 1]] == np.arange(n - 1)).all()
    cnt = np.bincount(ch.reshape(-1), minlength=2 * n - 1)
    assert cnt[0] == 0 and (cnt[1:] == 1).all()
    # mass conservation at the root (FP64 top levels)
    np.testing.assert_allclose(t["node4"][0, 2], mass.astype(np.float64).sum(), rtol=1e-6)
    sim.close()


@pytest.mark.parametrize("cfg", [
    dict(walk="group", mortonBits=64, softening="plummer", plummerEps=1e-4, bhTheta=0.5),
    dict(mortonDomain="bbox", softening="plummer", bhTheta=0.5),
], ids=["group-64bit", "reference-layout-32bit"])
def test_split_build_matches_oracle_beyond_2m(bh, orc, cfg):
    # From 2^21 bodies the build runs as a block-local kernel plus a climb of
    # the frontier nodes it leaves; both node layouts against the oracle.
    n = (1 << 21) + 4097
    sim = make_sim(bh, n, "gaussian-mixture", seed=3, **cfg)
    # reset, bbox, encode, sort passes, build (2 kernels), walk
    assert sim.kernels_per_step() == (1 + 1 + 1 + 8 + 2 + 1 if cfg.get("mortonBits") == 64
                                      else 1 + 1 + 1 + 4 + 2 + 1)
    mass, pos, vel = sim.download()
    sim.computeAccelerations()
    t = sim.tree()
    p = orc.params_from_config(sim.config)
    codes, ids = orc.morton(p, pos)
    codes, ids = orc.sort(codes, ids)
    left, right, parent = orc.build(codes, sim.config.mortonBits)
    com, mnode, aabb, length = orc.fill(ids, mass, pos, left, right, parent)
    assert (t["codes"].astype(np.uint64) == codes).all(), "Morton codes differ"
    assert (t["ids"] == ids).all(), "sorted permutation differs"
    assert (t["parent"] == parent).all(), "parent array differs"
    assert (t["children"][:, 0] == left[: n - 1]).all(), "left children differ"
    assert (t["children"][:, 1] == right[: n - 1]).all(), "right children differ"
    assert (t["aabb"] == aabb[: n - 1]).all(), "AABBs differ"
    assert (t["node4"][:, 3] == length).all(), "lengths differ"
    m_gpu = t["node4"][:, 2]
    assert np.all(np.abs(m_gpu - mnode) <= 1e-5 * np.abs(mnode) + 1e-30)
    scale = np.abs(com).max(1) + length
    assert np.all(np.abs(t["node4"][:, :2] - com).max(1) <= 1e-5 * scale + 1e-30)
    sim.close()


@pytest.mark.parametrize("n,scenario,cfg", [
    (2, "default", dict(mortonDomain="bbox", softening="plummer")),
    (3, "default", dict(walk="group", mortonDomain="bbox", softening="plummer")),
    (511, "two-clusters", dict(walk="group", mortonDomain="bbox", softening="plummer")),
    (5000, "default", dict(mortonDomain="bbox", softening="plummer")),
    (70001, "gaussian-mixture", dict(walk="group", mortonBits=64, softening="plummer",
                                     plummerEps=1e-4)),
    (300000, "colliding-disks", dict(walk="group", mortonDomain="bbox", softening="plummer")),
    (300000, "default", dict(mortonDomain="fixed2000")),   # the reference's duplicate-heavy keys
], ids=["n2", "n3", "n511", "n5000-ref-layout", "n70001-64bit", "n300k", "n300k-fixed2000"])
def test_split_build_every_size_matches_oracle(bh, orc, n, scenario, cfg):
    """The split build (block-local phase, then the device-scope climb of
    the frontier nodes it leaves) at sizes where the fused build normally
    runs: tree arrays bit for bit against the oracle."""
    sim = make_sim(bh, n, scenario, seed=2, **cfg)
    sim.debugSetLimits(flags=bh.BH_DEBUG_SPLIT_BUILD)
    bits64 = cfg.get("mortonBits") == 64
    bbox = 1 if bits64 or cfg.get("mortonDomain") == "bbox" else 0
    # reset, bbox, encode, sort passes, build (2 kernels), walk
    assert sim.kernels_per_step() == 1 + bbox + 1 + (8 if bits64 else 4) + 2 + 1
    compare_tree(orc, sim)
    sim.close()


@pytest.mark.parametrize("cfg", [
    dict(walk="group", mortonDomain="bbox", softening="plummer", plummerEps=1e-3, deltaTime=1e-3),
    dict(walk="group", mortonBits=64, softening="plummer", plummerEps=1e-4, deltaTime=1e-4,
         integrator="leapfrog-kdk"),
    dict(mortonDomain="bbox", softening="plummer", plummerEps=1e-3, deltaTime=1e-3),
], ids=["group-32bit", "group-64bit-kdk", "exact-walk"])
def test_split_build_steps_equal_fused_build(bh, cfg):
    """Node records, and so every step, are bit-identical between the fused
    build and the split build (same combine order, same FP64 rule): 200,000
    bodies over 4 steps."""
    n = 200000
    runs = []
    for flags in (0, bh.BH_DEBUG_SPLIT_BUILD):
        sim = make_sim(bh, n, "colliding-disks", seed=9, **cfg)
        sim.debugSetLimits(flags=flags)
        sim.step(4)
        m, p, v = sim.download()
        t = sim.tree()
        runs.append((p, v, t["node4"], t["aabb"], t["parent"]))
        sim.close()
    for x, y in zip(*runs):
        assert np.array_equal(x, y)


def test_headline_workload_tree_matches_oracle_800k(bh, orc):
    # The benchmark workload itself (800,000 bodies, two colliding disks,
    # 32-bit keys over the bounding box, group-walk records): every tree
    # array bit for bit against the oracle, node values within tolerance,
    # and the force error against the FP64 direct sum on 2,048 bodies.
    wl = bh.WORKLOADS["colliding-disks-800k"]
    n = wl["n"]
    sim = bh.Simulation(wl["config"])
    sim.setNumBodies(n)
    sim.setScenario(wl["scenario"], 1)
    mass, pos, vel = sim.download()
    acc = sim.computeAccelerations()
    t = sim.tree()
    p = orc.params_from_config(sim.config)
    codes, ids = orc.morton(p, pos)
    codes, ids = orc.sort(codes, ids)
    left, right, parent = orc.build(codes, sim.config.mortonBits)
    com, mnode, aabb, length = orc.fill(ids, mass, pos, left, right, parent)
    assert (t["codes"].astype(np.uint64) == codes).all(), "Morton codes differ"
    assert (t["ids"] == ids).all(), "sorted permutation differs"
    assert (t["parent"] == parent).all(), "parent array differs"
    assert (t["children"][:, 0] == left[: n - 1]).all(), "left children differ"
    assert (t["children"][:, 1] == right[: n - 1]).all(), "right children differ"
    assert (t["aabb"] == aabb[: n - 1]).all(), "AABBs differ"
    assert (t["node4"][:, 3] == length).all(), "lengths differ"
    assert np.all(np.abs(t["node4"][:, 2] - mnode) <= 1e-5 * np.abs(mnode) + 1e-30)
    scale = np.abs(com).max(1) + length
    assert np.all(np.abs(t["node4"][:, :2] - com).max(1) <= 1e-5 * scale + 1e-30)
    # Nodes below the FP64 threshold take the reference's f32 formula
    # (lbvh.wgsl:216-224) with every operation rounded as the oracle rounds
    # it, the division included: bit for bit, on every such node.
    small = node_body_counts(left, right, n) < 1024
    assert (t["node4"][small, 2] == mnode[small]).all(), "f32 node masses differ"
    assert (t["node4"][small, :2] == com[small]).all(), "f32 node centres differ"
    fe = sim.forceError(acc, nsample=2048, seed=5)
    print(f"800k group walk: FP64 error median {fe['median']:.3e} p99 {fe['p99']:.3e}")
    assert fe["median"] <= 1e-3
    sim.close()


def test_metric_workload_tree_matches_oracle_16m(bh, orc):
    # The 16.8M-body point of the metric (Gaussian mixture with 1% exact
    # duplicates, 64-bit keys, split build): every tree array bit for bit
    # against the oracle, node values within tolerance, and the force error
    # against the FP64 direct sum on 1,024 bodies.
    wl = bh.WORKLOADS["gaussian-mixture-16m"]
    n = wl["n"]
    sim = bh.Simulation(wl["config"])
    sim.setNumBodies(n)
    sim.setScenario(wl["scenario"], 1)
    mass, pos, vel = sim.download()
    acc = sim.computeAccelerations()
    t = sim.tree()
    p = orc.params_from_config(sim.config)
    codes, ids = orc.morton(p, pos)
    codes, ids = orc.sort(codes, ids)
    assert (t["codes"] == codes).all(), "Morton codes differ"
    assert (t["ids"] == ids).all(), "sorted permutation differs"
    left, right, parent = orc.build(codes, sim.config.mortonBits)
    assert (t["parent"] == parent).all(), "parent array differs"
    assert (t["children"][:, 0] == left[: n - 1]).all(), "left children differ"
    assert (t["children"][:, 1] == right[: n - 1]).all(), "right children differ"
    com, mnode, aabb, length = orc.fill(ids, mass, pos, left, right, parent)
    assert (t["aabb"] == aabb[: n - 1]).all(), "AABBs differ"
    assert (t["node4"][:, 3] == length).all(), "lengths differ"
    assert np.all(np.abs(t["node4"][:, 2] - mnode) <= 1e-5 * np.abs(mnode) + 1e-30)
    scale = np.abs(com).max(1) + length
    assert np.all(np.abs(t["node4"][:, :2] - com).max(1) <= 1e-5 * scale + 1e-30)
    fe = sim.forceError(acc, nsample=1024, seed=5)
    print(f"16.8M group walk: FP64 error median {fe['median']:.3e} p99 {fe['p99']:.3e}")
    assert fe["median"] <= 1e-3
    sim.close()


def test_direct_forces_fp64_matches_oracle(bh, orc):
    # The GPU FP64 direct sum used to measure every force error, against the
    # oracle's FP64 direct sum (both softening laws).
    for cfg in (dict(GROUP), dict(bhTheta=0.5)):
        sim = make_sim(bh, 30000, "colliding-disks" if "walk" in cfg else "default", seed=2, **cfg)
        mass, pos, _ = sim.download()
        sample = np.sort(np.random.default_rng(3).choice(30000, 500, replace=False))
        got = sim.directForcesFp64(sample)
        ref = orc.direct_sum_fp64(orc.params_from_config(sim.config), mass, pos, sample)
        rel = np.linalg.norm(got - ref, axis=1) / np.linalg.norm(ref, axis=1)
        assert rel.max() <= 1e-7, rel.max()  # FP32 sums would miss by ~1e-5
        sim.close()


def test_graph_and_direct_paths_agree(bh):
    outs = []
    for graphs in (True, False):
        sim = make_sim(bh, 10000, "two-clusters", seed=4, useGraphs=graphs)
        sim.step(4)
        sim.sync()
        outs.append(sim.download())
        sim.close()
    for a, b in zip(outs[0], outs[1]):
        assert np.array_equal(a, b)


def test_profile_and_kernel_count(bh):
    sim = make_sim(bh, 50000, "default", seed=1)
    sim.profile_begin(5)
    sim.step(5)
    ms, steps = sim.profile_end()
    assert steps == 5
    assert all(v >= 0 for v in ms.values()) and ms["walk"] > 0
    assert sim.kernels_per_step() == 1 + 1 + 4 + 1 + 1  # reset, encode, 4 sort passes, build+fill, walk
    # a second profiling window on the same captured graph
    sim.profile_begin(3)
    sim.step(3)
    ms2, steps2 = sim.profile_end()
    assert steps2 == 3 and ms2["walk"] > 0
    sim.close()


GROUP = dict(walk="group", softening="plummer", plummerEps=1e-3, bhTheta=0.5,
             mortonDomain="bbox", leafSize=8)


@pytest.mark.parametrize("bpl", [1, 2, 4])
@pytest.mark.parametrize("mp", [1, 2])
def test_group_walk_matches_oracle(bh, orc, bpl, mp):
    # Same interaction lists as the oracle up to criterion flips where a
    # node's COM (FP64-aggregated on the GPU for nodes of >= 1024 bodies)
    # differs in its last bit; values differ by rsqrt/FMA rounding.
    sim = make_sim(bh, 30000, "colliding-disks", seed=3, **dict(GROUP, multipole=mp,
                                                                bodiesPerLane=bpl))
    acc, acc_ref = compare_tree(orc, sim)
    err = acc_errors(acc, acc_ref)
    assert np.median(err) <= 1e-5
    assert err.max() <= 1e-3
    sim.close()


@pytest.mark.parametrize("n", [2, 3, 31, 33, 64, 65, 129])
def test_group_walk_small_n(bh, orc, n):
    sim = make_sim(bh, n, "uniform-disk-kepler", seed=n, **GROUP)
    acc, acc_ref = compare_tree(orc, sim)
    err = acc_errors(acc, acc_ref)
    assert err.max() <= 1e-4
    sim.close()


@pytest.mark.parametrize("bpl", [1, 2, 4])
@pytest.mark.parametrize("alpha", [0.25, 0.5])
def test_group_walk_far_field_matches_oracle(bh, orc, bpl, alpha):
    # Far nodes through the group's local expansion: the same lists and
    # expansions as the oracle's restatement (FP32 sums in another order;
    # far/near flips where a node's COM differs in its last bit), and the
    # same accuracy against the FP64 direct sum.
    sim = make_sim(bh, 30000, "colliding-disks", seed=3,
                   **dict(GROUP, bodiesPerLane=bpl, farAlpha=alpha))
    acc, acc_ref = compare_tree(orc, sim)
    err = acc_errors(acc, acc_ref)
    assert np.median(err) <= 1e-5
    assert err.max() <= 1e-3
    visits, multi, body, far = sim.walk_stats()
    assert far > 0
    mass, pos, _ = sim.download()
    fe = sim.forceError(acc, nsample=2000, seed=4)
    sample = np.sort(np.random.default_rng(4).choice(30000, 2000, replace=False))
    ref64 = orc.direct_sum_fp64(orc.params_from_config(sim.config), mass, pos, sample)
    e_orc = np.linalg.norm(acc_ref[sample] - ref64, axis=1) / np.linalg.norm(ref64, axis=1)
    assert abs(fe["median"] - np.median(e_orc)) <= 0.02 * np.median(e_orc)
    sim.close()


def test_group_walk_far_field_steps_and_ensemble(bh, orc):
    # The far field inside captured steps (leapfrog) against the oracle, and
    # on an ensemble (each group's expansion sums only its own system).
    sim = make_sim(bh, 20000, "colliding-disks", seed=8,
                   **dict(GROUP, integrator="leapfrog-kdk", deltaTime=5e-5, farAlpha=0.3))
    mass, pos, vel = sim.download()
    st = orc.State(oracle_params(orc, sim), mass, pos, vel)
    sim.step(4)
    sim.sync()
    st.step(4)
    _, p_gpu, v_gpu = sim.download()
    p_ref, v_ref = st.state()
    assert np.abs(v_gpu - v_ref).max() <= 1e-4 * np.abs(v_ref).max()
    assert np.abs(p_gpu - p_ref).max() <= 1e-5 * (np.abs(p_ref).max() + 1)
    sim.close()
    sizes = [3000, 700, 5000]
    ens = bh.Ensemble(sizes, bh.Config(**dict(GROUP, farAlpha=0.3)))
    ens.setScenarios(None, seed=3)
    m2, p2, v2 = ens.download()
    acc = ens.computeAccelerations()
    off = ens.offsets
    p = orc.params_from_config(ens.config)
    for k in range(len(sizes)):
        sl = slice(int(off[k]), int(off[k + 1]))
        ref = orc.State(p, m2[sl], p2[sl], v2[sl]).accelerations()
        e = acc_errors(acc[sl], ref)
        assert np.median(e) <= 1e-5, (k, np.median(e))
        assert e.max() <= 1e-3, (k, e.max())
    ens.close()


def test_group_walk_reference_softening(bh, orc):
    sim = make_sim(bh, 20000, "default", seed=6, walk="group", bhTheta=0.5, leafSize=4)
    acc, acc_ref = compare_tree(orc, sim)
    err = acc_errors(acc, acc_ref)
    assert np.median(err) <= 1e-5
    sim.close()


def test_group_walk_64bit_duplicates(bh, orc):
    sim = make_sim(bh, 100000, "gaussian-mixture", seed=9,
                   **dict(GROUP, mortonBits=64, plummerEps=1e-4))
    acc, acc_ref = compare_tree(orc, sim)
    err = acc_errors(acc, acc_ref)
    assert np.median(err) <= 1e-5
    assert (err > 1e-4).mean() <= 0.001
    sim.close()


def test_group_walk_accuracy_800k_vs_fp64(bh, orc):
    # The benchmark workload: median relative force error <= 1e-3 at theta 0.5.
    sim = make_sim(bh, 800_000, "colliding-disks", seed=1, **GROUP)
    mass, pos, vel = sim.download()
    acc = sim.computeAccelerations()
    sample = np.random.default_rng(0).choice(800_000, 300, replace=False)
    ref = orc.direct_sum_fp64(orc.params_from_config(sim.config), mass, pos, sample)
    err = np.linalg.norm(acc[sample] - ref, axis=1) / np.linalg.norm(ref, axis=1)
    assert np.median(err) <= 1e-3
    sim.close()


def test_group_walk_kdk_steps_match_oracle(bh, orc):
    sim = make_sim(bh, 20000, "colliding-disks", seed=8,
                   **dict(GROUP, integrator="leapfrog-kdk", deltaTime=5e-5))
    mass, pos, vel = sim.download()
    st = orc.State(oracle_params(orc, sim), mass, pos, vel)
    sim.step(4)
    sim.sync()
    st.step(4)
    _, p_gpu, v_gpu = sim.download()
    p_ref, v_ref = st.state()
    assert np.abs(v_gpu - v_ref).max() <= 1e-4 * np.abs(v_ref).max()
    assert np.abs(p_gpu - p_ref).max() <= 1e-5 * (np.abs(p_ref).max() + 1)
    sim.close()


def test_walk_stats_counts(bh):
    sim = make_sim(bh, 50000, "colliding-disks", seed=2, **GROUP)
    visits, multi, body, far = sim.walk_stats()
    assert visits > 0 and multi > 0 and body > 0 and far == 0
    sim2 = make_sim(bh, 50000, "colliding-disks", seed=2, softening="plummer", bhTheta=0.5,
                    mortonDomain="bbox")
    v2, m2, b2, f2 = sim2.walk_stats()
    assert v2 > 0 and m2 > 0 and b2 > 0 and f2 == 0
    # with the far field, far (node, group) pairs replace part of the multipole ones
    sim3 = make_sim(bh, 50000, "colliding-disks", seed=2, **dict(GROUP, farAlpha=0.25))
    v3, m3, b3, f3 = sim3.walk_stats()
    assert f3 > 0 and m3 < multi and b3 == body
    sim.close()
    sim2.close()
    sim3.close()


def test_autotune_picks_a_valid_config_and_stays_accurate(bh, orc):
    import ctypes
    sim = make_sim(bh, 100000, "colliding-disks", seed=4, **GROUP)
    mass, pos, vel = sim.download()
    r = sim.autotune(2)
    # 9 group shapes, then the other block shapes the best one allows
    assert r["candidates"] == (10 if r["bodiesPerLane"] == 4 else 11)
    assert r["walkBlock"] in ((64, 128) if r["bodiesPerLane"] == 4 else (64, 128, 256))
    assert r["bodiesPerLane"] in (1, 2, 4) and r["leafSize"] in (2, 4, 8) and r["walk_ms"] > 0
    c = bh._lib.bh_config() if hasattr(bh, "_lib") else None
    lib = bh.load()
    from importlib import import_module
    cfg = import_module("webgpu-fluid-sim_b200._lib").bh_config()
    assert lib.bh_get_config(sim._h, ctypes.byref(cfg)) == 0
    assert (cfg.bodies_per_lane, cfg.leaf_size) == (r["bodiesPerLane"], r["leafSize"])
    acc = sim.computeAccelerations()
    sample = np.random.default_rng(1).choice(100000, 200, replace=False)
    ref = orc.direct_sum_fp64(orc.params_from_config(sim.config), mass, pos, sample)
    err = np.linalg.norm(acc[sample] - ref, axis=1) / np.linalg.norm(ref, axis=1)
    assert np.median(err) <= 1e-3
    # the state did not move
    _, p2, _ = sim.download()
    assert np.array_equal(p2, pos)
    sim.close()


def test_unknown_scenario_raises(bh):
    sim = bh.Simulation()
    with pytest.raises(bh.BhError, match="Unknown scenario: nope"):
        sim.setScenario("nope")
    sim.close()
