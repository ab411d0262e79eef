"""The oracle against the reference's own shader logic.

tests/golden/*.npz were written by tests/golden/make_golden.py from a
mechanical C++ translation of the reference's lbvh.wgsl and barnes_hut.wgsl
(oracle/_ref/), run invocation by invocation in the reference's stage order
on the reference's three scenarios (seeded).  The oracle must reproduce them
bit for bit: Morton codes, permutation, tree arrays, node mass/COM/AABB/
length, and positions/velocities after one and after several steps.
Where the translation itself is built (the build container), random inputs
are also checked against it directly.
"""
import glob
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "ref_*.npz")))
REF = dict(G=1.0, dt=0.1 / 60.0, eps_mult=1.0, theta=0.6)


def test_fixtures_present():
    assert len(FIXTURES) >= 10


def _oracle_run(orc, mass, pos, vel, steps):
    st = orc.State(orc.params(**{"G": REF["G"], "dt": REF["dt"], "eps_mult": REF["eps_mult"],
                                 "theta": REF["theta"]}), mass, pos, vel)
    st.step(steps)
    p, v = st.state()
    return st.tree(), p, v


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p) for p in FIXTURES])
def test_oracle_matches_reference_bit_for_bit(orc, path):
    g = np.load(path)
    n = g["mass"].size
    t, p1, v1 = _oracle_run(orc, g["mass"], g["pos"], g["vel"], 1)
    ni = max(n - 1, 0)
    assert np.array_equal(t["codes"].astype(np.uint32), g["codes"])
    assert np.array_equal(t["ids"], g["ids"])
    assert np.array_equal(t["parent"], g["parent"])
    assert np.array_equal(t["left"][:ni], g["left"][:ni])
    assert np.array_equal(t["right"][:ni], g["right"][:ni])
    for k, gk in (("com", "com"), ("mass", "node_mass"), ("aabb", "aabb"), ("length", "length")):
        assert np.array_equal(t[k], g[gk]), k
    assert np.array_equal(p1, g["pos_1"]) and np.array_equal(v1, g["vel_1"])
    _, pn, vn = _oracle_run(orc, g["mass"], g["pos"], g["vel"], int(g["steps"]))
    assert np.array_equal(pn, g["pos_n"]) and np.array_equal(vn, g["vel_n"])


def test_oracle_matches_translated_reference_on_random_inputs(orc, bh):
    if not orc.ref_available():
        pytest.skip("oracle/_ref is built only where the reference checkout exists")
    rng = np.random.default_rng(11)
    for trial in range(6):
        n = int(rng.integers(2, 3000))
        scenario = ("default", "two-clusters", "planetary-disk")[trial % 3]
        mass, pos, vel, _ = bh.generate_scenario(scenario, n, int(rng.integers(1 << 30)))
        offset = int(rng.integers(n))
        r = orc.ref_run(mass, pos, vel, steps=2, offset=offset, **REF)
        t, p, v = _oracle_run(orc, mass, pos, vel, 2)
        assert np.array_equal(r["ids"], t["ids"]) and np.array_equal(r["parent"], t["parent"])
        assert np.array_equal(r["pos"], p) and np.array_equal(r["vel"], v)
