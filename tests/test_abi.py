"""CPU checks of the C-ABI library: it loads, exports every symbol that
include/bh.h declares, and its host-only entry points work without a GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for f in os.listdir(os.path.join(ROOT, "include")):
        if f.endswith(".h"):
            src = open(os.path.join(ROOT, "include", f)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names |= set(re.findall(r"\b(bh_[a-z0-9_]+)\s*\(", src))
    return sorted(names)


def test_header_declares_core_entry_points():
    names = declared_symbols()
    for must in ("bh_create", "bh_destroy", "bh_set_num_bodies", "bh_set_scenario", "bh_step",
                 "bh_get_buffers", "bh_get_num_bodies", "bh_upload", "bh_download"):
        assert must in names


def test_library_exports_every_declared_symbol(bh):
    lib = bh.load()
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_every_declared_symbol(bh):
    from importlib import import_module
    sigs = import_module("webgpu-fluid-sim_b200._lib").SIGNATURES
    assert set(declared_symbols()) <= set(sigs)


def test_default_config_matches_config_ts(bh):
    lib = bh.load()
    c = import_lib().bh_config()
    assert lib.bh_default_config(ctypes.byref(c)) == 0
    assert c.grav_constant == 1.0
    assert abs(c.bh_theta - 0.6) < 1e-7
    assert c.substeps == 1
    assert c.delta_time == np.float32(0.1 / 60.0)
    assert c.epsilon_multiplier == 1.0
    py = bh.getDefaultConfig().to_c()
    assert py.delta_time == c.delta_time and py.bh_theta == c.bh_theta


def import_lib():
    from importlib import import_module
    return import_module("webgpu-fluid-sim_b200._lib")


def test_version_string(bh):
    assert b"sm_100a" in bh.load().bh_version()


def test_generate_scenarios_host_only(bh):
    for name in bh.SCENARIOS:
        mass, pos, vel, rad = bh.generate_scenario(name, 1001, seed=3)
        assert np.isfinite(mass).all() and np.isfinite(pos).all() and np.isfinite(vel).all()
        assert (mass >= 0).all()
    # deterministic for a seed, different across seeds
    a = bh.generate_scenario("default", 100, seed=1)[1]
    b = bh.generate_scenario("default", 100, seed=1)[1]
    c = bh.generate_scenario("default", 100, seed=2)[1]
    assert np.array_equal(a, b) and not np.array_equal(a, c)


def test_reference_scenario_shapes(bh):
    mass, pos, vel, rad = bh.generate_scenario("default", 5000, seed=0)
    assert (mass == 1.0).all() and np.hypot(*pos.T).max() <= 5.0 + 1e-5    # simulation.ts:245-249
    mass, pos, vel, rad = bh.generate_scenario("two-clusters", 5000, seed=0)
    assert (pos[:2500, 0] < 0).all() and (pos[2500:, 0] > 0).all()        # :283-289
    mass, pos, vel, rad = bh.generate_scenario("planetary-disk", 5000, seed=0)
    assert mass[0] == 1000.0 and mass[1] == 10.0 and mass[2] == 10.0         # :316-339
    assert rad[0] == 12.0 and rad[1] == 5.0 and rad[2] == 5.0
    np.testing.assert_allclose(mass[3:], 1000.0 / (100.0 * 5000), rtol=1e-6)
    r = np.hypot(*pos[3:].T)
    assert r.min() >= 0.1 - 1e-5 and r.max() <= 15.0 + 1e-5


def test_benchmark_scenarios(bh):
    mass, pos, vel, _ = bh.generate_scenario("gaussian-mixture", 100000, seed=4)
    np.testing.assert_allclose(mass.astype(np.float64).sum(), 1.0, rtol=1e-5)
    dup = len(pos) - len(np.unique(pos, axis=0))
    assert 0.005 * len(pos) < dup < 0.02 * len(pos)  # ~1% exact duplicates
    mass, pos, vel, _ = bh.generate_scenario("colliding-disks", 100000, seed=4)
    np.testing.assert_allclose(mass.astype(np.float64).sum(), 1.0, rtol=1e-5)
    assert pos[0].tolist() == [1.5, 0.0] and pos[50000].tolist() == [-1.5, 0.0]


def test_unknown_scenario_is_an_error(bh):
    with pytest.raises(bh.BhError, match="Unknown scenario: galaxy"):
        bh.generate_scenario("galaxy", 10)


def test_create_without_gpu_fails_loudly(bh):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(bh.BhError):
        bh.Simulation()
