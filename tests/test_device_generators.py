"""Scenarios generated on the GPU (bh_set_scenario_device, one PCG32 stream
per body) against the oracle's restatement of the same generators.

Tolerance: every value within 1 ulp of FP32 (the formulas run in FP64; CUDA's
and the C library's double sin/cos/log/exp may differ in the last double bit,
which can move the FP32 rounding by one step); Gaussian-mixture masses within
2 ulp (their FP64 normalising total is summed in another order).
"""
import numpy as np
import pytest

NAMES = ["default", "two-clusters", "planetary-disk", "uniform-disk-kepler", "colliding-disks",
         "gaussian-mixture", "plummer-projection"]


def ulps(a, b):
    a = np.asarray(a, np.float32)
    b = np.asarray(b, np.float32)
    ia = a.view(np.int32).astype(np.int64)
    ib = b.view(np.int32).astype(np.int64)
    ia = np.where(ia < 0, -(ia & 0x7FFFFFFF), ia)
    ib = np.where(ib < 0, -(ib & 0x7FFFFFFF), ib)
    return np.abs(ia - ib)


def test_per_body_streams_keep_the_distributions(bh, orc):
    # Same distributions as the sequential host generators: compare quantiles.
    n = 200_000
    for name in ("colliding-disks", "uniform-disk-kepler", "plummer-projection", "default"):
        m1, p1, v1, _ = bh.generate_scenario(name, n, 3)
        m2, p2, v2, _ = orc.generate_per_body(name, n, 3)
        np.testing.assert_allclose(m1.sum(dtype=np.float64), m2.sum(dtype=np.float64), rtol=1e-6)
        q = [0.05, 0.25, 0.5, 0.75, 0.95]
        for a, b in ((p1, p2), (v1, v2)):
            r1 = np.quantile(np.hypot(a[:, 0], a[:, 1]), q)
            r2 = np.quantile(np.hypot(b[:, 0], b[:, 1]), q)
            np.testing.assert_allclose(r1, r2, rtol=0.02, atol=1e-3)


def test_per_body_planetary_fixed_bodies(bh, orc):
    m1, p1, v1, r1 = bh.generate_scenario("planetary-disk", 1000, 1)
    m2, p2, v2, r2 = orc.generate_per_body("planetary-disk", 1000, 1)
    assert np.array_equal(m1[:3], m2[:3]) and np.array_equal(p1[:3], p2[:3])
    assert np.array_equal(v1[:3], v2[:3]) and np.array_equal(r1, r2)


def test_mixture_duplicates_and_masses(orc):
    m, p, v, _ = orc.generate_per_body("gaussian-mixture", 100_000, 7)
    assert m.sum(dtype=np.float64) == pytest.approx(1.0, rel=1e-6)
    uniq = np.unique(p, axis=0).shape[0]
    dup = 1.0 - uniq / p.shape[0]
    assert 0.005 < dup < 0.02  # 1% of bodies copy an earlier body's coordinates
    assert (v == 0).all()


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_device_generator_matches_oracle(bh, orc, name):
    n = 50_001
    sim = bh.Simulation(bh.Config())
    sim.setNumBodies(n)
    sim.setScenarioOnDevice(name, 11)
    mass, pos, vel = sim.download()
    rad = sim.read_buffer("radius_multiplier", np.float32, n)
    rm, rp, rv, rr = orc.generate_per_body(name, n, 11)
    assert ulps(pos, rp).max() <= 1 and ulps(vel, rv).max() <= 1
    assert ulps(mass, rm).max() <= (2 if name == "gaussian-mixture" else 1)
    assert np.array_equal(rad, rr)
    # setNumBodies keeps generating on the GPU
    sim.setNumBodies(1000)
    m2, p2, v2 = sim.download()
    rm2, rp2, rv2, _ = orc.generate_per_body(name, 1000, 11)
    assert ulps(p2, rp2).max() <= 1
    sim.close()


@pytest.mark.gpu
def test_device_generator_raw_entry_and_errors(bh, orc):
    import ctypes
    import torch
    lib = bh.load()
    n = 4097
    dev = torch.device("cuda", 0)
    m = torch.empty(n, dtype=torch.float32, device=dev)
    p = torch.empty(2 * n, dtype=torch.float32, device=dev)
    v = torch.empty(2 * n, dtype=torch.float32, device=dev)
    r = torch.empty(n, dtype=torch.float32, device=dev)
    s = torch.cuda.current_stream(dev)
    rc = lib.bh_generate_scenario_device(b"colliding-disks", n, 5, 1.0,
                                         ctypes.c_void_p(m.data_ptr()), ctypes.c_void_p(p.data_ptr()),
                                         ctypes.c_void_p(v.data_ptr()), ctypes.c_void_p(r.data_ptr()),
                                         ctypes.c_void_p(s.cuda_stream))
    assert rc == 0
    torch.cuda.synchronize()
    rm, rp, rv, rr = orc.generate_per_body("colliding-disks", n, 5)
    assert ulps(p.cpu().numpy().reshape(n, 2), rp).max() <= 1
    assert lib.bh_generate_scenario_device(b"nope", n, 5, 1.0, None, None, None, None, None) == 4
    sim = bh.Simulation(bh.Config())
    with pytest.raises(bh.BhError, match="Unknown scenario: nope"):
        sim.setScenarioOnDevice("nope")
    sim.close()


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 2, 3, 7])
def test_device_generator_tiny_counts(bh, orc, n):
    for name in NAMES:
        sim = bh.Simulation(bh.Config())
        sim.setNumBodies(n)
        sim.setScenarioOnDevice(name, 4)
        mass, pos, vel = sim.download()
        rm, rp, rv, _ = orc.generate_per_body(name, n, 4)
        assert ulps(pos, rp).max() <= 1 and ulps(vel, rv).max() <= 1
        assert ulps(mass, rm).max() <= 2
        sim.close()
