"""FP64 diagnostics (bh_diagnostics_compute) and the JSON run log.

CPU: the oracle's FP64 sums on a two-body known answer.  GPU (marked): the
engine's diagnostics against the oracle on the same state -- moments to
1e-9 relative (FP64 sums of the same FP32 inputs, different order), the
potential to 1e-6 relative (FP32 pair terms summed in FP64); conservation
over a leapfrog run; the run log's entries.
"""
import io
import json
import math

import numpy as np
import pytest


def test_two_body_known_answer(orc):
    p = orc.params(G=2.0, dt=1e-3, softening="plummer", plummer_eps=0.5)
    mass = np.array([1.0, 3.0], np.float32)
    pos = np.array([[0.0, 0.0], [3.0, 4.0]], np.float32)
    vel = np.array([[1.0, 0.0], [0.0, -2.0]], np.float32)
    d = orc.diagnostics_fp64(p, mass, pos, vel)
    assert d["total_mass"] == 4.0
    np.testing.assert_allclose(d["com"], [2.25, 3.0])
    np.testing.assert_allclose(d["momentum"], [1.0, -6.0])
    assert d["angular_momentum"] == pytest.approx(3.0 * (3.0 * -2.0 - 4.0 * 0.0))
    assert d["kinetic_energy"] == pytest.approx(0.5 * 1.0 + 0.5 * 3.0 * 4.0)
    assert d["potential_energy"] == pytest.approx(-2.0 * 3.0 / math.sqrt(25.0 + 0.25))


def test_reference_softening_uses_pair_max_mass(orc):
    p = orc.params(G=1.0, dt=0.01, eps_mult=2.0)  # reference softening
    mass = np.array([1.0, 5.0], np.float32)
    pos = np.array([[0.0, 0.0], [1.0, 0.0]], np.float32)
    d = orc.diagnostics_fp64(p, mass, pos, np.zeros((2, 2), np.float32))
    e2 = np.float32(np.float32(2.0 * 2.0) * np.float32(1.0) * np.float32(0.01)) * 5.0
    assert d["potential_energy"] == pytest.approx(-5.0 / math.sqrt(1.0 + e2), rel=1e-7)


def _check(d, r):
    assert d["total_mass"] == pytest.approx(r["total_mass"], rel=1e-9)
    np.testing.assert_allclose(d["com"], r["com"], rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(d["momentum"], r["momentum"], rtol=1e-9, atol=1e-12)
    assert d["angular_momentum"] == pytest.approx(r["angular_momentum"], rel=1e-9, abs=1e-12)
    assert d["kinetic_energy"] == pytest.approx(r["kinetic_energy"], rel=1e-9)
    assert d["potential_energy"] == pytest.approx(r["potential_energy"], rel=1e-6)


@pytest.mark.gpu
@pytest.mark.parametrize("scenario,n,cfg", [
    ("default", 5000, {}),
    ("colliding-disks", 20000, dict(softening="plummer", plummerEps=1e-3)),
    ("planetary-disk", 3001, {}),
])
def test_diagnostics_match_oracle(bh, orc, scenario, n, cfg):
    sim = bh.Simulation(bh.Config(**cfg))
    sim.setNumBodies(n)
    sim.setScenario(scenario, 9)
    d = sim.diagnostics()
    mass, pos, vel = sim.download()
    r = orc.diagnostics_fp64(orc.params_from_config(sim.config), mass, pos, vel)
    _check(d, r)
    assert d["pairs"] == n * (n - 1) // 2
    nopot = sim.diagnostics(potential=False)
    assert "potential_energy" not in nopot
    assert nopot["kinetic_energy"] == pytest.approx(d["kinetic_energy"], rel=1e-12)  # FP64 atomics: any order
    sim.close()


@pytest.mark.gpu
def test_leapfrog_conserves_energy_and_momentum(bh):
    sim = bh.Simulation(bh.Config(walk="group", softening="plummer", plummerEps=1e-2, bhTheta=0.5,
                                  mortonDomain="bbox", integrator="leapfrog-kdk", deltaTime=1e-4))
    sim.setNumBodies(4096)
    sim.setScenario("uniform-disk-kepler", 3)
    d0 = sim.diagnostics()
    sim.step(200)
    d1 = sim.diagnostics()
    assert abs(d1["total_energy"] - d0["total_energy"]) <= 1e-3 * abs(d0["total_energy"])
    p_scale = sum(abs(x) for x in d0["momentum"]) + d0["total_mass"] * 1e-3
    assert np.abs(np.subtract(d1["momentum"], d0["momentum"])).max() <= 1e-2 * p_scale
    assert d1["total_mass"] == d0["total_mass"]
    sim.close()


@pytest.mark.gpu
def test_run_log_entries(bh):
    sim = bh.Simulation(bh.Config())
    sim.setNumBodies(2000)
    buf = io.StringIO()
    log = bh.RunLog(buf, sim, interval_s=0.0)
    for _ in range(3):
        bh.submit([sim.getCommands()])
        log.frame()
    lines = [json.loads(x) for x in buf.getvalue().splitlines()]
    assert len(lines) == 3
    for e in lines:
        for k in ("fps", "avg_frame_ms", "total_energy", "energy_drift", "momentum", "bodies"):
            assert k in e
    assert lines[0]["energy_drift"] == 0.0
    sim.close()


@pytest.mark.gpu
@pytest.mark.parametrize("n", [0, 1, 2])
def test_diagnostics_tiny_counts(bh, orc, n):
    sim = bh.Simulation(bh.Config(softening="plummer", plummerEps=1e-2))
    sim.setNumBodies(n)
    d = sim.diagnostics()
    assert d["pairs"] == n * (n - 1) // 2
    if n == 0:
        assert d["total_mass"] == 0.0 and d["potential_energy"] == 0.0
    else:
        mass, pos, vel = sim.download()
        _check(d, orc.diagnostics_fp64(orc.params_from_config(sim.config), mass, pos, vel))
    sim.close()
