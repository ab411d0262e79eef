"""Differentiable rollout: the adjoint tree walk and the reverse sweep.

CPU: the FP64 direct-sum adjoint of the oracle against central finite
differences of its own loss.
GPU: the engine's force VJP against the FP64 direct-sum VJP; the rollout
gradient (checkpoints every 20 steps, trees rebuilt on replay) against the
FP64 direct-sum adjoint at N = 4,096 and against central finite differences
of the engine's own FP32 loss (4,096 bodies and the benchmark's 65,536
bodies, both over 200 steps).
"""
import dataclasses

import numpy as np
import pytest

THETA = 0.5
EPS = 1e-3
DT = 1e-4


def adjoint_config(bh):
    return bh.Config(bhTheta=THETA, deltaTime=DT, softening="plummer", plummerEps=EPS,
                     mortonDomain="bbox", integrator="leapfrog-kdk", walk="group", leafSize=8)


def test_fp64_adjoint_matches_finite_differences(orc):
    rng = np.random.default_rng(0)
    n = 40
    pos = rng.normal(size=(n, 2)).astype(np.float32)
    vel = (0.3 * rng.normal(size=(n, 2))).astype(np.float32)
    mass = (rng.uniform(0.5, 1.5, n) / n).astype(np.float32)
    tgt = (pos + 0.01 * rng.normal(size=(n, 2))).astype(np.float32)
    p = orc.params(softening="plummer", plummer_eps=0.05, dt=1e-2)
    _, gx, gv, gm = orc.rollout_grad_fp64(p, mass, pos, vel, tgt, 8)

    def loss(m, x, v):
        return orc.rollout_grad_fp64(p, m, x, v, tgt, 8)[0]

    h = 1e-3
    for which, arr, g in (("x", pos, gx), ("v", vel, gv), ("m", mass, gm)):
        for idx in ((2, 0), (9, 1)) if which != "m" else ((2,), (9,)):
            a1, a2 = arr.copy(), arr.copy()
            a1[idx] += h
            a2[idx] -= h
            step = float(a1[idx]) - float(a2[idx])
            args = {"x": lambda a: (mass, a, vel), "v": lambda a: (mass, pos, a),
                    "m": lambda a: (a, pos, vel)}[which]
            fd = (loss(*args(a1)) - loss(*args(a2))) / step
            assert abs(fd - g[idx]) <= 1e-3 * abs(g[idx]) + 1e-9, (which, idx, fd, g[idx])


def _target(bh, n, seed, steps):
    """Target: the final positions of a rollout from velocities perturbed by N(0, 0.01^2)."""
    mass, pos, vel, _ = bh.generate_scenario("uniform-disk-kepler", n, seed)
    rng = np.random.default_rng(seed)
    vel_t = (vel + 0.01 * rng.normal(size=vel.shape)).astype(np.float32)
    sim = bh.Simulation(adjoint_config(bh))
    sim.setNumBodies(n)
    sim.upload(mass, pos, vel_t)
    sim.step(steps)
    _, tgt, _ = sim.download()
    sim.close()
    return mass, pos, vel, tgt


@pytest.mark.gpu
def test_force_vjp_matches_fp64_direct_sum(bh, orc):
    n = 4096
    mass, pos, vel, _ = bh.generate_scenario("uniform-disk-kepler", n, 3)
    sim = bh.Simulation(adjoint_config(bh))
    sim.setNumBodies(n)
    sim.upload(mass, pos, vel)
    abar = np.random.default_rng(1).normal(size=(n, 2)).astype(np.float32)
    xb, mb = sim.force_vjp(abar)
    xr, mr = orc.force_vjp_fp64(orc.params_from_config(sim.config), mass, pos, abar)
    assert np.linalg.norm(xb - xr) <= 2e-2 * np.linalg.norm(xr)
    assert np.linalg.norm(mb - mr) <= 2e-2 * np.linalg.norm(mr)
    sim.close()


@pytest.mark.gpu
def test_rollout_gradient_matches_fp64_adjoint_4096(bh, orc):
    n, steps = 4096, 200
    mass, pos, vel, tgt = _target(bh, n, 5, steps)
    sim = bh.Simulation(adjoint_config(bh))
    sim.setNumBodies(n)
    sim.upload(mass, pos, vel)
    L, gx, gv, gm = sim.rollout_grad(steps, 20, tgt)
    Lr, rx, rv, rm = orc.rollout_grad_fp64(orc.params_from_config(sim.config), mass, pos, vel, tgt,
                                          steps)
    assert abs(L - Lr) <= 1e-2 * Lr
    for name, g, r in (("x0", gx, rx), ("v0", gv, rv), ("m", gm, rm)):
        rel = float(np.linalg.norm(g - r) / np.linalg.norm(r))
        cos = float((g * r).sum() / (np.linalg.norm(g) * np.linalg.norm(r)))
        print(f"rollout gradient d/d{name} vs FP64 adjoint: relative error {rel:.3e}, cosine {cos:.8f}")
        # measured on B200: relative errors 4.4e-4 (x0), 6.5e-4 (v0), 4.8e-4 (m)
        assert rel <= 5e-3
        assert cos > 0.99999
    # the handle is left at step T
    _, p_end, _ = sim.download()
    assert np.isfinite(p_end).all()
    sim.close()


@pytest.mark.gpu
def test_rollout_gradient_split_build_equals_fused_build(bh):
    """The rollout gradient rebuilds a tree per replayed step; with the split
    build forced (what runs from 2^21 bodies) the trees, the rollout and its
    loss are the fused build's bit for bit, and the gradients agree to the
    rounding of their float atomic sums (the VJP scatters node adjoints with
    atomics, whose order varies from run to run)."""
    n, steps = 4096, 40
    mass, pos, vel, tgt = _target(bh, n, 8, steps)
    out = []
    for flags in (0, bh.BH_DEBUG_SPLIT_BUILD):
        sim = bh.Simulation(adjoint_config(bh))
        sim.setNumBodies(n)
        sim.debugSetLimits(flags=flags)
        sim.upload(mass, pos, vel)
        out.append(sim.rollout_grad(steps, 20, tgt))
        sim.close()
    (L0, *g0), (L1, *g1) = out
    assert L0 == L1
    for a, b in zip(g0, g1):
        rel = float(np.linalg.norm(a.astype(np.float64) - b) / np.linalg.norm(b.astype(np.float64)))
        assert rel <= 1e-5, rel


@pytest.mark.gpu
@pytest.mark.parametrize("n,steps,leaf", [(4096, 200, 8), (65536, 200, 4)])
def test_rollout_gradient_matches_finite_differences(bh, n, steps, leaf):
    """Central differences of the engine's own FP32 loss along one random
    direction per parameter block, sized per component: positions by 2.5e-5
    (RMS), velocities by 3e-5 / t (a velocity change dv moves a body by dv t,
    t = steps dt), masses by 1% of each mass.  The two errors of the
    estimate pull the position step both ways.  Truncation grows as the step
    squared, since close pairs at the softening length make the loss strongly
    non-linear in positions: 1,024 bodies over 40 steps gave 3.1%, 6.0% and
    83% at steps of 2.2e-5, 3e-5 and 2.2e-4, and 4,096 bodies over 200 steps
    4.8% at 3e-5, of which Richardson extrapolation removed all but 0.6%.
    The FP32 rounding noise of the loss grows as the step shrinks: at 65,536
    bodies the same extrapolation doubled the difference (2.3% -> 4.4%).
    With a velocity step as small as the position step the difference sat
    below that noise.  The 65,536-body case is the differentiable-rollout
    workload of the benchmark."""
    mass, pos, vel, tgt = _target(bh, n, 9, steps)
    cfg = dataclasses.replace(adjoint_config(bh), leafSize=leaf)
    sim = bh.Simulation(cfg)
    sim.setNumBodies(n)
    sim.upload(mass, pos, vel)
    _, gx, gv, gm = sim.rollout_grad(steps, 20, tgt)

    def loss(m, x, v):
        sim.upload(m, x, v)
        sim.step(steps)
        _, xT, _ = sim.download()
        return float(((xT.astype(np.float64) - tgt) ** 2).sum() / n)

    rng = np.random.default_rng(2)
    for which in ("x", "v", "m"):
        d = rng.normal(size=(n, 2) if which != "m" else n)
        d /= np.sqrt((d * d).mean())  # unit RMS per component
        base = {"x": pos, "v": vel, "m": mass}[which]
        if which == "x":
            step = 2.5e-5 * d
        elif which == "v":
            step = 3e-5 / (steps * DT) * d
        else:
            step = 1e-2 * d * mass
        args = {"x": lambda a: (mass, a, vel), "v": lambda a: (mass, pos, a),
                "m": lambda a: (a, pos, vel)}[which]
        g = {"x": gx, "v": gv, "m": gm}[which].astype(np.float64)

        plus = (base + step).astype(np.float32)
        minus = (base - step).astype(np.float32)
        # the step actually taken after rounding to FP32
        dd = (plus.astype(np.float64) - minus.astype(np.float64)) / 2
        fd = (loss(*args(plus)) - loss(*args(minus))) / 2
        ad = float((g * dd).sum())
        print(f"n={n} T={steps}: change along d{which}: adjoint {ad:.6e}, central FD {fd:.6e}, "
              f"relative difference {abs(fd - ad) / abs(ad):.3e}")
        assert abs(fd - ad) <= 5e-2 * abs(ad), (which, fd, ad)
    sim.close()
