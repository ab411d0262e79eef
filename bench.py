"""Benchmark: Barnes-Hut body-steps/s on the seeded colliding-disks workload.

Workload (default): N = 800,000 bodies, two colliding exponential disks,
theta = 0.5, Plummer eps = 1e-3, dt = 5e-5, the reference's symplectic Euler
integrator, 32-bit Morton keys over the bounding box.  One "step" = one full
pipeline pass (Morton, sort, build + fill, walk + kick + drift) over all
bodies.

Own arm (default):
  value      body-steps/s with the state resident in HBM, K steps timed with
             CUDA events on the engine's stream; L2 (126 MB) is flushed
             between timed steps (flush outside the timed events).
  e2e        the same metric through the public API with host buffers: per
             step upload(mass, pos, vel) from page-locked memory, one step,
             download(pos, vel) into page-locked memory -- pipelined (the
             download asynchronous, one sync after the loop); the same loop
             with every download waiting is reported beside it ("serial").
  roofline   the dominant kernel (walk), from per-stage CUDA events recorded
             in the step graph during the timed steps.
  cpu_baseline  the oracle (C restatement, OpenMP, all host threads) on a
             bounded sample of the same workload.
  secondary  the 16.8M-body Gaussian-mixture point of the metric with the
             same figures (value, stages, roofline, e2e, force error,
             cpu_baseline).
Reference arm (--impl reference): the reference's own pipeline logic on the
host cores: its WGSL compute shaders mechanically translated to C++
(oracle/_ref, built where the reference checkout exists), all host threads;
if that build is absent, the oracle port.  The WGSL itself needs a WebGPU
device, which this machine lacks.  W untimed steps, then exactly K timed
steps, each a bounded sample of the workload (the walk on every k-th sorted
slot, scaled by k, when a whole step would not fit the run's few minutes).
That arm imports nothing from the engine package: its inputs come from the
oracle's generators.

Both arms print the same `config` (the workload, the parallelism and the
cache treatment); the own arm's implementation choices (key width, walk
shape, autotuning) are in its `engine` object.

Multi-GPU (torchrun): by default one system on all ranks (--shard: every
rank builds the same tree, walks its range of sorted slots, and the ranks
all-gather the updated bodies once per step: strong scaling); --replicas
runs an independently seeded copy per rank instead (weak scaling, no
collective).  The timed region is bracketed by barriers and the max over
ranks is reported.
"""
from __future__ import annotations

import argparse
import dataclasses
import importlib
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
PKG = "webgpu-fluid-sim_b200"
DEFAULT_WORKLOAD = "colliding-disks-800k"
FLUSH_BYTES = 256 << 20  # > 126 MB L2
# DRAM bytes (read + write) of one launch of the dominant kernel (the walk),
# from one ncu capture of the same workload; the 16.8M point from a capture
# of its 4.2M-body case (same generator and settings, 1.364 GB) scaled by
# the bodies processed.
NCU_WALK_TRAFFIC_BYTES = {"colliding-disks-800k": 72.04e6,  # far-field walk, 128-body groups
                          "gaussian-mixture-4m": 1.364e9,
                          "gaussian-mixture-16m": 1.364e9 * 4.0}
# Algorithmic HBM bytes per body and step of the stream stages: encode =
# position 8 + mass 4 read, key 4|8 + packed leaf record 16 written; sort =
# first pass key read + key and id written, later passes key and id read and
# written; build = key 4|8 + id 4 + leaf gather 16 read, leaf record 16 +
# parents 8 + one 64-B internal-node record written.
STREAM_BYTES = {4: {"morton": 8 + 4 + 4 + 16, "sort": 12 + 3 * 16, "tree": 4 + 4 + 16 + 16 + 8 + 64},
                8: {"morton": 8 + 4 + 8 + 16, "sort": 20 + 7 * 24, "tree": 8 + 4 + 16 + 16 + 8 + 64}}
# Plain parameters of the workloads for the CPU legs, which must not import
# the engine package: body count, scenario and the oracle's parameters
# (oracle.params keywords).  tests/test_bench.py checks them against the
# package's WORKLOADS.
def _orc_params(theta, eps, dt, bits, domain, integrator, far_alpha=0.0):
    return dict(G=1.0, dt=dt, theta=theta, softening="plummer", plummer_eps=eps,
                morton_bits=bits, morton_domain=domain, integrator=integrator, leaf_size=8,
                walk="group", multipole=2, bodies_per_lane=2, far_alpha=far_alpha)


REF_WORKLOADS = {
    "uniform-disk-16k": dict(n=16384, scenario="uniform-disk-kepler",
                             oracle=_orc_params(0.7, 1e-3, 1e-4, 32, "bbox", "leapfrog-kdk")),
    "colliding-disks-800k": dict(n=800_000, scenario="colliding-disks",
                                 oracle=_orc_params(0.5, 1e-3, 5e-5, 32, "bbox",
                                                    "symplectic-euler", 0.4)),
    "gaussian-mixture-16m": dict(n=16_777_216, scenario="gaussian-mixture",
                                 oracle=_orc_params(0.5, 1e-4, 1e-5, 64, "fixed2000",
                                                    "symplectic-euler", 0.4)),
    "gaussian-mixture-4m": dict(n=4_194_304, scenario="gaussian-mixture",
                                oracle=_orc_params(0.5, 1e-4, 1e-5, 64, "fixed2000",
                                                   "symplectic-euler", 0.4)),
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="own", choices=["own", "reference"])
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--walk-shape", default=None, metavar="BPL,LEAF",
                    help="pin the group walk's bodies_per_lane and leaf size (no autotuner): "
                         "profiling runs use the shape a plain run picked")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-secondary", action="store_true")
    ap.add_argument("--no-ensemble", action="store_true")
    ap.add_argument("--no-render", action="store_true")
    ap.add_argument("--no-exact-walk", action="store_true")
    ap.add_argument("--shard", action="store_true",
                    help="one system on all ranks (strong scaling); the default with N > 1")
    ap.add_argument("--replicas", action="store_true",
                    help="with N > 1: an independently seeded copy of the workload per rank")
    return ap.parse_args()


def adjoint_cost(pkg, device: int, n: int = 65536, steps: int = 200, every: int = 20) -> dict:
    """Differentiable-rollout cost: N = 65,536 uniform disk, theta 0.5, eps 1e-3,
    dt 1e-4, T = 200 leapfrog steps, checkpoints every 20; the target is the
    rollout from velocities perturbed by N(0, 0.01^2).  Reports adjoint time /
    forward-rollout time and the speed-up over a central finite-difference
    gradient (2 rollouts per parameter, 5 parameters per body)."""
    cfg = pkg.Config(bhTheta=0.5, deltaTime=1e-4, softening="plummer", plummerEps=1e-3,
                     mortonDomain="bbox", integrator="leapfrog-kdk", walk="group", leafSize=4)
    mass, pos, vel, _ = pkg.generate_scenario("uniform-disk-kepler", n, 3)
    sim = pkg.Simulation(cfg, device=device)
    sim.setNumBodies(n)
    rng = np.random.default_rng(0)
    sim.upload(mass, pos, (vel + 0.01 * rng.normal(size=vel.shape)).astype(np.float32))
    sim.step(steps)
    _, tgt, _ = sim.download()
    best_f, best_a = 1e30, 1e30
    for _ in range(3):
        sim.upload(mass, pos, vel)
        sim.sync()
        t0 = time.perf_counter()
        sim.step(steps)
        sim.sync()
        best_f = min(best_f, time.perf_counter() - t0)
        sim.upload(mass, pos, vel)
        sim.sync()
        t0 = time.perf_counter()
        loss, _, _, _ = sim.rollout_grad(steps, every, tgt)
        best_a = min(best_a, time.perf_counter() - t0)
    sim.close()
    fd = best_f * 2 * 5 * n
    return {"bodies": n, "steps": steps, "checkpoint_every": every, "forward_s": best_f,
            "adjoint_s": best_a, "adjoint_over_forward": best_a / best_f,
            "fd_gradient_s_estimate": fd, "speedup_vs_fd": fd / best_a, "loss": loss,
            "timing": "host wall clock around synchronised calls, best of 3"}


FAR_PAIR_FLOPS = 435.0  # one node's local coefficients (far_field.cuh, counted from the code)
FAR_BODY_FLOPS = 50.0   # one body's local-expansion evaluation


def walk_roofline(cfg, walk_ms: float, multi_inter: int, body_inter: int, visits: int,
                  sm_max_mhz, traffic=None, far_pairs: int = 0, n: int = 0) -> dict:
    """Roofline of the walk: algorithmic FP32 flops per launch over its time,
    against the nominal FP32 FMA rate.  Flops: 16 per monopole interaction
    (2 sub, 3 for d^2+eps^2, 4 for rsqrt, 2 for inv^3, 1 for m inv^3, 4 for
    two FMA) and 35 per monopole + quadrupole interaction (the 16 plus Q'r 6,
    r.Q'r 3, inv^5 1, 2.5 r.Q'r inv^7 3, two extra FMA 4, one add 2), times
    the interactions an instrumented launch of the same walk counts; with the
    far field, 435 per (far node, group) pair (local coefficients of orders
    1-4: 79 polynomial terms of kernel derivatives up to order 6 at 3 flops,
    14 coefficients at 12, set-up 30) and 50 per body for the expansion's
    evaluation."""
    quad = cfg.walk == "group" and cfg.multipole >= 2
    flops = (35.0 if quad else 16.0) * multi_inter + 16.0 * body_inter
    if far_pairs:
        flops += FAR_PAIR_FLOPS * far_pairs + FAR_BODY_FLOPS * n
    mhz = sm_max_mhz or 1965.0
    fp32_peak = 148 * 128 * 2 * mhz * 1e6 / 1e12  # nominal FMA peak at max clock
    achieved = flops / (walk_ms / 1e3) / 1e12
    return {"bound": "fp32", "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
            "frac": achieved / fp32_peak, "traffic": traffic,
            "traffic_unit": "bytes per launch (ncu dram read + write)",
            "peak_source": "nominal FP32 FMA rate (148 SMs x 128 lanes x 2 x max SM clock);"
                           " no measured FP32 peak exists for this pool",
            "kernel": "walk", "kernel_ms": walk_ms,
            "multipole_interactions_per_step": multi_inter,
            "body_interactions_per_step": body_inter,
            "far_node_group_pairs_per_step": far_pairs,
            "node_visits_per_step": visits, "flops_per_step": flops}


def stream_rooflines(stages: dict, n: int, key_bytes: int, hbm_gbs: float) -> dict:
    """HBM fraction of each stream stage: its algorithmic bytes over its time."""
    out = {}
    for stage, per_body in STREAM_BYTES[key_bytes].items():
        ms = stages.get(stage, 0.0)
        if ms <= 0.0:
            continue
        gbs = per_body * n / (ms / 1e3) / 1e9
        out[stage] = {"bytes_per_body": per_body, "ms": ms, "achieved_gbs": gbs,
                      "peak_gbs": hbm_gbs, "frac": gbs / hbm_gbs}
    return out


def e2e_rate(sim, step, n: int, steps: int, ext, barrier=lambda: None, dist=None, units=None):
    """The metric through the public API with host buffers: every step
    uploads masses, positions and velocities from page-locked memory, runs
    one step and downloads positions and velocities into page-locked memory.
    Two loops over the same calls, CUDA events on the engine's stream around
    each: pipelined (the download is asynchronous and nothing waits inside
    the loop, so step k's download and step k+1's position upload overlap
    the neighbouring steps; one sync after the loop, inside the events) and
    serial (every download waits before the next upload is issued)."""
    import torch
    mass, pos, vel = sim.download()
    h_mass = torch.from_numpy(mass).pin_memory()
    h_pos = torch.from_numpy(pos).pin_memory()
    h_vel = torch.from_numpy(vel).pin_memory()
    o_pos = torch.empty_like(h_pos).pin_memory()
    o_vel = torch.empty_like(h_vel).pin_memory()
    sim.upload(h_mass, h_pos, h_vel)
    step(1)
    sim.download_into(None, o_pos, o_vel)

    def timed(wait: bool) -> float:
        sim.sync()
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(ext)
        for _ in range(steps):
            sim.upload(h_mass, h_pos, h_vel)
            step(1)
            sim.download_into(None, o_pos, o_vel, wait=wait)
        sim.sync()  # the last download has reached the host
        e1.record(ext)
        e1.synchronize()
        t = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64,
                         device=torch.device("cuda", sim.device))
        if dist is not None:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    ms_pipe = timed(wait=False)
    ms_serial = timed(wait=True)
    rate = lambda ms: (units or n) * steps / (ms / 1e3)
    return {"value": rate(ms_pipe), "unit": "body-steps/s",
            "h2d_bytes_per_step": int(h_mass.nbytes + h_pos.nbytes + h_vel.nbytes),
            "d2h_bytes_per_step": int(o_pos.nbytes + o_vel.nbytes), "steps": steps,
            "ms_per_step": ms_pipe / steps,
            "loop": "pipelined: upload, step, asynchronous download per step; one sync after the loop",
            "serial": {"value": rate(ms_serial), "ms_per_step": ms_serial / steps,
                       "loop": "every download waits before the next upload"}}


def secondary_16m(pkg, device: int, steps: int = 5, e2e_steps: int = 3, sm_max_mhz=None,
                  hbm_gbs: float = 6650.0, with_cpu: bool = True) -> dict:
    """The 16.8M-body Gaussian-mixture point of the metric (64-bit keys), with
    the same figures as the headline: device rate, stages, walk roofline and
    stream-stage HBM fractions, e2e through the public API, FP64 force error
    on 1,024 bodies and the reference's CPU rate on a bounded sample."""
    import torch
    wl = pkg.WORKLOADS["gaussian-mixture-16m"]
    n = wl["n"]
    sim = pkg.Simulation(wl["config"], device=device)
    sim.setNumBodies(n)
    sim.setScenario(wl["scenario"], 1)
    tune = sim.autotune(2)
    for _ in range(3):
        sim.step(1)
    sim.sync()
    ext = torch.cuda.ExternalStream(sim.getBuffers().stream, device=torch.device("cuda", device))
    # per-step CUDA events on the engine's stream, summed (as for the
    # headline): host-side gaps between step launches are not step time
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    sim.profile_begin(steps)
    for i in range(steps):
        starts[i].record(ext)
        sim.step(1)
        ends[i].record(ext)
    sim.sync()
    stage_ms, rec = sim.profile_end()
    ms = sum(a.elapsed_time(b) for a, b in zip(starts, ends)) / steps
    stages = {k: v / max(rec, 1) for k, v in stage_ms.items()}
    cfg = sim.config
    visits, multi, body, far = sim.walk_stats()
    acc = sim.read_buffer("acc", np.float32, 2 * n).reshape(n, 2)
    ferr = sim.forceError(acc, nsample=1024, seed=1)
    e2e = e2e_rate(sim, sim.step, n, e2e_steps, ext)
    kps = sim.kernels_per_step()
    sim.close()
    out = {"workload": "gaussian-mixture-16m", "bodies": n, "metric": "body-steps/s",
           "value": n / (ms / 1e3), "unit": "body-steps/s", "ms_per_step": ms, "steps": steps,
           "stages_ms": stages,
           "roofline": dict(walk_roofline(cfg, stages["walk"], multi, body, visits, sm_max_mhz,
                                          traffic=NCU_WALK_TRAFFIC_BYTES["gaussian-mixture-16m"],
                                          far_pairs=far, n=n),
                            traffic_source="ncu capture of the 4.2M-body case scaled by 4"),
           "stream_stages": stream_rooflines(stages, n, 8, hbm_gbs),
           "force_error_vs_fp64": ferr, "e2e": e2e, "autotune": tune,
           "gpu_launches": kps * steps,
           "config": {"theta": cfg.bhTheta, "softening": f"plummer {cfg.plummerEps}",
                      "dt": cfg.deltaTime, "integrator": cfg.integrator,
                      "morton_bits": cfg.mortonBits, "bodies_per_lane": cfg.bodiesPerLane,
                      "leaf_size": cfg.leafSize},
           "l2": "working set ~3 GB > L2 (no flush needed)"}
    if with_cpu:
        out["cpu_baseline"] = reference_baseline(REF_WORKLOADS["gaussian-mixture-16m"], 20.0)
    return out


def exact_walk_cost(pkg, device: int, steps: int = 10) -> dict:
    """The reference-semantics walk (walk_mode exact: every body visits the
    nodes of barnes_hut.wgsl:48-111's per-body monopole DFS, leaf size 1) on
    the headline workload, with its FP64 force error."""
    import torch
    wl = pkg.WORKLOADS["colliding-disks-800k"]
    n = wl["n"]
    cfg = dataclasses.replace(wl["config"], walk="exact", leafSize=1)
    sim = pkg.Simulation(cfg, device=device)
    sim.setNumBodies(n)
    sim.setScenario(wl["scenario"], 1)
    for _ in range(3):
        sim.step(1)
    sim.sync()
    ext = torch.cuda.ExternalStream(sim.getBuffers().stream, device=torch.device("cuda", device))
    flush = torch.empty(FLUSH_BYTES // 4, dtype=torch.float32, device=torch.device("cuda", device))
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    sim.profile_begin(steps)
    with torch.cuda.stream(ext):
        for i in range(steps):
            flush.zero_()
            starts[i].record(ext)
            sim.step(1)
            ends[i].record(ext)
    sim.sync()
    stage_ms, rec = sim.profile_end()
    ms = sum(s.elapsed_time(e) for s, e in zip(starts, ends)) / steps
    acc = sim.computeAccelerations()
    ferr = sim.forceError(acc, nsample=1024, seed=2)
    sim.close()
    return {"workload": "colliding-disks-800k", "walk": "exact (reference per-body walk)",
            "value": n / (ms / 1e3), "unit": "body-steps/s", "ms_per_step": ms,
            "stages_ms": {k: v / max(rec, 1) for k, v in stage_ms.items()},
            "force_error_vs_fp64": ferr}


def ensemble_cost(pkg, device: int, systems: int = 1024, steps: int = 100,
                  loop_steps: int = 10) -> dict:
    """Batched ensemble: 1,024 systems, sizes log-uniform in [1024, 262144],
    Plummer projection (a = 0.1) or uniform disk 50/50, theta 0.5, eps 1e-3,
    dt 1e-4, leapfrog; `steps` steps of the whole ensemble (one launch per
    stage, one graph per step, autotuned) against looping the single-system
    solver over the same systems (each system its own handle and stream, all
    systems issued back to back per step with no host sync, graphs on).  Both
    sides are timed with CUDA events after warm-up; the loop is timed over
    `loop_steps` steps."""
    import torch
    cfg = pkg.Config(bhTheta=0.5, deltaTime=1e-4, softening="plummer", plummerEps=1e-3,
                     mortonDomain="bbox", integrator="leapfrog-kdk", walk="group", leafSize=8,
                     farAlpha=pkg.config.FAR_ALPHA)
    sizes = pkg.ensemble_sizes(systems, 2024, 1024, 262144)
    total = int(sizes.sum())
    dev = torch.device("cuda", device)
    ens = pkg.Ensemble(sizes, cfg, device=device)
    ens.setScenarios(None, seed=2024)
    mass, pos, vel = ens.download()
    tune = ens.autotune(2)
    tuned = ens.config
    for _ in range(3):
        ens.step(1)
    ens.sync()
    ext = torch.cuda.ExternalStream(ens.getBuffers().stream, device=dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    ens.profile_begin(steps)
    e0.record(ext)
    ens.step(steps)
    e1.record(ext)
    ens.sync()
    stage_ms, rec = ens.profile_end()
    ens_ms = e0.elapsed_time(e1) / steps
    acc = ens.computeAccelerations()
    m2, p2, _ = ens.download()
    # force error on a sample of systems (each against its own FP64 direct sum)
    off = ens.offsets
    rng = np.random.default_rng(1)
    errs = []
    for k in rng.choice(systems, 16, replace=False):
        sl = slice(int(off[k]), int(off[k + 1]))
        med, p99, ns = force_error_vs_fp64(acc[sl], m2[sl], p2[sl], cfg, nsample=16, seed=int(k))
        errs.append(med)
    kps = ens.kernels_per_step()
    ens.close()

    # looped single-system solver over the same systems and initial states,
    # each system its own handle (tuned walk parameters, graphs on)
    sims = []
    for k in range(systems):
        sl = slice(int(off[k]), int(off[k + 1]))
        sim = pkg.Simulation(tuned, device=device)
        sim.setNumBodies(int(sizes[k]))
        sim.upload(mass[sl], pos[sl], vel[sl])
        sims.append(sim)
    for sim in sims:
        sim.step(2)
    torch.cuda.synchronize(dev)
    # (a) system by system: each system's steps, then the next system
    t0 = time.perf_counter()
    for sim in sims:
        sim.step(loop_steps)
        sim.sync()
    seq_ms = (time.perf_counter() - t0) * 1e3 / loop_steps
    # (b) all systems issued back to back per step on their own streams
    t0 = time.perf_counter()
    for _ in range(loop_steps):
        for sim in sims:
            sim.step(1)
    for sim in sims:
        sim.sync()
    conc_ms = (time.perf_counter() - t0) * 1e3 / loop_steps
    for sim in sims:
        sim.close()
    return {"systems": systems, "bodies": total, "steps": steps,
            "sizes": {"min": int(sizes.min()), "max": int(sizes.max()),
                      "median": float(np.median(sizes))},
            "value": total / (ens_ms / 1e3), "unit": "body-steps/s", "ms_per_step": ens_ms,
            "stages_ms": {k: v / max(rec, 1) for k, v in stage_ms.items()},
            "kernels_per_step": kps, "autotune": tune,
            "force_error_vs_fp64_median_of_system_medians": float(np.median(errs)),
            "loop_ms_per_step": seq_ms, "loop_value": total / (seq_ms / 1e3),
            "speedup_vs_loop": seq_ms / ens_ms,
            "concurrent_loop_ms_per_step": conc_ms, "speedup_vs_concurrent_loop": conc_ms / ens_ms,
            "timing": "ensemble: CUDA events on the engine stream; loops: host clock around "
                      "synchronised calls (one handle and stream per system), same systems "
                      "and states"}


def generate_cost(pkg, device: int, name: str = "gaussian-mixture", n: int = 16_777_216) -> dict:
    """Initial conditions for the 16.8M-body Gaussian mixture: the host
    generator (one PCG32 stream, then the 400 MB upload a step needs) against
    the GPU generator (one stream per body) into device arrays."""
    import ctypes
    import torch
    dev = torch.device("cuda", device)
    t0 = time.perf_counter()
    mass, pos, vel, rad = pkg.generate_scenario(name, n, 1)
    host_s = time.perf_counter() - t0
    lib = pkg.load()
    bufs = [torch.empty(k * n, dtype=torch.float32, device=dev) for k in (1, 2, 2, 1)]
    stream = torch.cuda.current_stream(dev)
    args = [ctypes.c_void_p(b.data_ptr()) for b in bufs]
    lib.bh_generate_scenario_device(name.encode(), n, 1, 1.0, *args,
                                    ctypes.c_void_p(stream.cuda_stream))  # warm-up
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    rc = lib.bh_generate_scenario_device(name.encode(), n, 1, 1.0, *args,
                                         ctypes.c_void_p(stream.cuda_stream))
    e1.record(stream)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    h = [torch.from_numpy(a.reshape(-1)).pin_memory() for a in (mass, pos, vel, rad)]
    pin_s = time.perf_counter() - t0
    u0 = torch.cuda.Event(enable_timing=True)
    u1 = torch.cuda.Event(enable_timing=True)
    u0.record(stream)
    for b, a in zip(bufs, h):
        b.copy_(a, non_blocking=True)
    u1.record(stream)
    torch.cuda.synchronize(dev)
    return {"scenario": name, "bodies": n, "host_generate_s": host_s,
            "host_upload_ms": u0.elapsed_time(u1), "host_pin_s": pin_s,
            "device_generate_ms": e0.elapsed_time(e1) if rc == 0 else None,
            "timing": "host: wall clock, one thread; upload from page-locked memory and the GPU "
                      "generator: CUDA events"}


def render_cost(pkg, device: int, width: int = 1920, height: int = 1080, frames: int = 20) -> dict:
    """Density render of the 800k colliding-disks bodies (the reference's
    Renderer.getCommands: clear, density splat, tone map) into a 1920 x 1080
    headless target, timed with CUDA events on the engine's stream."""
    import torch
    wl = pkg.WORKLOADS["colliding-disks-800k"]
    sim = pkg.Simulation(wl["config"], device=device)
    sim.setNumBodies(wl["n"])
    sim.setScenario(wl["scenario"], 1)
    r = pkg.Renderer(sim, width, height)
    r.setCamera(0.0, 0.0, 3.0 * width / height, 3.0)  # both disks on screen
    for _ in range(3):
        r.frame()
    sim.sync()
    ext = torch.cuda.ExternalStream(sim.getBuffers().stream, device=torch.device("cuda", device))
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(ext)
    for _ in range(frames):
        r.frame()
    e1.record(ext)
    sim.sync()
    ms = e0.elapsed_time(e1) / frames
    dens = r.readDensity()
    covered = int((dens > 0).sum())
    r.close()
    sim.close()
    return {"bodies": wl["n"], "canvas": [width, height], "ms_per_frame": ms,
            "frames_per_s": 1e3 / ms, "bodies_per_s": wl["n"] / (ms / 1e3),
            "covered_pixels": covered, "kernels_per_frame": 2,
            "timing": "CUDA events on the engine stream, mean of %d frames" % frames}


# ---------------------------------------------------------------- helpers

class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": float(max(smax)) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def load_pkg():
    return importlib.import_module(PKG)


def force_error_vs_fp64(acc, mass, pos, cfg, nsample=256, seed=0):
    """Median / p99 relative force error against an FP64 direct sum (numpy)."""
    rng = np.random.default_rng(seed)
    n = mass.size
    idx = rng.choice(n, size=min(nsample, n), replace=False)
    P = pos.astype(np.float64)
    M = mass.astype(np.float64)
    eps2 = float(cfg.plummerEps) ** 2
    errs = []
    for i in idx:
        r = P - P[i]
        d2 = (r * r).sum(1) + eps2
        inv3 = d2 ** -1.5
        inv3[i] = 0.0
        a = cfg.gravConstant * (M * inv3) @ r
        errs.append(np.linalg.norm(acc[i] - a) / max(np.linalg.norm(a), 1e-300))
    errs = np.array(errs)
    return float(np.median(errs)), float(np.percentile(errs, 99)), int(idx.size)


def _oracle():
    d = os.path.join(ROOT, "oracle")
    if d not in sys.path:
        sys.path.insert(0, d)
    import oracle as orc
    return orc


def _ref_setup(wp: dict):
    """Inputs of the reference's own shader logic (oracle/_ref: a mechanical
    C++ translation of lbvh.wgsl + barnes_hut.wgsl, independent stages on all
    host threads) for a workload: its bodies from the oracle's generator (one
    PCG32 stream per body: the workload's distribution and size), its theta
    and dt.  The reference knows only its own softening, eps = epsMult
    sqrt(G max(m1, m2) dt); epsMult is set so that eps equals the workload's
    Plummer eps at the median body mass."""
    orc = _oracle()
    op = wp["oracle"]
    n, G, dt = wp["n"], op["G"], op["dt"]
    mass, pos, vel, _ = orc.generate_per_body(wp["scenario"], n, 1, G)
    m_med = float(np.median(mass))
    eps_mult = float(op["plummer_eps"] / np.sqrt(G * m_med * dt))
    kw = dict(G=G, dt=dt, eps_mult=eps_mult, theta=op["theta"])
    return orc, n, (mass, pos, vel), kw


def _ref_seconds(st: dict, stride: int) -> float:
    """Host seconds of timed reference steps, the sampled walk scaled."""
    return st["morton"] + st["sort"] + st["build_fill"] + stride * st["vel_step"] + st["pos_step"]


def _ordinal(k: int) -> str:
    suffix = "th" if 10 <= k % 100 <= 20 else {1: "st", 2: "nd", 3: "rd"}.get(k % 10, "th")
    return f"{k}{suffix}"


def _ref_sample(what: str, n: int, stride: int, eps_mult: float, threads: int) -> str:
    walk = ("the whole walk" if stride == 1 else
            f"the walk timed on every {_ordinal(stride)} sorted slot and scaled by {stride}")
    return (f"{what} of the {n}-body workload, {walk} (reference WGSL logic translated to C++: "
            f"the reference's fixed 2000-unit Morton domain (lbvh.wgsl:49-57), so the workload's "
            f"bodies share few grid cells; per-body monopole walk; epsMult {eps_mult:.1f}; "
            f"{threads} OpenMP threads; fill serial; bodies from the oracle's generator)")


def reference_baseline(wp: dict, seconds_budget=20.0):
    """cpu_baseline leg: the reference's own shader logic (_ref_setup) for
    about `seconds_budget` of whole steps.  Up to a million bodies every step
    runs whole; above, the walk (velocity step) runs on every k-th sorted
    slot and its time is scaled by k, the other stages run whole."""
    orc = _oracle()
    if not orc.ref_available():
        return None
    orc, n, bodies, kw = _ref_setup(wp)
    stride = 1 if n <= 1_000_000 else max(1, n // 250_000)
    one = orc.ref_run_timed(*bodies, steps=1, walk_stride=stride, **kw)  # warm-up, sizes the sample
    per_step = _ref_seconds(one, 1) + one["vel_step"] * (stride - 1)
    steps = int(max(1, min(50, seconds_budget / max(per_step, 1e-3))))
    st = orc.ref_run_timed(*bodies, steps=steps, walk_stride=stride, **kw)
    threads = orc.ref_threads()
    return {"value": n * steps / _ref_seconds(st, stride), "unit": "body-steps/s", "cores": threads,
            "kind": "reference", "stages_s_per_step": {k: v / steps for k, v in st.items()},
            "walk_stride": stride,
            "sample": _ref_sample(f"{steps} steps", n, stride, kw["eps_mult"], threads)}


def reference_arm(wp: dict, steps: int, warmup: int, seconds_total=180.0):
    """--impl reference: `warmup` untimed steps, then exactly `steps` timed
    steps of the reference's own shader logic (_ref_setup) on the workload,
    each a bounded sample so that the whole run takes about `seconds_total`
    of host time.  A probe step (the walk on every k-th sorted slot above a
    million bodies) measures the stages; a step runs whole when it fits its
    share of the time, else its walk runs on every k-th sorted slot, k the
    smallest that fits, and the walk's time is scaled by k.  Falls back to
    the oracle port when oracle/_ref was not built."""
    orc = _oracle()
    steps = max(1, int(steps))
    warmup = max(0, int(warmup))
    if not orc.ref_available():
        return port_arm(wp, steps, warmup)
    orc, n, bodies, kw = _ref_setup(wp)
    probe = 1 if n <= 1_000_000 else max(1, n // 250_000)
    one = orc.ref_run_timed(*bodies, steps=1, walk_stride=probe, **kw)
    walk = one["vel_step"] * probe  # whole-walk seconds of one step
    other = _ref_seconds(one, probe) - walk
    share = seconds_total / (steps + warmup)
    avail = max(share - other, 0.05)
    stride = 1 if walk <= avail else min(n, math.ceil(walk / avail))
    if warmup:
        orc.ref_run_timed(*bodies, steps=warmup, walk_stride=stride, **kw)
    st = orc.ref_run_timed(*bodies, steps=steps, walk_stride=stride, **kw)
    threads = orc.ref_threads()
    return {"value": n * steps / _ref_seconds(st, stride), "unit": "body-steps/s",
            "cores": threads, "kind": "reference",
            "stages_s_per_step": {k: v / steps for k, v in st.items()}, "walk_stride": stride,
            "sample": _ref_sample(f"{warmup} untimed then {steps} timed steps", n, stride,
                                  kw["eps_mult"], threads)}


def port_arm(wp: dict, steps: int, warmup: int):
    """The oracle port (C restatement, OpenMP) in place of oracle/_ref:
    `warmup` untimed steps, then `steps` timed whole steps."""
    orc = _oracle()
    op = wp["oracle"]
    n = wp["n"]
    mass, pos, vel, _ = orc.generate_per_body(wp["scenario"], n, 1, op["G"])
    st = orc.State(orc.params(**op), mass, pos, vel)
    threads = orc.load().orc_max_threads()
    st.step(1)  # includes the initial force evaluation of the leapfrog
    if warmup:
        st.step(warmup)
    t0 = time.perf_counter()
    st.step(steps)
    el = time.perf_counter() - t0
    return {"value": n * steps / el, "unit": "body-steps/s", "cores": threads, "kind": "port",
            "sample": f"{warmup} untimed then {steps} timed whole steps of the {n}-body workload "
                      f"(oracle C restatement, same algorithm as the engine: {op['walk']} walk, "
                      f"{threads} OpenMP threads)"}


def cpu_baseline(wp: dict, seconds_budget=20.0):
    """The reference's own logic when it was built here, else the oracle port."""
    ref = reference_baseline(wp, seconds_budget)
    return ref if ref is not None else port_baseline(wp, seconds_budget)


def port_baseline(wp: dict, seconds_budget=20.0):
    """The oracle (C restatement, OpenMP) on a bounded sample of the workload."""
    orc = _oracle()
    op = wp["oracle"]
    n = wp["n"]
    mass, pos, vel, _ = orc.generate_per_body(wp["scenario"], n, 1, op["G"])
    st = orc.State(orc.params(**op), mass, pos, vel)
    threads = orc.load().orc_max_threads()
    st.step(1)  # first step includes the initial force evaluation of the leapfrog
    steps, t0 = 0, time.perf_counter()
    while True:
        st.step(1)
        steps += 1
        el = time.perf_counter() - t0
        if el > seconds_budget or steps >= 50:
            break
    return {"value": n * steps / el, "unit": "body-steps/s", "cores": threads, "kind": "port",
            "sample": f"{steps} steps of the full {n}-body workload after 1 warm-up step "
                      f"(oracle C restatement, same algorithm as the engine: {op['walk']} walk, "
                      f"{threads} OpenMP threads)"}


# ---------------------------------------------------------------- both arms

def run_config(args, n, theta, plummer_eps, dt, integrator, world):
    """The line's `config`: the workload both arms run, how a run with
    `world` ranks divides it, and how timed steps treat the caches.  Both
    arms build it here from the same values (the workload table the test
    suite checks against the package's), so the two lines carry one config;
    each implementation's own choices are reported beside it."""
    sharded = args.shard or (world > 1 and not args.replicas)
    return {"workload": args.workload, "bodies": n, "theta": theta,
            "softening": f"plummer {plummer_eps}", "dt": dt, "integrator": integrator,
            "parallelism": (f"shard{world} (sorted-slot ranges, one all-gather of "
                            f"16 B/body per step)" if sharded else
                            f"replicas{world}" if world > 1 else "single"),
            "l2": ("device timing: L2 flushed between timed steps (256 MB write, outside the "
                   "events); host timing: no device cache involved")}


def run_data(scenario: str) -> str:
    return f"synthetic (seeded PCG32 scenario {scenario!r}; no dataset exists for this path)"


# ---------------------------------------------------------------- reference arm

def run_reference(args):
    """The reference arm: rank 0 alone times the reference's own pipeline
    logic on the host cores; nothing of the engine package is imported."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    wp = REF_WORKLOADS[args.workload]
    op = wp["oracle"]
    # W untimed steps, then K timed ones, each a bounded sample of the
    # workload so the whole run stays within a few minutes.
    cb = reference_arm(wp, args.steps, args.warmup)
    line = {"impl": "reference", "metric": "body-steps/s", "value": cb["value"],
            "unit": "body-steps/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": run_data(wp["scenario"]),
            "config": run_config(args, wp["n"], op["theta"], op["plummer_eps"], op["dt"],
                                 op["integrator"], int(os.environ.get("WORLD_SIZE", "1"))),
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": "body-steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------- own arm

def _rel_change(new: float, old: float):
    """(new - old) / |old|, or None when the starting value is exactly zero
    (a system at rest in angular momentum, e.g. the Gaussian mixture)."""
    return (new - old) / abs(old) if old != 0.0 else None


def run_own(args):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    pkg = load_pkg()
    wl = pkg.WORKLOADS[args.workload]
    cfg = wl["config"]
    n = wl["n"]
    if args.walk_shape:
        bpl, leaf = (int(v) for v in args.walk_shape.split(","))
        cfg = dataclasses.replace(cfg, bodiesPerLane=bpl, leafSize=leaf)
        args.no_autotune = True
    sharded = None
    # With several ranks the default is the single system sharded over them
    # (the path's own exchange step); --replicas opts out.
    if args.shard or (world > 1 and not args.replicas):
        # One system on all ranks: rank 0 picks the walk shape, everyone uses it
        # (the ranks must build identical trees and groups).
        tune = None
        if not args.no_autotune:
            probe = pkg.Simulation(cfg, device=local)
            probe.setNumBodies(n)
            probe.setScenario(wl["scenario"], 1)
            tune = probe.autotune(3) if rank == 0 else None
            probe.close()
            if dist is not None:
                box = [tune]
                dist.broadcast_object_list(box, src=0)
                tune = box[0]
            cfg = dataclasses.replace(cfg, bodiesPerLane=tune["bodiesPerLane"],
                                      leafSize=tune["leafSize"], walkBlock=tune["walkBlock"])
        sharded = pkg.ShardedSimulation(cfg, n, wl["scenario"], seed=1, device=local)
        sim = sharded.sim
    else:
        sim = pkg.Simulation(cfg, device=local)
        sim.setNumBodies(n)
        sim.setScenario(wl["scenario"], 1 + rank)
        tune = None if args.no_autotune else sim.autotune(3)
    step = sharded.step if sharded is not None else sim.step
    cfg = sim.config
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    ext = torch.cuda.ExternalStream(sim.getBuffers().stream, device=dev)
    flush = torch.empty(FLUSH_BYTES // 4, dtype=torch.float32, device=dev)

    def barrier():
        if dist is not None:
            dist.barrier()

    # FP64 diagnostics before the run (energy / momentum drift, untimed)
    diag0 = sim.diagnostics() if rank == 0 else None

    # Warm-up also instantiates the profiled step graph used in the timed region.
    sim.profile_begin(max(args.warmup, 1))
    for _ in range(args.warmup):
        step(1)
    sim.sync()
    sim.profile_end()

    # ---- timed region: K steps, per-step events on the engine stream ----
    K = args.steps
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    clocks = ClockSampler(local)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    sim.profile_begin(K)
    t_wall = time.perf_counter()
    with torch.cuda.stream(ext):
        for i in range(K):
            flush.zero_()                  # L2 flush, outside the timed events
            starts[i].record(ext)
            step(1)
            ends[i].record(ext)
    sim.sync()
    torch.cuda.synchronize()
    wall = time.perf_counter() - t_wall
    barrier()
    clk = clocks.stop()
    stage_ms, recorded = sim.profile_end()
    step_ms = sum(s.elapsed_time(e) for s, e in zip(starts, ends))
    t = torch.tensor([step_ms], dtype=torch.float64, device=dev)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    step_ms_max = float(t.item())
    # replicas: every rank advances its own system; shard: one system on all ranks
    units = n if sharded is not None else world * n
    value = units * K / (step_ms_max / 1e3)

    diag1 = sim.diagnostics() if rank == 0 else None

    # ---- walk statistics + force error (untimed) ----
    visits, multi_inter, body_inter, far_pairs = sim.walk_stats()
    acc = sim.read_buffer("acc", np.float32, 2 * n).reshape(n, 2)
    ferr = sim.forceError(acc, nsample=2048, seed=0) if rank == 0 else None

    # ---- e2e through the public API with host buffers ----
    e2e = e2e_rate(sim, step, n, args.e2e_steps, ext, barrier, dist, units)

    out = None
    if rank == 0:
        peaks = {}
        try:
            peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        except OSError:
            pass
        # dominant kernel: the walk
        stages = {k: v / max(recorded, 1) for k, v in stage_ms.items()}
        roofline = walk_roofline(cfg, stages["walk"], multi_inter, body_inter, visits,
                                 clk.get("sm_max_mhz"), NCU_WALK_TRAFFIC_BYTES.get(args.workload),
                                 far_pairs=far_pairs, n=n)
        hbm = peaks.get("hbm_gbs", 6650.0)
        kps = sim.kernels_per_step()
        cb = None
        if not args.no_cpu_baseline and world == 1:  # the CPU baseline runs at N = 1 only
            cb = cpu_baseline(REF_WORKLOADS[args.workload])
        out = {
            "metric": "body-steps/s", "value": value, "unit": "body-steps/s", "n_gpus": world,
            "steps": K, "warmup": args.warmup, "ms_per_step": step_ms_max / K,
            "higher_is_better": True, "scaling": "strong" if sharded is not None else "weak",
            "vs_baseline": None, "dtype": "f32",
            "data": run_data(wl["scenario"]),
            "config": run_config(args, n, cfg.bhTheta, cfg.plummerEps, cfg.deltaTime,
                                 cfg.integrator, world),
            "engine": {"morton_bits": cfg.mortonBits,
                       "walk": f"{cfg.walk}, multipole order {cfg.multipole}",
                       "bodies_per_lane": cfg.bodiesPerLane, "leaf_size": cfg.leafSize,
                       "walk_block": cfg.walkBlock, "far_alpha": cfg.farAlpha,
                       "autotuned": tune is not None, "shape_pinned": bool(args.walk_shape)},
            "roofline": roofline,
            "stages_ms": stages,
            "stream_stages": stream_rooflines(stages, n, 8 if cfg.mortonBits == 64 else 4, hbm),
            "hbm_peak_gbs": hbm,
            "hbm_peak_source": ("MEASURED_PEAKS.json hbm_gbs" if "hbm_gbs" in peaks
                                else "fallback 6650 GB/s (no measured peaks file)"),
            "force_error_vs_fp64": ferr,
            "cpu_baseline": cb,
            "e2e": e2e,
            "diagnostics": {
                "steps": args.warmup + K,
                "energy_drift": _rel_change(diag1["total_energy"], diag0["total_energy"]),
                "momentum_change": [a - b for a, b in zip(diag1["momentum"], diag0["momentum"])],
                "angular_momentum_change": diag1["angular_momentum"] - diag0["angular_momentum"],
                "angular_momentum_drift": _rel_change(diag1["angular_momentum"],
                                                      diag0["angular_momentum"]),
                "total_energy_start": diag0["total_energy"],
                "how": "FP64 sums, direct-sum potential, before warm-up and after the timed steps"},
            "gpu_launches": kps * K,
            "clocks": clk,
            "wall_s_timed_region": wall,
        }
    sim.close()
    # The secondary points (16.8M, adjoint, ensemble, render, generators) are
    # single-GPU measurements: a multi-GPU run skips them, so the other ranks
    # do not wait on rank 0 for minutes at the closing barrier.
    extras = world == 1
    if rank == 0 and extras:
        if not args.no_secondary and args.workload != "gaussian-mixture-16m":
            out["secondary"] = secondary_16m(pkg, local, sm_max_mhz=clk.get("sm_max_mhz"),
                                             hbm_gbs=out["hbm_peak_gbs"],
                                             with_cpu=not args.no_cpu_baseline)
        if not args.no_exact_walk and args.workload == "colliding-disks-800k":
            out["exact_walk"] = exact_walk_cost(pkg, local)
        if not args.no_adjoint:
            out["adjoint"] = adjoint_cost(pkg, local)
        if not args.no_ensemble:
            out["ensemble"] = ensemble_cost(pkg, local)
        if not args.no_render:
            out["render"] = render_cost(pkg, local)
        if not args.no_secondary:
            out["generate"] = generate_cost(pkg, local)
    if rank == 0:
        print(json.dumps(out))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_own(args)


if __name__ == "__main__":
    sys.exit(main())
