"""Generate the golden fixtures of tests/golden/ from the reference's own shaders.

Render fixture (render_fragments.npz): the translated fragment stages of
density.wgsl and tone_map.wgsl (oracle/_ref/libref_render.so) evaluated on
seeded quad coordinates, radius multipliers and camera half sizes (density
added or discarded), on r16float texel values (tone-mapped rgb) and on
colormap arguments.

Run in the build container, where the reference checkout exists:

    python tests/golden/make_golden.py

It builds oracle/_ref/ (a mechanical C++ translation of the reference's
lbvh.wgsl and barnes_hut.wgsl, dispatched invocation by invocation in the
order of simulation.ts:393-420; the unvendored webgpu-radix-sort stage is the
stable sort of (key, id)), runs it on seeded inputs, and writes one
compressed .npz per case: the inputs (mass, pos, vel); the Morton codes,
permutation, left/right/parent arrays and node COM/mass/AABB/length of the
first step's tree (built from the inputs) with the state after that step
(pos_1, vel_1); and the state after `steps` steps (pos_n, vel_n).  The
reference parameters are config.ts's defaults (G = 1, dt = 0.1/60,
epsilonMultiplier = 1, theta = 0.6).
"""
from __future__ import annotations

import importlib
import importlib.util
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))

# (scenario, n, seed, steps); scenarios are the reference's three (simulation.ts:243-361)
CASES = [("default", n, n, 2) for n in (1, 2, 3, 63, 64, 65, 257, 1000, 2048)] + [
    ("two-clusters", 2000, 5, 2),
    ("planetary-disk", 2000, 6, 2),
]
PARAMS = dict(G=1.0, dt=0.1 / 60.0, eps_mult=1.0, theta=0.6, offset=0)


def case_path(scenario: str, n: int) -> str:
    return os.path.join(HERE, f"ref_{scenario}_{n}.npz")


def main() -> None:
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    spec = importlib.util.spec_from_file_location("oracle_build", os.path.join(ROOT, "oracle", "build.py"))
    ob = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(ob)
    if ob.build_ref(force=True) is None:
        raise SystemExit("the reference checkout is not available: fixtures cannot be regenerated")
    import oracle as orc
    bh = importlib.import_module("webgpu-fluid-sim_b200")
    for scenario, n, seed, steps in CASES:
        mass, pos, vel, _ = bh.generate_scenario(scenario, n, seed)
        # The tree of the first step (built from the inputs) and the state after it ...
        out = orc.ref_run(mass, pos, vel, steps=1, **PARAMS)
        out = {("pos_1" if k == "pos" else "vel_1" if k == "vel" else
                "node_mass" if k == "mass" else k): v for k, v in out.items()}
        # ... and the state after `steps` steps.
        last = orc.ref_run(mass, pos, vel, steps=steps, **PARAMS)
        np.savez_compressed(case_path(scenario, n), mass=mass, pos=pos, vel=vel,
                            steps=np.int32(steps), seed=np.int64(seed),
                            pos_n=last["pos"], vel_n=last["vel"], **out)
        print("wrote", case_path(scenario, n))
    render_fixture(orc)


def render_fixture(orc) -> None:
    if not orc.ref_render_available():
        raise SystemExit("oracle/_ref/libref_render.so is missing")
    rng = np.random.default_rng(2024)
    uv = rng.uniform(-1.05, 1.05, size=(2000, 2)).astype(np.float32)
    uv = np.concatenate([uv, np.array([[0, 0], [1, 0], [0, -1], [0.6, 0.8], [0.5, 0.5]],
                                      np.float32)])
    rms = np.array([0.5, 1.0, 1.0001, 5.0, 12.0], np.float32)
    halves = np.array([[10.0, 10.0], [16.0, 9.0], [40.0, 20.0], [0.5, 0.25]], np.float32)
    dens = np.zeros((len(halves), len(rms), len(uv)), np.float32)
    disc = np.zeros(dens.shape, np.uint8)
    for a, (hx, hy) in enumerate(halves):
        for b, rm in enumerate(rms):
            for c, (ux, uy) in enumerate(uv):
                dens[a, b, c], disc[a, b, c] = orc.ref_density_fragment(ux, uy, rm, hx, hy)
    # every 8th finite non-negative FP16 value, and a few fixed ones
    halfs = np.arange(0, 0x7C00, 8, dtype=np.uint16).view(np.float16).astype(np.float32)
    texels = np.concatenate([halfs, np.float32([0.125, 1.0, 1e-3, 6e4])])
    rgb = np.stack([orc.ref_tone_map_fragment(t) for t in texels]).astype(np.float32)
    ts = np.linspace(-0.1, 1.1, 1201, dtype=np.float32)
    cmap = np.stack([orc.ref_colormap(t) for t in ts])
    path = os.path.join(HERE, "render_fragments.npz")
    np.savez_compressed(path, uv=uv, radius_multipliers=rms, half_sizes=halves, density=dens,
                        discarded=disc, texels=texels, rgb=rgb, colormap_t=ts,
                        colormap_rgb=cmap.astype(np.float32))
    print("wrote", path)


if __name__ == "__main__":
    main()
