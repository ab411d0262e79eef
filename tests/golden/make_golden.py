"""Generate the golden fixtures of tests/golden/ from the reference's own shaders.

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


if __name__ == "__main__":
    main()
