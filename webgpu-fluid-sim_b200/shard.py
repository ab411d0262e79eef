"""Several GPUs, one process per GPU (torch.distributed over NCCL).

Two ways to spread the work, as the path allows:

* ``ShardedSimulation`` -- one system.  Every rank holds the whole state and
  builds the same tree; rank r integrates the groups whose first sorted slot
  lies in its range of [0, n) (``slot_ranges``); after each step one
  all-gather of fixed-size chunks (the bodies each rank updated, in
  sorted-slot order) leaves every rank with the state one GPU would have.
  Per step that is 16 bytes per body over NVLink; the sort, the tree and the
  opening kick-drift are repeated on every rank.
* ``partition_systems`` -- an ensemble of independent systems.  Systems go to
  ranks by estimated walk cost (n log n, largest first, to the least loaded
  rank); each rank advances its own ``Ensemble`` with no collective at all.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import _lib
from .simulation import Simulation


def slot_ranges(n: int, world: int) -> list[tuple[int, int]]:
    """Consecutive sorted-slot ranges [lo, hi) of the ranks (they tile [0, n))."""
    if world < 1:
        raise ValueError("world size must be >= 1")
    return [(r * n // world, (r + 1) * n // world) for r in range(world)]


def chunk_capacity(n: int, world: int, bodies_per_lane: int) -> int:
    """Bodies one rank's chunk must hold: its slot range plus at most one group
    (a range ends at the first group that starts at or after its end)."""
    return -(-n // world) + 32 * max(int(bodies_per_lane), 1)


def chunk_bytes(capacity: int) -> int:
    return 16 + 16 * capacity


def partition_systems(sizes, world: int) -> list[list[int]]:
    """Systems of an ensemble per rank: largest estimated cost (n log2 n) first,
    each to the least loaded rank (ties to the lowest rank); every rank gets
    the same answer from the same sizes."""
    sizes = [int(x) for x in sizes]
    cost = [s * math.log2(max(s, 2)) for s in sizes]
    order = sorted(range(len(sizes)), key=lambda k: (-cost[k], k))
    load = [0.0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for k in order:
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(k)
        load[r] += cost[k]
    return [sorted(p) for p in parts]


def all_gather_chunks(out, chunk, group=None) -> None:
    """out[r] = rank r's chunk (torch tensors, out shaped (world, bytes))."""
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        out[0].copy_(chunk)
        return
    if dist.get_backend(group) == "nccl":
        dist.all_gather_into_tensor(out.view(-1), chunk, group=group)
    elif chunk.is_cuda:
        # gloo gathers host tensors: the chunks cross host memory (on the
        # current stream, so after the pack and before the unpack)
        import torch
        host = chunk.cpu()
        parts = [torch.empty_like(host) for _ in range(out.shape[0])]
        dist.all_gather(parts, host, group=group)
        out.copy_(torch.stack(parts))
    else:
        dist.all_gather(list(out.unbind(0)), chunk, group=group)


class ShardedSimulation:
    """One system stepped by all ranks of the default process group."""

    def __init__(self, config, numBodies: int, scenario: str, seed: int = 0, device: int = 0,
                 group=None):
        import torch
        import torch.distributed as dist
        self.group = group
        if dist.is_available() and dist.is_initialized():
            self.rank = dist.get_rank(group)
            self.world = dist.get_world_size(group)
        else:
            self.rank, self.world = 0, 1
        self.sim = Simulation(config, device=device)
        self.sim.setNumBodies(int(numBodies))
        self.sim.setScenario(scenario, seed)  # same seed on every rank: same state
        self.n = int(numBodies)
        self.lo, self.hi = slot_ranges(self.n, self.world)[self.rank]
        _lib.check(self.sim._lib.bh_set_walk_slots(self.sim._h, self.lo, self.hi), self.sim._h)
        bpl = self.sim.config.bodiesPerLane or 2
        self.capacity = chunk_capacity(self.n, self.world, bpl)
        dev = torch.device("cuda", device)
        nb = chunk_bytes(self.capacity)
        self.chunk = torch.empty(nb, dtype=torch.uint8, device=dev)
        self.gathered = torch.empty((self.world, nb), dtype=torch.uint8, device=dev)
        self.stream = torch.cuda.ExternalStream(self.sim.getBuffers().stream, device=dev)

    def step(self, frames: int = 1) -> None:
        import torch
        steps = int(frames) * int(self.sim.config.substeps)
        lib = self.sim._lib
        for _ in range(steps):
            self.sim.step(1)
            _lib.check(lib.bh_shard_pack(self.sim._h, ctypes.c_void_p(self.chunk.data_ptr()),
                                         self.capacity), self.sim._h)
            with torch.cuda.stream(self.stream):
                all_gather_chunks(self.gathered, self.chunk, self.group)
            _lib.check(lib.bh_shard_unpack(self.sim._h, ctypes.c_void_p(self.gathered.data_ptr()),
                                           self.world, self.capacity), self.sim._h)

    def sync(self) -> None:
        self.sim.sync()

    def download(self):
        return self.sim.download()

    def close(self) -> None:
        self.sim.close()
