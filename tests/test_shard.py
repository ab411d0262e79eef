"""Several GPUs: one system sharded by sorted-slot ranges with one all-gather
per step, and ensembles partitioned by systems.

CPU: the partitions, and the chunk all-gather over a world of 2 gloo ranks
(processes on this host).  GPU (marked): on one GPU the ranks run one after
the other (no rank waits on another inside a kernel) -- each integrates its
slot range, packs, and every rank unpacks all chunks -- and the result must
equal the unsharded step bit for bit, since every rank builds the same tree.
"""
import ctypes
import os
import socket

import numpy as np
import pytest


def test_slot_ranges_tile_the_slots(bh):
    for n in (1, 2, 5, 1000, 800_001):
        for world in (1, 2, 3, 8):
            rs = bh.slot_ranges(n, world)
            assert rs[0][0] == 0 and rs[-1][1] == n
            assert all(rs[k][1] == rs[k + 1][0] for k in range(world - 1))
            assert max(h - lo for lo, h in rs) <= -(-n // world)
    assert bh.chunk_capacity(1000, 3, 4) == 334 + 128
    assert bh.chunk_bytes(10) == 176


def test_partition_systems_balanced_and_complete(bh):
    sizes = bh.ensemble_sizes(1024, 2024, 1024, 262144)
    for world in (1, 2, 4, 8):
        parts = bh.partition_systems(sizes, world)
        flat = sorted(k for p in parts for k in p)
        assert flat == list(range(len(sizes)))
        cost = [sum(int(sizes[k]) * np.log2(int(sizes[k])) for k in p) for p in parts]
        assert max(cost) <= 1.02 * (sum(cost) / world)
        assert parts == bh.partition_systems(list(sizes), world)  # same answer everywhere


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _gloo_rank(rank, world, port, q):
    import importlib
    import sys
    import torch
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    bh = importlib.import_module("webgpu-fluid-sim_b200")
    import datetime
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    try:
        dist.init_process_group("gloo", rank=rank, world_size=world,
                                timeout=datetime.timedelta(seconds=60))
        nb = bh.chunk_bytes(5)
        chunk = torch.full((nb,), rank + 1, dtype=torch.uint8)
        out = torch.zeros((world, nb), dtype=torch.uint8)
        bh.all_gather_chunks(out, chunk)
        ok = all(bool((out[r] == r + 1).all()) for r in range(world))
        parts = bh.partition_systems([300, 5000, 77, 4096, 1024], world)
        q.put((rank, ok, parts))
        dist.destroy_process_group()
    except Exception as e:  # report instead of leaving the parent waiting
        q.put((rank, False, repr(e)))


def test_chunk_all_gather_over_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gloo_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert all(ok for _, ok, _ in res)
    assert res[0][2] == res[1][2]


CFGS = {
    "leapfrog": dict(walk="group", softening="plummer", plummerEps=1e-3, bhTheta=0.5,
                     mortonDomain="bbox", integrator="leapfrog-kdk", bodiesPerLane=2),
    "euler": dict(walk="group", softening="plummer", plummerEps=1e-3, bhTheta=0.5,
                  mortonDomain="bbox", bodiesPerLane=4, leafSize=4),
}


@pytest.mark.gpu
@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("mode", ["leapfrog", "euler"])
def test_emulated_ranks_equal_one_gpu(bh, world, mode):
    import torch
    n = 60_001
    ref = bh.Simulation(bh.Config(**CFGS[mode]))
    ref.setNumBodies(n)
    ref.setScenario("colliding-disks", 8)
    ranks = []
    for r, (lo, hi) in enumerate(bh.slot_ranges(n, world)):
        s = bh.Simulation(bh.Config(**CFGS[mode]))
        s.setNumBodies(n)
        s.setScenario("colliding-disks", 8)
        assert s._lib.bh_set_walk_slots(s._h, lo, hi) == 0
        ranks.append(s)
    cap = bh.chunk_capacity(n, world, CFGS[mode]["bodiesPerLane"])
    dev = torch.device("cuda", 0)
    gathered = torch.zeros((world, bh.chunk_bytes(cap)), dtype=torch.uint8, device=dev)
    for step in range(3):
        ref.step(1)
        for r, s in enumerate(ranks):
            s.step(1)
            assert s._lib.bh_shard_pack(s._h, ctypes.c_void_p(gathered[r].data_ptr()), cap) == 0
            s.sync()
        counts = gathered[:, 4:8].cpu().numpy().view(np.uint32).ravel()
        assert counts.sum() == n  # the ranks' updated ranges tile the slots
        for s in ranks:
            assert s._lib.bh_shard_unpack(s._h, ctypes.c_void_p(gathered.data_ptr()), world,
                                          cap) == 0
            s.sync()
        want = ref.download()
        for s in ranks:
            got = s.download()
            for a, b in zip(got, want):
                assert np.array_equal(a, b), f"step {step}: rank state differs from one GPU"
    for s in ranks + [ref]:
        s.close()


def _gloo_sharded_rank(rank, world, port, mode, n, steps, q):
    # One rank of a sharded run: its own process and CUDA context on the one
    # GPU; the all-gather goes through gloo on the host, so no kernel waits
    # on another rank.
    import datetime
    import importlib
    import sys
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    try:
        bh = importlib.import_module("webgpu-fluid-sim_b200")
        dist.init_process_group("gloo", rank=rank, world_size=world,
                                timeout=datetime.timedelta(seconds=60))
        sh = bh.ShardedSimulation(bh.Config(**CFGS[mode]), n, "colliding-disks", seed=8)
        sh.step(steps)
        sh.sync()
        mass, pos, vel = sh.download()
        sh.close()
        dist.barrier()
        dist.destroy_process_group()
        q.put((rank, True, (mass, pos, vel)))
    except Exception as e:  # report instead of leaving the parent waiting
        q.put((rank, False, repr(e)))


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["leapfrog", "euler"])
def test_sharded_simulation_two_gloo_processes_equal_one_gpu(bh, mode):
    # ShardedSimulation end to end over two processes (gloo, chunks staged
    # through host memory) against one unsharded Simulation, bit for bit.
    import torch.multiprocessing as mp
    n, steps = 40_001, 3
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gloo_sharded_rank, args=(r, 2, port, mode, n, steps, q))
             for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert all(ok for _, ok, _ in res), [r[2] for r in res if not r[1]]
    ref = bh.Simulation(bh.Config(**CFGS[mode]))
    ref.setNumBodies(n)
    ref.setScenario("colliding-disks", 8)
    ref.step(steps)
    want = ref.download()
    ref.close()
    for rank, _, got in res:
        for a, b in zip(got, want):
            assert np.array_equal(a, b), f"rank {rank} differs from one GPU"


@pytest.mark.gpu
def test_sharded_simulation_world_one_equals_simulation(bh):
    cfg = bh.Config(**CFGS["leapfrog"])
    sh = bh.ShardedSimulation(cfg, 30_000, "colliding-disks", seed=2)
    ref = bh.Simulation(cfg)
    ref.setNumBodies(30_000)
    ref.setScenario("colliding-disks", 2)
    sh.step(4)
    ref.step(4)
    sh.sync()
    for a, b in zip(sh.download(), ref.download()):
        assert np.array_equal(a, b)
    sh.close()
    ref.close()


@pytest.mark.gpu
def test_shard_chunk_too_small_is_reported(bh):
    import torch
    sim = bh.Simulation(bh.Config(**CFGS["euler"]))
    sim.setNumBodies(5000)
    assert sim._lib.bh_set_walk_slots(sim._h, 0, 2500) == 0
    sim.step(1)
    chunk = torch.zeros(bh.chunk_bytes(4), dtype=torch.uint8, device="cuda")
    assert sim._lib.bh_shard_pack(sim._h, ctypes.c_void_p(chunk.data_ptr()), 4) == 0
    with pytest.raises(bh.BhError, match="shard chunk too small"):
        sim.sync()
    assert chunk[4:8].cpu().numpy().view(np.uint32)[0] == 0  # nothing packed
    sim.close()
