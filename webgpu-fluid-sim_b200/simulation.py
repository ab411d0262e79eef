"""Simulation -- the reference's host class (src/simulation.ts:39-433) over
the CUDA engine's C ABI.

Method names, argument meaning and error behaviour follow simulation.ts:
``setNumBodies`` / ``setScenario`` regenerate the bodies and hand out new
buffers (simulation.ts:227-374), ``getCommands()`` returns the work of one
frame (``config.substeps`` steps, simulation.ts:386-425) which ``submit``
enqueues like ``device.queue.submit`` (main.ts:38-41), and an unknown
scenario raises ``Error("Unknown scenario: ...")`` (simulation.ts:363-365).
"""
from __future__ import annotations

import ctypes
import dataclasses

import numpy as np

from . import _lib
from .config import Config, getDefaultConfig

SCENARIOS = ("default", "two-clusters", "planetary-disk",
             "uniform-disk-kepler", "colliding-disks", "gaussian-mixture",
             "plummer-projection")


@dataclasses.dataclass(frozen=True)
class SimBuffers:
    """getBuffers() (simulation.ts:8-18): borrowed device pointers, valid until
    the next setNumBodies / setScenario / destroy."""

    mass: int
    pos: int
    vel: int
    radiusMultiplier: int
    acc: int
    mortonCodes: int
    bodyIndices: int
    nodeData: int          # float4 {com.x, com.y, mass, length} x (2n-1)
    nodeChildren: int      # uint2 {left, right} x (n-1)
    nodeParent: int        # uint32 x (2n-1)
    nodeAabb: int          # float4 {min.x, min.y, max.x, max.y} x (n-1)
    numBodies: int
    mortonBits: int
    stream: int


class CommandBuffer:
    """The work of one frame; submitting it enqueues config.substeps steps."""

    def __init__(self, sim: "Simulation", frames: int = 1):
        self._sim = sim
        self.frames = frames

    def submit(self) -> None:
        self._sim.step(self.frames)


def submit(command_buffers) -> None:
    """device.queue.submit([...]) for engine command buffers (main.ts:38-41)."""
    for cb in command_buffers:
        cb.submit()


class Simulation:
    """B200 Barnes-Hut engine behind the reference's Simulation API."""

    def __init__(self, config: Config | None = None, device: int = 0):
        self.config = config or getDefaultConfig()
        self._lib = _lib.load()
        c = self.config.to_c(device)
        h = ctypes.c_void_p()
        _lib.check(self._lib.bh_create(ctypes.byref(c), ctypes.byref(h)))
        self._h = h
        self.device = device
        self.currentScenario = "default"  # simulation.ts:59
        self.seed = 0

    # -- lifetime -----------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.bh_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, status: int) -> None:
        _lib.check(status, self._h)

    # -- reference API ------------------------------------------------------
    def updateMetadataBuffer(self) -> None:
        """simulation.ts:212-225 (the engine's fill needs no random offset)."""
        self._check(self._lib.bh_update_metadata(self._h))

    def setNumBodies(self, numBodies: int) -> None:
        """simulation.ts:227-231: new body count, current scenario regenerated."""
        if numBodies < 0:
            raise ValueError("numBodies must be >= 0")
        self._check(self._lib.bh_set_num_bodies(self._h, int(numBodies)))

    def setScenario(self, scenario: str, seed: int | None = None) -> None:
        """simulation.ts:233-374 with Math.random() replaced by seeded PCG32."""
        if seed is not None:
            self.seed = int(seed)
        st = self._lib.bh_set_scenario(self._h, scenario.encode(), self.seed)
        if st == _lib.BH_ERR_UNKNOWN_SCENARIO:
            raise _lib.BhError(st, f"Unknown scenario: {scenario}")
        self._check(st)
        self.currentScenario = scenario

    def setScenarioOnDevice(self, scenario: str, seed: int | None = None) -> None:
        """setScenario with the bodies generated on the GPU (one PCG32 stream
        per body; same distributions, a different sample than setScenario)."""
        if seed is not None:
            self.seed = int(seed)
        st = self._lib.bh_set_scenario_device(self._h, scenario.encode(), self.seed)
        if st == _lib.BH_ERR_UNKNOWN_SCENARIO:
            raise _lib.BhError(st, f"Unknown scenario: {scenario}")
        self._check(st)
        self.currentScenario = scenario

    def getCommands(self, frames: int = 1) -> CommandBuffer:
        """simulation.ts:386-425: one frame = config.substeps steps."""
        return CommandBuffer(self, frames)

    def getBuffers(self) -> SimBuffers:
        b = _lib.bh_buffers()
        self._check(self._lib.bh_get_buffers(self._h, ctypes.byref(b)))
        return SimBuffers(mass=b.mass, pos=b.pos, vel=b.vel, radiusMultiplier=b.radius_multiplier,
                          acc=b.acc, mortonCodes=b.morton_codes, bodyIndices=b.body_indices,
                          nodeData=b.node4, nodeChildren=b.node_children,
                          nodeParent=b.node_parent, nodeAabb=b.node_aabb,
                          numBodies=b.num_bodies, mortonBits=b.morton_bits,
                          stream=b.stream or 0)

    def getNumBodies(self) -> int:
        n = ctypes.c_uint32()
        self._check(self._lib.bh_get_num_bodies(self._h, ctypes.byref(n)))
        return int(n.value)

    # -- engine extras ----------------------------------------------------------
    def step(self, frames: int = 1) -> None:
        """Enqueue ``frames`` frames (asynchronous)."""
        self._check(self._lib.bh_step(self._h, int(frames)))

    def sync(self) -> None:
        self._check(self._lib.bh_sync(self._h))
        self._pending_host = []

    def upload(self, mass=None, pos=None, vel=None) -> None:
        n = self.getNumBodies()
        args = []
        for a, width in ((mass, 1), (pos, 2), (vel, 2)):
            if a is None:
                args.append(None)
                continue
            a = _as_host_f32(a, n * width)
            args.append(a)
        # Host memory must outlive the asynchronous copies: held until the next
        # sync or download, which wait for them.
        self._pending_host = getattr(self, "_pending_host", []) + [args]
        ptrs = [_ptr(a) for a in args]
        self._check(self._lib.bh_upload(self._h, *ptrs, n))

    def download(self):
        n = self.getNumBodies()
        mass = np.empty(n, np.float32)
        pos = np.empty((n, 2), np.float32)
        vel = np.empty((n, 2), np.float32)
        self._check(self._lib.bh_download(self._h, _ptr(mass), _ptr(pos), _ptr(vel), n))
        self._pending_host = []
        return mass, pos, vel

    def download_into(self, mass=None, pos=None, vel=None, wait: bool = True) -> None:
        """Download into caller-owned host arrays (page-locked for async speed).

        wait=False returns at once (bh_download_async): the arrays are written
        by the next sync() or waiting download, and the steps enqueued
        meanwhile run while the copy is under way."""
        n = self.getNumBodies()
        if wait:
            self._check(self._lib.bh_download(self._h, _ptr(mass), _ptr(pos), _ptr(vel), n))
            self._pending_host = []
            return
        self._check(self._lib.bh_download_async(self._h, _ptr(mass), _ptr(pos), _ptr(vel), n))
        # the host arrays must outlive the copy: held until the next sync
        self._pending_host = getattr(self, "_pending_host", []) + [[mass, pos, vel]]

    def computeAccelerations(self) -> np.ndarray:
        n = self.getNumBodies()
        acc = np.empty((n, 2), np.float32)
        self._check(self._lib.bh_compute_accelerations(self._h, _ptr(acc)))
        return acc

    def read_buffer(self, name: str, dtype, count: int) -> np.ndarray:
        out = np.empty(count, dtype)
        self._check(self._lib.bh_read_buffer(self._h, name.encode(), _ptr(out), out.nbytes))
        return out

    def tree(self) -> dict:
        """Sorted codes and ids and the hierarchy of the last tree built."""
        n = self.getNumBodies()
        bits = self.config.mortonBits
        nn, ni = max(2 * n - 1, 0), max(n - 1, 0)
        codes = self.read_buffer("morton_codes", np.uint64 if bits == 64 else np.uint32, n)
        ids = self.read_buffer("body_indices", np.uint32, n)
        node4 = self.read_buffer("node4", np.float32, 4 * nn).reshape(nn, 4)
        children = self.read_buffer("node_children", np.uint32, 2 * ni).reshape(ni, 2)
        parent = self.read_buffer("node_parent", np.uint32, nn)
        aabb = self.read_buffer("node_aabb", np.float32, 4 * ni).reshape(ni, 4)
        return dict(codes=codes, ids=ids, node4=node4, children=children, parent=parent, aabb=aabb)

    def profile_begin(self, max_steps: int) -> None:
        self._check(self._lib.bh_profile_begin(self._h, int(max_steps)))

    def profile_end(self) -> tuple[dict, int]:
        ms = (ctypes.c_double * 5)()
        cnt = ctypes.c_uint32()
        self._check(self._lib.bh_profile_end(self._h, ms, ctypes.byref(cnt)))
        return {k: float(ms[i]) for i, k in enumerate(_lib.BH_STAGE_NAMES)}, int(cnt.value)

    def autotune(self, trials: int = 3) -> dict:
        """Pick the fastest (bodies per lane, leaf size, walk block) for the group walk."""
        r = _lib.bh_tune_result()
        self._check(self._lib.bh_autotune(self._h, int(trials), ctypes.byref(r)))
        self.config = dataclasses.replace(self.config, bodiesPerLane=r.bodies_per_lane,
                                          leafSize=r.leaf_size, walkBlock=r.walk_block)
        return {"bodiesPerLane": r.bodies_per_lane, "leafSize": r.leaf_size,
                "walkBlock": r.walk_block, "walk_ms": r.walk_ms, "candidates": r.candidates}

    def force_vjp(self, abar) -> tuple[np.ndarray, np.ndarray]:
        """(da/dx)^T abar and (da/dm)^T abar at the current positions."""
        n = self.getNumBodies()
        ab = _as_host_f32(abar, 2 * n)
        xbar = np.empty((n, 2), np.float32)
        mbar = np.empty(n, np.float32)
        self._check(self._lib.bh_force_vjp(self._h, _ptr(ab), _ptr(xbar), _ptr(mbar)))
        return xbar, mbar

    def rollout_grad(self, steps: int, checkpoint_every: int, target_pos):
        """Loss (1/n) sum |x_T - target|^2 after `steps` steps and its gradient
        w.r.t. the initial positions, velocities and masses."""
        n = self.getNumBodies()
        tg = _as_host_f32(target_pos, 2 * n)
        loss = ctypes.c_float()
        gx = np.empty((n, 2), np.float32)
        gv = np.empty((n, 2), np.float32)
        gm = np.empty(n, np.float32)
        self._check(self._lib.bh_rollout_grad(self._h, int(steps), int(checkpoint_every), _ptr(tg),
                                              ctypes.byref(loss), _ptr(gx), _ptr(gv), _ptr(gm)))
        return float(loss.value), gx, gv, gm

    def walk_stats(self) -> tuple[int, int, int, int]:
        """(node visits, multipole interactions, body interactions, far-field
        (node, group) pairs) at the current positions."""
        v = ctypes.c_uint64()
        m = ctypes.c_uint64()
        b = ctypes.c_uint64()
        f = ctypes.c_uint64()
        self._check(self._lib.bh_walk_stats(self._h, ctypes.byref(v), ctypes.byref(m),
                                            ctypes.byref(b), ctypes.byref(f)))
        return int(v.value), int(m.value), int(b.value), int(f.value)

    def diagnostics(self, potential: bool = True) -> dict:
        """FP64 conserved quantities of the current state (bh_diagnostics_compute):
        total mass, centre of mass, momentum, angular momentum (z), kinetic and
        -- with ``potential`` -- direct-sum potential energy."""
        d = _lib.bh_diagnostics()
        self._check(self._lib.bh_diagnostics_compute(self._h, 1 if potential else 0,
                                                     ctypes.byref(d)))
        out = dict(total_mass=d.total_mass, com=[d.com[0], d.com[1]],
                   momentum=[d.momentum[0], d.momentum[1]],
                   angular_momentum=d.angular_momentum, kinetic_energy=d.kinetic_energy)
        if potential:
            out["potential_energy"] = d.potential_energy
            out["total_energy"] = d.kinetic_energy + d.potential_energy
            out["pairs"] = int(d.pairs)
        return out

    def directForcesFp64(self, sample) -> np.ndarray:
        """FP64 direct-sum accelerations (G included) of the bodies whose
        original indices are in ``sample``, at the current positions."""
        idx = np.ascontiguousarray(sample, dtype=np.uint32).reshape(-1)
        out = np.empty((idx.size, 2), np.float64)
        self._check(self._lib.bh_direct_forces_fp64(self._h, _ptr(idx), int(idx.size), _ptr(out)))
        return out

    def forceError(self, acc, nsample: int = 1024, seed: int = 0) -> dict:
        """Relative error |acc_i - a_i| / |a_i| of walk accelerations ``acc``
        (original order) against the FP64 direct sum, on ``nsample`` bodies
        drawn without replacement: median, p99, max and the sample size."""
        n = self.getNumBodies()
        rng = np.random.default_rng(seed)
        idx = np.sort(rng.choice(n, size=min(nsample, n), replace=False)).astype(np.uint32)
        ref = self.directForcesFp64(idx)
        a = np.asarray(acc, dtype=np.float64).reshape(n, 2)[idx]
        den = np.maximum(np.linalg.norm(ref, axis=1), 1e-300)
        err = np.linalg.norm(a - ref, axis=1) / den
        return {"median": float(np.median(err)), "p99": float(np.percentile(err, 99)),
                "max": float(err.max()), "sample": int(idx.size)}

    def debugSetLimits(self, flags: int = 0, lookback_spin_cap: int = 0,
                       walk_stack_cap: int = 0) -> None:
        """Test hook (bh_debug_set_limits): lower the bounded waits and stack
        capacities of the device-side checks; zeros restore the defaults."""
        self._check(self._lib.bh_debug_set_limits(self._h, int(flags), int(lookback_spin_cap),
                                                  int(walk_stack_cap)))

    def kernels_per_step(self) -> int:
        k = ctypes.c_uint32()
        self._check(self._lib.bh_kernels_per_step(self._h, ctypes.byref(k)))
        return int(k.value)


def _as_host_f32(a, count: int) -> np.ndarray:
    if hasattr(a, "data_ptr"):  # torch tensor in (pinned) host memory
        if a.numel() != count:
            raise ValueError(f"expected {count} floats, got {a.numel()}")
        return a
    arr = np.ascontiguousarray(a, dtype=np.float32).reshape(-1)
    if arr.size != count:
        raise ValueError(f"expected {count} floats, got {arr.size}")
    return arr


def _ptr(a):
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return ctypes.c_void_p(a.data_ptr())
    return a.ctypes.data_as(ctypes.c_void_p)


def generate_scenario(name: str, n: int, seed: int = 0, grav_constant: float = 1.0):
    """Host-side initial conditions, identical to what setScenario uploads."""
    lib = _lib.load()
    mass = np.empty(n, np.float32)
    pos = np.empty((n, 2), np.float32)
    vel = np.empty((n, 2), np.float32)
    rad = np.empty(n, np.float32)
    st = lib.bh_generate_scenario(name.encode(), n, seed, grav_constant, _ptr(mass), _ptr(pos),
                                  _ptr(vel), _ptr(rad))
    if st == _lib.BH_ERR_UNKNOWN_SCENARIO:
        raise _lib.BhError(st, f"Unknown scenario: {name}")
    _lib.check(st)
    return mass, pos, vel, rad


def ensemble_sizes(num_systems: int, seed: int, min_bodies: int, max_bodies: int) -> np.ndarray:
    """Log-uniform system sizes in [min_bodies, max_bodies] (PCG32 stream)."""
    lib = _lib.load()
    out = np.empty(num_systems, np.uint32)
    _lib.check(lib.bh_ensemble_sizes(num_systems, seed, min_bodies, max_bodies, _ptr(out)))
    return out


class Ensemble(Simulation):
    """Many independent systems advanced by one launch per stage.

    The bodies of all systems are concatenated (system k owns
    ``offsets[k]:offsets[k+1]``); every Simulation call (step, upload,
    download, getBuffers, computeAccelerations, ...) acts on the
    concatenation.  setNumBodies / setScenario have no meaning for an
    ensemble and raise; use ``setScenarios``.
    """

    def __init__(self, sizes, config: Config | None = None, device: int = 0):
        self.config = config or getDefaultConfig()
        self._lib = _lib.load()
        c = self.config.to_c(device)
        sz = np.ascontiguousarray(sizes, dtype=np.uint32)
        h = ctypes.c_void_p()
        _lib.check(self._lib.bh_ensemble_create(ctypes.byref(c), _ptr(sz), int(sz.size),
                                                ctypes.byref(h)))
        self._h = h
        self.device = device
        self.currentScenario = "ensemble"
        self.seed = 0
        self.sizes = sz.copy()
        self.offsets = np.zeros(sz.size + 1, np.uint32)
        self._check(self._lib.bh_get_system_offsets(self._h, _ptr(self.offsets)))

    def setScenarios(self, names=None, seed: int = 0) -> None:
        """names[k] = scenario of system k; None = Plummer projection (a=0.1)
        or uniform disk, 1/2 each, per system."""
        self.seed = int(seed)
        if names is None:
            self._check(self._lib.bh_ensemble_set_scenarios(self._h, None, self.seed))
            return
        if len(names) != self.sizes.size:
            raise ValueError(f"expected {self.sizes.size} scenario names, got {len(names)}")
        enc = [n.encode() for n in names]
        arr = (ctypes.c_char_p * len(enc))(*enc)
        st = self._lib.bh_ensemble_set_scenarios(self._h, ctypes.cast(arr, ctypes.c_void_p),
                                                 self.seed)
        if st == _lib.BH_ERR_UNKNOWN_SCENARIO:
            raise _lib.BhError(st, "Unknown scenario in ensemble")
        self._check(st)

    def numSystems(self) -> int:
        k = ctypes.c_uint32()
        self._check(self._lib.bh_get_num_systems(self._h, ctypes.byref(k)))
        return int(k.value)
