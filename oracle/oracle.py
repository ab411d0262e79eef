"""ctypes wrapper of the oracle library (libbh_oracle.so).

TEST INFRASTRUCTURE ONLY: used by tests/, the smoke check and the CPU
baseline of bench.py as the checker.  The engine never imports this module.
The C restatement it wraps follows lbvh.wgsl / barnes_hut.wgsl of the
reference line by line (see bh_oracle.h for the citations).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbh_oracle.so")

SOFT = {"reference": 0, "plummer": 1}
DOMAIN = {"fixed2000": 0, "bbox": 1}
INTEGRATOR = {"symplectic-euler": 0, "leapfrog-kdk": 1}


class OrcParams(ctypes.Structure):
    _fields_ = [
        ("grav_constant", ctypes.c_float),
        ("delta_time", ctypes.c_float),
        ("epsilon_multiplier", ctypes.c_float),
        ("bh_theta", ctypes.c_float),
        ("softening", ctypes.c_int),
        ("plummer_eps", ctypes.c_float),
        ("morton_bits", ctypes.c_int),
        ("morton_domain", ctypes.c_int),
        ("integrator", ctypes.c_int),
        ("leaf_size", ctypes.c_int),
        ("threads", ctypes.c_int),
        ("walk_mode", ctypes.c_int),
        ("multipole", ctypes.c_int),
        ("bodies_per_lane", ctypes.c_int),
        ("far_alpha", ctypes.c_float),
    ]


WALK = {"exact": 0, "group": 1}


class OrcDomain(ctypes.Structure):
    _fields_ = [("lo_x", ctypes.c_float), ("lo_y", ctypes.c_float),
                ("extent", ctypes.c_float), ("pow2_exp", ctypes.c_int)]


_lib = None
_P = ctypes.c_void_p


def load() -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        import importlib.util
        spec = importlib.util.spec_from_file_location("oracle_build", os.path.join(HERE, "build.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        mod.build_oracle()
    lib = ctypes.CDLL(LIB_PATH)
    P = ctypes.POINTER(OrcParams)
    sig = {
        "orc_domain_compute": (None, [P, ctypes.c_uint32, _P, ctypes.POINTER(OrcDomain)]),
        "orc_morton": (None, [P, ctypes.POINTER(OrcDomain), ctypes.c_uint32, _P, _P, _P]),
        "orc_sort": (None, [ctypes.c_uint32, _P, _P]),
        "orc_build": (None, [ctypes.c_uint32, ctypes.c_int, _P, _P, _P, _P]),
        "orc_fill": (None, [ctypes.c_uint32, ctypes.c_uint32, _P, _P, _P, _P, _P, _P, _P, _P,
                            _P, _P]),
        "orc_walk": (None, [P, ctypes.c_uint32, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
        "orc_walk_counts": (None, [P, ctypes.c_uint32, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
        "orc_direct_sum_fp64": (None, [P, ctypes.c_uint32, _P, _P, ctypes.c_uint32, _P, _P]),
        "orc_create": (_P, [P, ctypes.c_uint32, _P, _P, _P]),
        "orc_destroy": (None, [_P]),
        "orc_step": (None, [_P, ctypes.c_uint32]),
        "orc_accelerations": (None, [_P, _P]),
        "orc_get_state": (None, [_P, _P, _P]),
        "orc_get_tree": (None, [_P] + [_P] * 9),
        "orc_num_bodies": (ctypes.c_uint32, [_P]),
        "orc_rollout_grad_fp64": (ctypes.c_double, [P, ctypes.c_uint32, _P, _P, _P, _P,
                                                    ctypes.c_uint32, _P, _P, _P]),
        "orc_force_vjp_fp64": (None, [P, ctypes.c_uint32, _P, _P, _P, _P, _P]),
        "orc_max_threads": (ctypes.c_int, []),
        "orc_render_density": (None, [_P, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, _P, _P,
                                      _P]),
        "orc_tone_map": (None, [ctypes.c_uint32, _P, _P]),
        "orc_colormap": (None, [ctypes.c_float, _P]),
        "orc_splat_weight": (ctypes.c_float, [ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                              ctypes.c_float, ctypes.POINTER(ctypes.c_int)]),
        "orc_tone_map_rgb": (None, [ctypes.c_float, _P]),
        "orc_diagnostics_fp64": (None, [P, ctypes.c_uint32, _P, _P, _P, _P]),
        "orc_generate_per_body": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_uint32, ctypes.c_uint64,
                                                 ctypes.c_double, _P, _P, _P, _P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def params(G=1.0, dt=0.1 / 60.0, eps_mult=1.0, theta=0.6, softening="reference",
           plummer_eps=1e-3, morton_bits=32, morton_domain="fixed2000",
           integrator="symplectic-euler", leaf_size=1, threads=0, walk="exact", multipole=2,
           bodies_per_lane=2, far_alpha=0.0) -> OrcParams:
    return OrcParams(G, dt, eps_mult, theta, SOFT[softening], plummer_eps, morton_bits,
                     DOMAIN[morton_domain], INTEGRATOR[integrator], leaf_size, threads,
                     WALK[walk], multipole, bodies_per_lane, far_alpha)


def params_from_config(cfg, threads: int = 0) -> OrcParams:
    """OrcParams equal to an engine Config (duck-typed: the field names of config.ts)."""
    return params(G=cfg.gravConstant, dt=cfg.deltaTime, eps_mult=cfg.epsilonMultiplier,
                  theta=cfg.bhTheta, softening=cfg.softening, plummer_eps=cfg.plummerEps,
                  morton_bits=cfg.mortonBits, morton_domain=cfg.mortonDomain,
                  integrator=cfg.integrator, leaf_size=cfg.leafSize, threads=threads,
                  walk=getattr(cfg, "walk", "exact"), multipole=getattr(cfg, "multipole", 2),
                  bodies_per_lane=getattr(cfg, "bodiesPerLane", 2) or 2,
                  far_alpha=getattr(cfg, "farAlpha", 0.0))


def f32(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a.reshape(shape) if shape is not None else a


def morton(p: OrcParams, pos) -> tuple[np.ndarray, np.ndarray]:
    lib = load()
    pos = f32(pos, (-1, 2))
    n = pos.shape[0]
    dom = OrcDomain()
    lib.orc_domain_compute(ctypes.byref(p), n, _p(pos), ctypes.byref(dom))
    codes = np.empty(n, np.uint64)
    ids = np.empty(n, np.uint32)
    lib.orc_morton(ctypes.byref(p), ctypes.byref(dom), n, _p(pos), _p(codes), _p(ids))
    return codes, ids


def sort(codes, ids):
    lib = load()
    codes = np.ascontiguousarray(codes, np.uint64).copy()
    ids = np.ascontiguousarray(ids, np.uint32).copy()
    lib.orc_sort(codes.size, _p(codes), _p(ids))
    return codes, ids


def build(codes, bits: int = 32):
    lib = load()
    codes = np.ascontiguousarray(codes, np.uint64)
    n = codes.size
    nn = max(2 * n - 1, 1)
    left = np.zeros(nn, np.uint32)
    right = np.zeros(nn, np.uint32)
    parent = np.zeros(nn, np.uint32)
    lib.orc_build(n, bits, _p(codes), _p(left), _p(right), _p(parent))
    return left, right, parent


def fill(ids, mass, pos, left, right, parent, offset: int = 0):
    lib = load()
    n = len(ids)
    nn = max(2 * n - 1, 1)
    com = np.zeros((nn, 2), np.float32)
    mnode = np.zeros(nn, np.float32)
    aabb = np.zeros((nn, 4), np.float32)
    length = np.zeros(nn, np.float32)
    lib.orc_fill(n, offset, _p(np.ascontiguousarray(ids, np.uint32)), _p(f32(mass)),
                 _p(f32(pos, (-1, 2))), _p(left), _p(right), _p(parent), _p(com), _p(mnode),
                 _p(aabb), _p(length))
    return com, mnode, aabb, length


def walk(p: OrcParams, ids, mass, pos, com, mnode, length, left, right):
    lib = load()
    n = len(ids)
    acc = np.zeros((n, 2), np.float32)
    lib.orc_walk(ctypes.byref(p), n, _p(np.ascontiguousarray(ids, np.uint32)), _p(f32(mass)),
                 _p(f32(pos, (-1, 2))), _p(com), _p(mnode), _p(length), _p(left), _p(right),
                 _p(acc))
    return acc


def walk_counts(p: OrcParams, ids, mass, pos, com, mnode, length, left, right):
    lib = load()
    n = len(ids)
    v = ctypes.c_uint64()
    i = ctypes.c_uint64()
    lib.orc_walk_counts(ctypes.byref(p), n, _p(np.ascontiguousarray(ids, np.uint32)),
                        _p(f32(mass)), _p(f32(pos, (-1, 2))), _p(com), _p(mnode), _p(length),
                        _p(left), _p(right), ctypes.byref(v), ctypes.byref(i))
    return int(v.value), int(i.value)


def direct_sum_fp64(p: OrcParams, mass, pos, sample) -> np.ndarray:
    lib = load()
    mass = f32(mass)
    pos = f32(pos, (-1, 2))
    sample = np.ascontiguousarray(sample, np.uint32)
    out = np.zeros((sample.size, 2), np.float64)
    lib.orc_direct_sum_fp64(ctypes.byref(p), mass.size, _p(mass), _p(pos), sample.size,
                            _p(sample), _p(out))
    return out


def rollout_grad_fp64(p: OrcParams, mass, pos, vel, target, steps: int):
    """FP64 direct-sum KDK rollout and its exact adjoint: (L, dL/dx0, dL/dv0, dL/dm)."""
    lib = load()
    mass = f32(mass)
    pos = f32(pos, (-1, 2))
    vel = f32(vel, (-1, 2))
    target = f32(target, (-1, 2))
    n = mass.size
    gx = np.zeros((n, 2), np.float64)
    gv = np.zeros((n, 2), np.float64)
    gm = np.zeros(n, np.float64)
    L = lib.orc_rollout_grad_fp64(ctypes.byref(p), n, _p(mass), _p(pos), _p(vel), _p(target),
                                  steps, _p(gx), _p(gv), _p(gm))
    return float(L), gx, gv, gm


def force_vjp_fp64(p: OrcParams, mass, pos, abar):
    """FP64 direct-sum (da/dx)^T abar, (da/dm)^T abar."""
    lib = load()
    mass = f32(mass)
    pos = f32(pos, (-1, 2))
    abar = f32(abar, (-1, 2))
    n = mass.size
    xb = np.zeros((n, 2), np.float64)
    mb = np.zeros(n, np.float64)
    lib.orc_force_vjp_fp64(ctypes.byref(p), n, _p(mass), _p(pos), _p(abar), _p(xb), _p(mb))
    return xb, mb


def diagnostics_fp64(p: OrcParams, mass, pos, vel) -> dict:
    """FP64 conserved quantities: M, COM, P, Lz, K, W (direct pair sum)."""
    lib = load()
    mass = f32(mass)
    out = np.zeros(8, np.float64)
    lib.orc_diagnostics_fp64(ctypes.byref(p), mass.size, _p(mass), _p(f32(pos, (-1, 2))),
                             _p(f32(vel, (-1, 2))), _p(out))
    return dict(total_mass=out[0], com=out[1:3], momentum=out[3:5], angular_momentum=out[5],
                kinetic_energy=out[6], potential_energy=out[7])


def generate_per_body(name: str, n: int, seed: int, G: float = 1.0):
    """Scenario with one PCG32 stream per body: (mass, pos, vel, radius)."""
    lib = load()
    mass = np.zeros(n, np.float32)
    pos = np.zeros((n, 2), np.float32)
    vel = np.zeros((n, 2), np.float32)
    rad = np.zeros(n, np.float32)
    if lib.orc_generate_per_body(name.encode(), n, seed, G, _p(mass), _p(pos), _p(vel), _p(rad)):
        raise ValueError(f"Unknown scenario: {name}")
    return mass, pos, vel, rad


def render_density(cam, width: int, height: int, pos, radius_multiplier) -> np.ndarray:
    """density.wgsl restated: (height, width) FP64 density, display orientation."""
    lib = load()
    cam = np.ascontiguousarray(cam, np.float32)
    pos = f32(pos, (-1, 2))
    rm = f32(radius_multiplier)
    out = np.zeros((height, width), np.float64)
    lib.orc_render_density(_p(cam), width, height, rm.size, _p(pos), _p(rm), _p(out))
    return out


def tone_map(density) -> np.ndarray:
    """tone_map.wgsl restated: RGBA8 image of a (height, width) float32 density."""
    lib = load()
    d = f32(density)
    h, w = np.shape(density)
    out = np.zeros((h, w, 4), np.uint8)
    lib.orc_tone_map(h * w, _p(d), _p(out))
    return out


def splat_weight(ux: float, uy: float, radius_multiplier: float, zoom_scale: float):
    """(density added, discarded) of one pixel at quad coordinates (ux, uy)."""
    d = ctypes.c_int(0)
    w = load().orc_splat_weight(ux, uy, radius_multiplier, zoom_scale, ctypes.byref(d))
    return float(w), bool(d.value)


def tone_map_rgb(texel: float) -> np.ndarray:
    out = np.zeros(3, np.float32)
    load().orc_tone_map_rgb(float(texel), _p(out))
    return out


REF_RENDER_LIB = os.path.join(HERE, "_ref", "libref_render.so")


def ref_render_available() -> bool:
    return os.path.exists(REF_RENDER_LIB)


def _ref_render():
    lib = ctypes.CDLL(REF_RENDER_LIB)
    lib.ref_density_fragment.restype = ctypes.c_float
    lib.ref_density_fragment.argtypes = [ctypes.c_float] * 5 + [ctypes.POINTER(ctypes.c_int)]
    lib.ref_tone_map_fragment.restype = None
    lib.ref_tone_map_fragment.argtypes = [ctypes.c_float, _P]
    lib.ref_colormap.restype = None
    lib.ref_colormap.argtypes = [ctypes.c_float, _P]
    return lib


def ref_density_fragment(ux, uy, radius_multiplier, half_x, half_y):
    """The reference's translated density.wgsl fragment: (density, discarded)."""
    d = ctypes.c_int(0)
    w = _ref_render().ref_density_fragment(ux, uy, radius_multiplier, half_x, half_y,
                                           ctypes.byref(d))
    return float(w), bool(d.value)


def ref_tone_map_fragment(texel: float) -> np.ndarray:
    out = np.zeros(3, np.float32)
    _ref_render().ref_tone_map_fragment(float(texel), _p(out))
    return out


def ref_colormap(t: float) -> np.ndarray:
    """The reference's translated colormap (tone_map.wgsl:24-46)."""
    out = np.zeros(3, np.float32)
    _ref_render().ref_colormap(float(t), _p(out))
    return out


def colormap(t: float) -> np.ndarray:
    lib = load()
    out = np.zeros(3, np.float32)
    lib.orc_colormap(float(t), _p(out))
    return out


REF_LIB = os.path.join(HERE, "_ref", "libref_wgsl.so")
_ref = None


def ref_available() -> bool:
    return os.path.exists(REF_LIB)


def _ref_lib():
    global _ref
    if _ref is None:
        lib = ctypes.CDLL(REF_LIB)
        lib.ref_run.restype = ctypes.c_int
        lib.ref_run.argtypes = [ctypes.c_uint32, _P, _P, _P, ctypes.c_float, ctypes.c_float,
                                ctypes.c_float, ctypes.c_float, ctypes.c_uint32, ctypes.c_uint32,
                                ctypes.c_int] + [_P] * 11
        lib.ref_max_threads.restype = ctypes.c_int
        lib.ref_max_threads.argtypes = []
        lib.ref_run_timed.restype = ctypes.c_int
        lib.ref_run_timed.argtypes = [ctypes.c_uint32, _P, _P, _P, ctypes.c_float, ctypes.c_float,
                                      ctypes.c_float, ctypes.c_float, ctypes.c_uint32,
                                      ctypes.c_uint32, ctypes.c_int, _P]
        _ref = lib
    return _ref


def ref_threads() -> int:
    return _ref_lib().ref_max_threads()


def ref_run(mass, pos, vel, G=1.0, dt=0.1 / 60.0, eps_mult=1.0, theta=0.6, offset=0, steps=1,
            parallel=False):
    """Run the mechanically translated reference WGSL (oracle/_ref) for
    `steps` steps; returns the final state and the last step's tree.
    parallel=True runs the independent stages on all host threads (same
    results)."""
    _ref_lib()
    mass = f32(mass)
    pos = f32(pos, (-1, 2))
    vel = f32(vel, (-1, 2))
    n = mass.size
    nn = max(2 * n - 1, 1)
    out = dict(pos=np.zeros((n, 2), np.float32), vel=np.zeros((n, 2), np.float32),
               codes=np.zeros(n, np.uint32), ids=np.zeros(n, np.uint32),
               left=np.zeros(nn, np.uint32), right=np.zeros(nn, np.uint32),
               parent=np.zeros(nn, np.uint32), com=np.zeros((nn, 2), np.float32),
               mass=np.zeros(nn, np.float32), aabb=np.zeros((nn, 4), np.float32),
               length=np.zeros(nn, np.float32))
    _ref.ref_run(n, _p(mass), _p(pos), _p(vel), G, dt, eps_mult, theta, offset, steps,
                 1 if parallel else 0,
                 _p(out["pos"]), _p(out["vel"]), _p(out["codes"]), _p(out["ids"]), _p(out["left"]),
                 _p(out["right"]), _p(out["parent"]), _p(out["com"]), _p(out["mass"]),
                 _p(out["aabb"]), _p(out["length"]))
    return out


REF_STAGES = ("morton", "sort", "build_fill", "vel_step", "pos_step")


def ref_run_timed(mass, pos, vel, G=1.0, dt=0.1 / 60.0, eps_mult=1.0, theta=0.6, steps=1,
                  walk_stride=1, parallel=True) -> dict:
    """Wall time per stage of `steps` steps of the translated reference
    pipeline on all host threads; the velocity step (the walk) runs for every
    `walk_stride`-th sorted slot only, so its time is a sample to be scaled
    by walk_stride."""
    _ref_lib()
    mass = f32(mass)
    out = np.zeros(5, np.float64)
    rc = _ref.ref_run_timed(mass.size, _p(mass), _p(f32(pos, (-1, 2))), _p(f32(vel, (-1, 2))), G,
                            dt, eps_mult, theta, steps, walk_stride, 1 if parallel else 0, _p(out))
    if rc != 0:
        raise ValueError("ref_run_timed: bad arguments")
    return dict(zip(REF_STAGES, out.tolist()))


class State:
    """Whole-step oracle run (simulation.ts:386-425 stage order)."""

    def __init__(self, p: OrcParams, mass, pos, vel):
        self.lib = load()
        self.p = p
        self.mass = f32(mass)
        self.n = self.mass.size
        self._h = self.lib.orc_create(ctypes.byref(p), self.n, _p(self.mass),
                                      _p(f32(pos, (-1, 2))), _p(f32(vel, (-1, 2))))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self.lib.orc_destroy(h)
            self._h = None

    def step(self, nsteps: int = 1) -> None:
        self.lib.orc_step(self._h, nsteps)

    def accelerations(self) -> np.ndarray:
        acc = np.zeros((self.n, 2), np.float32)
        self.lib.orc_accelerations(self._h, _p(acc))
        return acc

    def state(self):
        pos = np.zeros((self.n, 2), np.float32)
        vel = np.zeros((self.n, 2), np.float32)
        self.lib.orc_get_state(self._h, _p(pos), _p(vel))
        return pos, vel

    def tree(self) -> dict:
        n = self.n
        nn = max(2 * n - 1, 1)
        codes = np.zeros(n, np.uint64)
        ids = np.zeros(n, np.uint32)
        left = np.zeros(nn, np.uint32)
        right = np.zeros(nn, np.uint32)
        parent = np.zeros(nn, np.uint32)
        com = np.zeros((nn, 2), np.float32)
        mnode = np.zeros(nn, np.float32)
        aabb = np.zeros((nn, 4), np.float32)
        length = np.zeros(nn, np.float32)
        self.lib.orc_get_tree(self._h, _p(codes), _p(ids), _p(left), _p(right), _p(parent),
                              _p(com), _p(mnode), _p(aabb), _p(length))
        return dict(codes=codes, ids=ids, left=left, right=right, parent=parent, com=com,
                    mass=mnode, aabb=aabb, length=length)
