"""ctypes binding of include/bh.h (libbh_b200.so).

Loading fails loudly when the library is missing: there is no fallback path.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# BH_B200_LIB overrides the library location (e.g. a build with other tunables).
LIB_PATH = os.environ.get("BH_B200_LIB") or os.path.join(HERE, "libbh_b200.so")

BH_OK = 0
BH_ERR_INVALID_ARGUMENT = 1
BH_ERR_CUDA = 2
BH_ERR_OUT_OF_MEMORY = 3
BH_ERR_UNKNOWN_SCENARIO = 4
BH_ERR_DEVICE_CHECK = 5
BH_ERR_NO_DEVICE = 6
BH_ERR_NOT_SUPPORTED = 7

BH_SOFTENING_REFERENCE = 0
BH_SOFTENING_PLUMMER = 1
BH_DOMAIN_FIXED2000 = 0
BH_DOMAIN_BBOX = 1
BH_INTEGRATOR_SYMPLECTIC_EULER = 0
BH_INTEGRATOR_LEAPFROG_KDK = 1

BH_STAGE_NAMES = ("morton", "sort", "tree", "walk", "other")

BH_DEBUG_LOOKBACK_UNPUBLISHED = 1
BH_DEBUG_SPLIT_BUILD = 2


class bh_config(ctypes.Structure):
    _fields_ = [
        ("grav_constant", ctypes.c_float),
        ("bh_theta", ctypes.c_float),
        ("substeps", ctypes.c_int32),
        ("delta_time", ctypes.c_float),
        ("epsilon_multiplier", ctypes.c_float),
        ("softening", ctypes.c_int32),
        ("plummer_eps", ctypes.c_float),
        ("morton_bits", ctypes.c_int32),
        ("morton_domain", ctypes.c_int32),
        ("integrator", ctypes.c_int32),
        ("leaf_size", ctypes.c_int32),
        ("walk_block", ctypes.c_int32),
        ("device", ctypes.c_int32),
        ("use_graphs", ctypes.c_int32),
        ("fp64_levels", ctypes.c_int32),
        ("walk_mode", ctypes.c_int32),
        ("multipole_order", ctypes.c_int32),
        ("bodies_per_lane", ctypes.c_int32),
        ("far_alpha", ctypes.c_float),
        ("reserved", ctypes.c_int32 * 3),
    ]


BH_WALK_EXACT = 0
BH_WALK_GROUP = 1


class bh_tune_result(ctypes.Structure):
    _fields_ = [
        ("bodies_per_lane", ctypes.c_int32),
        ("leaf_size", ctypes.c_int32),
        ("walk_ms", ctypes.c_float),
        ("candidates", ctypes.c_int32),
        ("walk_block", ctypes.c_int32),
    ]


class bh_buffers(ctypes.Structure):
    _fields_ = [
        ("mass", ctypes.c_void_p),
        ("pos", ctypes.c_void_p),
        ("vel", ctypes.c_void_p),
        ("radius_multiplier", ctypes.c_void_p),
        ("acc", ctypes.c_void_p),
        ("morton_codes", ctypes.c_void_p),
        ("body_indices", ctypes.c_void_p),
        ("node4", ctypes.c_void_p),
        ("node_children", ctypes.c_void_p),
        ("node_parent", ctypes.c_void_p),
        ("node_aabb", ctypes.c_void_p),
        ("num_bodies", ctypes.c_uint32),
        ("morton_bits", ctypes.c_int32),
        ("stream", ctypes.c_void_p),
    ]


class bh_diagnostics(ctypes.Structure):
    _fields_ = [
        ("total_mass", ctypes.c_double),
        ("com", ctypes.c_double * 2),
        ("momentum", ctypes.c_double * 2),
        ("angular_momentum", ctypes.c_double),
        ("kinetic_energy", ctypes.c_double),
        ("potential_energy", ctypes.c_double),
        ("pairs", ctypes.c_uint64),
    ]


# name -> (restype, argtypes); every symbol declared in include/bh.h
_P = ctypes.c_void_p
_F = ctypes.POINTER(ctypes.c_float)
SIGNATURES = {
    "bh_default_config": (ctypes.c_int, [ctypes.POINTER(bh_config)]),
    "bh_create": (ctypes.c_int, [ctypes.POINTER(bh_config), ctypes.POINTER(_P)]),
    "bh_destroy": (ctypes.c_int, [_P]),
    "bh_set_num_bodies": (ctypes.c_int, [_P, ctypes.c_uint32]),
    "bh_set_scenario": (ctypes.c_int, [_P, ctypes.c_char_p, ctypes.c_uint64]),
    "bh_update_metadata": (ctypes.c_int, [_P]),
    "bh_upload": (ctypes.c_int, [_P, _P, _P, _P, ctypes.c_uint32]),
    "bh_download": (ctypes.c_int, [_P, _P, _P, _P, ctypes.c_uint32]),
    "bh_download_async": (ctypes.c_int, [_P, _P, _P, _P, ctypes.c_uint32]),
    "bh_step": (ctypes.c_int, [_P, ctypes.c_uint32]),
    "bh_sync": (ctypes.c_int, [_P]),
    "bh_compute_accelerations": (ctypes.c_int, [_P, _P]),
    "bh_get_buffers": (ctypes.c_int, [_P, ctypes.POINTER(bh_buffers)]),
    "bh_get_num_bodies": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_uint32)]),
    "bh_read_buffer": (ctypes.c_int, [_P, ctypes.c_char_p, _P, ctypes.c_size_t]),
    "bh_generate_scenario": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_uint32, ctypes.c_uint64,
                                            ctypes.c_float, _P, _P, _P, _P]),
    "bh_profile_begin": (ctypes.c_int, [_P, ctypes.c_uint32]),
    "bh_profile_end": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_double),
                                      ctypes.POINTER(ctypes.c_uint32)]),
    "bh_kernels_per_step": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_uint32)]),
    "bh_walk_stats": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_uint64),
                                     ctypes.POINTER(ctypes.c_uint64),
                                     ctypes.POINTER(ctypes.c_uint64),
                                     ctypes.POINTER(ctypes.c_uint64)]),
    "bh_ensemble_create": (ctypes.c_int, [ctypes.POINTER(bh_config), _P, ctypes.c_uint32,
                                          ctypes.POINTER(_P)]),
    "bh_ensemble_set_scenarios": (ctypes.c_int, [_P, _P, ctypes.c_uint64]),
    "bh_ensemble_sizes": (ctypes.c_int, [ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint32,
                                         ctypes.c_uint32, _P]),
    "bh_get_num_systems": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_uint32)]),
    "bh_get_system_offsets": (ctypes.c_int, [_P, _P]),
    "bh_autotune": (ctypes.c_int, [_P, ctypes.c_uint32, ctypes.POINTER(bh_tune_result)]),
    "bh_get_config": (ctypes.c_int, [_P, ctypes.POINTER(bh_config)]),
    "bh_force_vjp": (ctypes.c_int, [_P, _P, _P, _P]),
    "bh_rollout_grad": (ctypes.c_int, [_P, ctypes.c_uint32, ctypes.c_uint32, _P,
                                       ctypes.POINTER(ctypes.c_float), _P, _P, _P]),
    "bh_build_hierarchy_static": (ctypes.c_int, [_P, ctypes.c_int32, _P, _P, _P, ctypes.c_uint32,
                                                 _P, _P, _P, _P, ctypes.c_int32, _P]),
    "bh_set_scenario_device": (ctypes.c_int, [_P, ctypes.c_char_p, ctypes.c_uint64]),
    "bh_generate_scenario_device": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_uint32, ctypes.c_uint64,
                                                   ctypes.c_float, _P, _P, _P, _P, _P]),
    "bh_set_walk_slots": (ctypes.c_int, [_P, ctypes.c_uint32, ctypes.c_uint32]),
    "bh_shard_pack": (ctypes.c_int, [_P, _P, ctypes.c_uint32]),
    "bh_shard_unpack": (ctypes.c_int, [_P, _P, ctypes.c_uint32, ctypes.c_uint32]),
    "bh_diagnostics_compute": (ctypes.c_int, [_P, ctypes.c_int, ctypes.POINTER(bh_diagnostics)]),
    "bh_direct_forces_fp64": (ctypes.c_int, [_P, _P, ctypes.c_uint32, _P]),
    "bh_debug_set_limits": (ctypes.c_int, [_P, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32]),
    "bh_renderer_create": (ctypes.c_int, [_P, ctypes.c_uint32, ctypes.c_uint32, ctypes.POINTER(_P)]),
    "bh_renderer_destroy": (ctypes.c_int, [_P]),
    "bh_renderer_resize": (ctypes.c_int, [_P, ctypes.c_uint32, ctypes.c_uint32]),
    "bh_renderer_pan": (ctypes.c_int, [_P, ctypes.c_float, ctypes.c_float]),
    "bh_renderer_zoom": (ctypes.c_int, [_P, ctypes.c_float, ctypes.c_float, ctypes.c_float]),
    "bh_renderer_set_camera": (ctypes.c_int, [_P, _F]),
    "bh_renderer_get_camera": (ctypes.c_int, [_P, _F]),
    "bh_renderer_frame": (ctypes.c_int, [_P]),
    "bh_renderer_get_targets": (ctypes.c_int, [_P, ctypes.POINTER(_P), ctypes.POINTER(_P),
                                               ctypes.POINTER(ctypes.c_uint32),
                                               ctypes.POINTER(ctypes.c_uint32)]),
    "bh_renderer_read_density": (ctypes.c_int, [_P, _P]),
    "bh_renderer_read_image": (ctypes.c_int, [_P, _P]),
    "bh_renderer_last_error": (ctypes.c_char_p, [_P]),
    "bh_last_error": (ctypes.c_char_p, [_P]),
    "bh_global_last_error": (ctypes.c_char_p, []),
    "bh_version": (ctypes.c_char_p, []),
}

_lib = None


def load(path: str | None = None) -> ctypes.CDLL:
    """Load libbh_b200.so (once) and attach the prototypes of include/bh.h."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(
            f"{p} is missing: build the CUDA engine first (python webgpu-fluid-sim_b200/build.py); "
            "the engine has no CPU fallback")
    lib = ctypes.CDLL(p)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


class BhError(RuntimeError):
    """A non-zero status from the engine, with the handle's message."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


def check(status: int, handle=None) -> None:
    if status == BH_OK:
        return
    lib = load()
    msg = lib.bh_last_error(handle) if handle else lib.bh_global_last_error()
    raise BhError(status, (msg or b"").decode(errors="replace") or f"bh status {status}")
