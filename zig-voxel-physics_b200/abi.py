"""ctypes / numpy mirror of include/vxp.h.

The numpy dtypes describe the same bytes as the C structs so that arrays of
bodies, bricks, pairs and manifolds cross the C ABI without copies.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

VXP_OK = 0
VXP_ERR_ARG = -1
BATCH_SCHEDULES = 8  # VXP_BATCH_SCHEDULES
VXP_ERR_OOM = -2
VXP_ERR_CUDA = -3
VXP_ERR_TIMEOUT = -4
VXP_ERR_CAP = -5
VXP_ERR_STATE = -6

BODY_STATIC, BODY_KINEMATIC, BODY_DYNAMIC = 0, 1, 2
COLOUR_PROJECT, COLOUR_REFERENCE = 0, 1

BRICK_DTYPE = np.dtype([("pos", "<i4", (3,)), ("voxels", "u1", (512,))], align=False)
assert BRICK_DTYPE.itemsize == 524

EDIT_SET, EDIT_OCCUPANCY = 0, 1

# vxp_collider_info
COLLIDER_INFO_DTYPE = np.dtype(
    [
        ("voxel_size", "<f4"),
        ("min_bound", "<i4", (3,)),
        ("max_bound", "<i4", (3,)),
        ("aabb_min", "<f4", (3,)),
        ("aabb_max", "<f4", (3,)),
        ("solid_count", "<u4"),
        ("n_bricks", "<u4"),
        ("has_table", "<u4"),
    ]
)
assert COLLIDER_INFO_DTYPE.itemsize == 64

BODY_DTYPE = np.dtype(
    [
        ("id", "<u4"),
        ("body_type", "<u4"),
        ("collider_id", "<u4"),
        ("is_sleeping", "<u4"),
        ("position", "<f4", (3,)),
        ("rotation", "<f4", (4,)),
        ("linear_velocity", "<f4", (3,)),
        ("angular_velocity", "<f4", (3,)),
        ("inv_mass", "<f4"),
        ("inv_inertia_local", "<f4", (9,)),
        ("friction", "<f4"),
        ("restitution", "<f4"),
        ("linear_damping", "<f4"),
        ("angular_damping", "<f4"),
        ("sleep_timer", "<f4"),
    ]
)
assert BODY_DTYPE.itemsize == 128

PAIR_DTYPE = np.dtype([("body_a", "<u4"), ("body_b", "<u4")])

CONTACT_DTYPE = np.dtype(
    [
        ("point", "<f4", (3,)),
        ("normal", "<f4", (3,)),
        ("penetration", "<f4"),
        ("local_anchor_a", "<f4", (3,)),
        ("local_anchor_b", "<f4", (3,)),
        ("normal_impulse", "<f4"),
        ("tangent_impulse", "<f4", (2,)),
        ("normal_mass", "<f4"),
        ("tangent_mass", "<f4", (2,)),
        ("_pad", "<u4"),
        ("feature_id", "<u8"),
    ]
)
assert CONTACT_DTYPE.itemsize == 88

MANIFOLD_DTYPE = np.dtype(
    [
        ("body_a_id", "<u4"),
        ("body_b_id", "<u4"),
        ("contact_count", "<u4"),
        ("friction", "<f4"),
        ("restitution", "<f4"),
        ("_pad", "<u4"),
        ("contacts", CONTACT_DTYPE, (4,)),
    ]
)
assert MANIFOLD_DTYPE.itemsize == 376

CANDIDATE_DTYPE = np.dtype(
    [("pair_index", "<u4"), ("a", "<i4", (3,)), ("b", "<i4", (3,)), ("passed", "<u4"), ("dist_sq", "<f4")]
)
assert CANDIDATE_DTYPE.itemsize == 36


class Config(ctypes.Structure):
    """vxp_config: PhysicsConfig + SolverConfig + NarrowPhaseConfig + flags."""

    _fields_ = [
        ("gravity", ctypes.c_float * 3),
        ("fixed_timestep", ctypes.c_float),
        ("enable_sleeping", ctypes.c_uint32),
        ("enable_warm_starting", ctypes.c_uint32),
        ("substeps", ctypes.c_uint32),
        ("velocity_iterations", ctypes.c_uint32),
        ("position_iterations", ctypes.c_uint32),
        ("disable_rotation", ctypes.c_uint32),
        ("hertz", ctypes.c_float),
        ("damping_ratio", ctypes.c_float),
        ("position_correction_rate", ctypes.c_float),
        ("max_position_correction", ctypes.c_float),
        ("slop", ctypes.c_float),
        ("warm_starting", ctypes.c_uint32),
        ("warm_start_scale", ctypes.c_float),
        ("enable_friction", ctypes.c_uint32),
        ("enable_restitution", ctypes.c_uint32),
        ("use_brick_sat", ctypes.c_uint32),
        ("use_brick_pair_cache", ctypes.c_uint32),
        ("brick_pair_cache_size", ctypes.c_uint32),
        ("reference_caps", ctypes.c_uint32),
        ("colouring", ctypes.c_uint32),
        ("enable_islands", ctypes.c_uint32),
        ("max_bodies", ctypes.c_uint32),
        ("max_pairs", ctypes.c_uint32),
    ]


class Stats(ctypes.Structure):
    """vxp_stats."""

    _fields_ = [
        ("pairs_in", ctypes.c_uint32),
        ("pairs_tested", ctypes.c_uint32),
        ("pairs_colliding", ctypes.c_uint32),
        ("voxels_checked", ctypes.c_uint32),
        ("contacts_generated", ctypes.c_uint32),
        ("pairs_skipped_sleeping", ctypes.c_uint32),
        ("manifolds_preserved", ctypes.c_uint32),
        ("cache_hits", ctypes.c_uint32),
        ("cache_misses", ctypes.c_uint32),
        ("cache_evictions", ctypes.c_uint32),
        ("manifolds", ctypes.c_uint32),
        ("constraints", ctypes.c_uint32),
        ("contact_points", ctypes.c_uint32),
        ("colours", ctypes.c_uint32),
        ("position_iterations_run", ctypes.c_uint32),
        ("step_skipped", ctypes.c_uint32),
        ("max_penetration", ctypes.c_float),
        ("candidates", ctypes.c_uint32),
        ("bricks_touched", ctypes.c_uint32),
        ("sweep_path", ctypes.c_uint32),
        ("island_count", ctypes.c_uint32),
        ("active_islands", ctypes.c_uint32),
        ("sleeping_islands", ctypes.c_uint32),
        ("largest_island_size", ctypes.c_uint32),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class StateView(ctypes.Structure):
    """vxp_state_view: one pointer per exported field (null = skipped)."""
    _fields_ = [
        ("position", ctypes.c_void_p),
        ("rotation", ctypes.c_void_p),
        ("linear_velocity", ctypes.c_void_p),
        ("angular_velocity", ctypes.c_void_p),
        ("aabb_min", ctypes.c_void_p),
        ("aabb_max", ctypes.c_void_p),
        ("sleeping", ctypes.c_void_p),
    ]


# Exported fields and their per-body shape and type (vxp_bodies_export).
EXPORT_FIELDS = {
    "position": (3, np.float32), "rotation": (4, np.float32), "linear_velocity": (3, np.float32),
    "angular_velocity": (3, np.float32), "aabb_min": (3, np.float32), "aabb_max": (3, np.float32),
    "sleeping": (1, np.uint8),
}


def default_config(**overrides) -> Config:
    """The reference defaults: PhysicsConfig{} + SolverConfig{} + NarrowPhaseConfig{}
    (system.zig:47-88, solver.zig:75-119, narrow_phase.zig:1325-1343)."""
    c = Config()
    c.gravity[:] = (0.0, -9.81, 0.0)
    c.fixed_timestep = np.float32(1.0) / np.float32(60.0)
    c.enable_sleeping = 1
    c.enable_warm_starting = 1
    c.substeps = 4
    c.velocity_iterations = 1
    c.position_iterations = 2
    c.disable_rotation = 0
    c.hertz = 30.0
    c.damping_ratio = 1.0
    c.position_correction_rate = 0.2
    c.max_position_correction = 0.04
    c.slop = 0.005
    c.warm_starting = 1
    c.warm_start_scale = 0.8
    c.enable_friction = 1
    c.enable_restitution = 1
    c.use_brick_sat = 1
    c.use_brick_pair_cache = 1
    c.brick_pair_cache_size = 1024
    c.reference_caps = 0
    c.colouring = COLOUR_PROJECT
    c.enable_islands = 1
    c.max_bodies = 0
    c.max_pairs = 0
    for k, v in overrides.items():
        if k == "gravity":
            c.gravity[:] = v
        else:
            setattr(c, k, v)
    return c


def ptr(a: np.ndarray) -> ctypes.c_void_p:
    return ctypes.c_void_p(a.ctypes.data) if a is not None and a.size else ctypes.c_void_p(0)


# Every symbol include/vxp.h declares, with its ctypes signature.
_VP = ctypes.c_void_p
_U32 = ctypes.c_uint32
_F = ctypes.c_float
_I = ctypes.c_int
_PU32 = ctypes.POINTER(ctypes.c_uint32)
SIGNATURES = {
    "vxp_config_default": (None, [_VP]),
    "vxp_create": (_I, [_VP, _I, ctypes.POINTER(_VP)]),
    "vxp_destroy": (None, [_VP]),
    "vxp_last_error": (_I, [_VP, ctypes.c_char_p, ctypes.c_size_t]),
    "vxp_abi_version": (_I, []),
    "vxp_collider_upload": (_I, [_VP, _U32, _F, _VP, _U32]),
    "vxp_collider_edit": (_I, [_VP, _U32, _VP, _VP, _U32, _I]),
    "vxp_collider_read": (_I, [_VP, _U32, _VP, _VP, _U32, _VP]),
    "vxp_invalidate_cache_for_body": (_I, [_VP, _U32, _VP]),
    "vxp_bodies_set": (_I, [_VP, _VP, _U32]),
    "vxp_bodies_get": (_I, [_VP, _VP, _U32]),
    "vxp_bodies_export": (_I, [_VP, _VP, _U32, _U32, _I, _VP]),
    "vxp_mass_properties": (_I, [_F, _VP, _U32, _F, ctypes.POINTER(_F), _VP]),
    "vxp_step": (_I, [_VP, _F, _VP, _U32]),
    "vxp_step_device_pairs": (_I, [_VP, _F, _F]),
    "vxp_narrow_phase": (_I, [_VP, _VP, _U32]),
    "vxp_solve": (_I, [_VP, _F]),
    "vxp_manifolds_get": (_I, [_VP, _VP, _U32, _PU32]),
    "vxp_set_candidate_dump": (_I, [_VP, _U32]),
    "vxp_candidates_get": (_I, [_VP, _VP, _U32, _PU32]),
    "vxp_stats_get": (_I, [_VP, _VP]),
    "vxp_colours_get": (_I, [_VP, _VP, _U32, _PU32]),
    "vxp_pairs_from_bodies": (_I, [_VP, _F, _VP, _U32, _PU32]),
    "vxp_last_step_ms": (_I, [_VP, _VP]),
    "vxp_last_kernel_ms": (_I, [_VP, _VP]),
    "vxp_last_solve_split_ms": (_I, [_VP, _VP]),
    "vxp_cluster_size": (_I, [_VP, _VP]),
    "vxp_set_cluster_shared_bytes": (_I, [_VP, _U32]),
    "vxp_set_cluster_constraints": (_I, [_VP, _I]),
    "vxp_set_traffic_accounting": (_I, [_VP, _I]),
    "vxp_snapshot_substeps": (_I, [_VP, _I]),
    "vxp_substeps_get": (_I, [_VP, _VP, _U32, _VP]),
    "vxp_synchronize": (_I, [_VP]),
    "vxp_set_launch_mode": (_I, [_VP, _I]),
    "vxp_phase_times": (_I, [_VP, _VP, _U32]),
    "vxp_set_solver_blocks_divisor": (_I, [_VP, _U32]),
    "vxp_set_solver_mode": (_I, [_VP, _U32]),
    "vxp_set_heavy_pair_voxels": (_I, [_VP, _U32]),
    "vxp_set_wait_limit_ns": (_I, [_VP, ctypes.c_uint64]),
    "vxp_set_probe_tables": (_I, [_VP, _I]),
    "vxp_pairs_noalloc": (_I, [_VP, _VP, _VP, _VP, _VP, _U32, _F, _VP, _U32, _VP, _VP]),
    "vxp_batch_create": (_I, [_VP, _I, _U32, ctypes.POINTER(_VP)]),
    "vxp_batch_destroy": (None, [_VP]),
    "vxp_batch_last_error": (_I, [_VP, ctypes.c_char_p, ctypes.c_size_t]),
    "vxp_batch_collider_upload": (_I, [_VP, _U32, _F, _VP, _U32]),
    "vxp_batch_collider_edit": (_I, [_VP, _U32, _VP, _VP, _U32, _I]),
    "vxp_batch_collider_read": (_I, [_VP, _U32, _VP, _VP, _U32, _VP]),
    "vxp_batch_invalidate_cache_for_body": (_I, [_VP, _U32, _U32, _VP]),
    "vxp_batch_world_set": (_I, [_VP, _U32, _VP, _U32, _U32]),
    "vxp_batch_world_clear": (_I, [_VP, _U32]),
    "vxp_batch_world_release": (_I, [_VP, _U32]),
    "vxp_batch_world_export": (_I, [_VP, _U32, _VP, _U32, _U32, _I, _VP]),
    "vxp_batch_world_get": (_I, [_VP, _U32, _VP, _U32]),
    "vxp_batch_world_stats": (_I, [_VP, _U32, _VP]),
    "vxp_batch_world_bytes": (ctypes.c_uint64, [_VP, _U32]),
    "vxp_batch_step": (_I, [_VP, _F, _U32]),
    "vxp_batch_synchronize": (_I, [_VP]),
    "vxp_batch_times": (_I, [_VP, _VP, _VP, _U32]),
    "vxp_batch_set_schedule": (_I, [_VP, _U32, _U32]),
    "vxp_batch_autotune": (_I, [_VP, _F, _U32, _VP, _VP]),
    "vxp_batch_set_tiles": (_I, [_VP, _U32, _U32]),
}

_LIB = None


def lib_path() -> str:
    return os.path.join(HERE, "libvxp.so")


def load(path: str | None = None) -> ctypes.CDLL:
    """Loads libvxp.so (built in-tree).  Raises if it is missing: there is no
    CPU fallback for the hot path."""
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    p = path or lib_path()
    if not os.path.exists(p):
        raise RuntimeError(f"libvxp.so not built at {p}; run __graft_entry__.build()")
    lib = ctypes.CDLL(p)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _LIB = lib
    return lib


def declared_symbols(header: str) -> list[str]:
    """Function names declared in a C header (for the symbol-export test)."""
    import re

    src = open(header).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(vxp_[a-z0-9_]+)\s*\(", src)))
