"""ctypes wrapper over oracle/liboracle.so (the CPU restatement of the
reference), with the same method names as the package's VoxelPhysicsSystem so
that parity tests drive both sides the same way.  Test infrastructure only."""
from __future__ import annotations

import ctypes
import importlib
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
LIB_PATH = os.path.join(ORACLE_DIR, "liboracle.so")

abi = importlib.import_module("zig-voxel-physics_b200.abi")


def _build():
    srcs = [os.path.join(ORACLE_DIR, f) for f in ("oracle_capi.cpp", "vxp_oracle.hpp")]
    srcs.append(os.path.join(ROOT, "include", "vxp.h"))
    if not os.path.exists(LIB_PATH) or any(os.path.getmtime(s) > os.path.getmtime(LIB_PATH) for s in srcs):
        subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)


_build()
L = ctypes.CDLL(LIB_PATH)
_VP, _U32, _F, _I = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_float, ctypes.c_int
_PU32 = ctypes.POINTER(ctypes.c_uint32)
for name, res, args in [
    ("vxo_world_create", _VP, [_VP, _I]),
    ("vxo_world_destroy", None, [_VP]),
    ("vxo_collider_add", _I, [_VP, _U32, _F, _VP, _U32]),
    ("vxo_collider_edit", _I, [_VP, _U32, _VP, _VP, _U32, _I]),
    ("vxo_collider_read", _I, [_VP, _U32, _VP, _VP, _U32, _PU32]),
    ("vxo_invalidate_cache_for_body", _U32, [_VP, _U32]),
    ("vxo_bodies_set", _I, [_VP, _VP, _U32]),
    ("vxo_bodies_get", _I, [_VP, _VP, _U32]),
    ("vxo_step", _I, [_VP, _F, _VP, _U32]),
    ("vxo_narrow_phase", _I, [_VP, _VP, _U32]),
    ("vxo_solve", _I, [_VP, _F]),
    ("vxo_manifolds_get", _I, [_VP, _VP, _U32, _PU32]),
    ("vxo_stats_get", _I, [_VP, _VP]),
    ("vxo_colours_get", _I, [_VP, _VP, _U32, _PU32]),
    ("vxo_set_candidate_dump", _I, [_VP, _I]),
    ("vxo_set_substep_record", _I, [_VP, _I]),
    ("vxo_substeps_get", _I, [_VP, _VP, _U32, _PU32]),
    ("vxo_candidates_get", _I, [_VP, _VP, _U32, _PU32]),
    ("vxo_pairs_find", _I, [_VP, _F, _VP, _U32, _PU32]),
    ("vxo_world_aabbs", _I, [_VP, _VP, _VP, _U32]),
    ("vxo_islands_kat", _I, [_VP, _U32, _U32, _VP, _U32, _VP, _U32, _PU32, _PU32]),
    ("vxo_narrow_phase_threaded", _I, [_VP, _VP, _U32, _I]),
    ("vxo_step_threaded", _I, [_VP, _F, _VP, _U32, _I]),
    ("vxo_mass_properties", _I, [_F, _VP, _U32, _F, ctypes.POINTER(_F), _VP]),
    ("vxo_collider_metadata", _I, [_F, _VP, _U32, _VP, _VP, _PU32]),
    ("vxo_classify", ctypes.c_uint8, [_I, ctypes.c_uint8]),
    ("vxo_classify_from_neighbors", ctypes.c_uint8, [_I, _I, _I, _I, _I, _I, _I]),
    ("vxo_compute_normal_index", ctypes.c_uint8, [ctypes.c_uint8]),
    ("vxo_find_closest_normal", ctypes.c_uint8, [_F, _F, _F]),
    ("vxo_normal_vec", None, [ctypes.c_uint8, _VP]),
    ("vxo_should_collide", _I, [ctypes.c_uint8, ctypes.c_uint8]),
    ("vxo_feature_id", ctypes.c_uint64, [_VP, _VP]),
    ("vxo_brick_coords", None, [_VP, _VP, _VP]),
    ("vxo_sat_early_out", _I, [_VP, _VP]),
    ("vxo_sat_with_penetration", _I, [_VP, _VP, ctypes.POINTER(_F), _VP]),
    ("vxo_soft_params", None, [_F, _F, _F, _VP]),
    ("vxo_compute_orthogonal", None, [_VP, _VP]),
    ("vxo_integrate_rotation_small", None, [_VP, _VP, _VP]),
    ("vxo_integrate_rotation", None, [_VP, _VP, _F, _VP]),
    ("vxo_from_axis_angle", None, [_VP, _F, _VP]),
    ("vxo_transform_point", None, [_VP, _VP, _VP, _VP]),
    ("vxo_inverse_transform_point", None, [_VP, _VP, _VP, _VP]),
    ("vxo_quat_rotate", None, [_VP, _VP, _VP]),
    ("vxo_mat3_inverse", None, [_VP, _VP]),
    ("vxo_world_inv_inertia", None, [_VP, _VP, _VP]),
    ("vxo_sinf", _F, [_F]),
    ("vxo_cosf", _F, [_F]),
    ("vxo_manifold_replay", _I, [_VP, _VP, _U32, _VP, _PU32]),
    ("vxo_contact_manager_warm", _F, [ctypes.c_uint64, _F, ctypes.c_uint64]),
    ("vxo_cache_create", _VP, [_U32]),
    ("vxo_cache_destroy", None, [_VP]),
    ("vxo_cache_get", _I, [_VP, _VP, _VP, _VP, _PU32]),
    ("vxo_cache_put", None, [_VP, _VP, _VP, _VP, _I, _U32]),
    ("vxo_cache_invalidate", None, [_VP, _U32]),
    ("vxo_cache_begin_frame", None, [_VP]),
    ("vxo_cache_stats", None, [_VP, _VP]),
    ("vxo_cache_key_eq", _I, [_VP, _VP, _VP, _VP, _VP, _VP]),
    ("vxo_graph_colouring", _I, [_VP, _U32, _VP]),
    ("vxo_sleep_after", _I, [_U32, _F]),
    ("vxo_jp_priority", _U32, [_U32]),
]:
    fn = getattr(L, name)
    fn.restype = res
    fn.argtypes = args


def f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def mass_fn(vs, bricks, density):
    bricks = np.ascontiguousarray(bricks, dtype=abi.BRICK_DTYPE)
    im = ctypes.c_float(0)
    inv = np.zeros(9, dtype=np.float32)
    rc = L.vxo_mass_properties(np.float32(vs), abi.ptr(bricks), len(bricks), np.float32(density), ctypes.byref(im),
                               abi.ptr(inv))
    assert rc == 0
    return np.float32(im.value), inv


def islands_kat(manifolds, body_count, types=None, n_ids=None):
    """The oracle's IslandManager over (a, b) manifolds: (island index per body
    id or -1, total islands, largest island size)."""
    ms = np.ascontiguousarray(np.array(manifolds, dtype=np.uint32).reshape(-1, 2)).view(abi.PAIR_DTYPE).reshape(-1)
    n_ids = body_count if n_ids is None else n_ids
    out = np.zeros(n_ids, dtype=np.int32)
    tot, lg = ctypes.c_uint32(0), ctypes.c_uint32(0)
    t = None if types is None else np.ascontiguousarray(types, dtype=np.uint32)
    assert L.vxo_islands_kat(abi.ptr(ms), len(ms), int(body_count), abi.ptr(t) if t is not None else None,
                             0 if t is None else len(t), abi.ptr(out), n_ids, ctypes.byref(tot), ctypes.byref(lg)) == 0
    return out, tot.value, lg.value


class OracleWorld:
    """The reference's VoxelPhysicsSystem step on the CPU (f32 or f64)."""

    def __init__(self, config=None, precision: int = 32, pair_margin: float = 0.1, **overrides):
        self.config = config if config is not None else abi.default_config(**overrides)
        self.h = L.vxo_world_create(ctypes.byref(self.config), precision)
        self.pair_margin = pair_margin
        self.n_bodies = 0

    def close(self):
        if self.h:
            L.vxo_world_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def add_collider(self, cid, vs, bricks):
        bricks = np.ascontiguousarray(bricks, dtype=abi.BRICK_DTYPE)
        assert L.vxo_collider_add(self.h, int(cid), np.float32(vs), abi.ptr(bricks), len(bricks)) == 0

    def edit_collider(self, cid, coords, values, mode="occupancy"):
        coords = np.ascontiguousarray(coords, dtype=np.int32).reshape(-1, 3)
        values = np.ascontiguousarray(values, dtype=np.uint8).reshape(-1)
        mode = {"set": abi.EDIT_SET, "occupancy": abi.EDIT_OCCUPANCY}.get(mode, mode)
        assert L.vxo_collider_edit(self.h, int(cid), abi.ptr(coords), abi.ptr(values), len(values), int(mode)) == 0

    def read_collider(self, cid):
        info = np.zeros(1, dtype=abi.COLLIDER_INFO_DTYPE)
        n = ctypes.c_uint32(0)
        assert L.vxo_collider_read(self.h, int(cid), abi.ptr(info), None, 0, ctypes.byref(n)) == 0
        bricks = np.zeros(n.value, dtype=abi.BRICK_DTYPE)
        assert L.vxo_collider_read(self.h, int(cid), abi.ptr(info), abi.ptr(bricks), len(bricks), ctypes.byref(n)) == 0
        return info[0], bricks

    def invalidate_cache_for_body(self, body_id):
        return int(L.vxo_invalidate_cache_for_body(self.h, int(body_id)))

    def set_bodies(self, bodies):
        bodies = np.ascontiguousarray(bodies, dtype=abi.BODY_DTYPE)
        assert L.vxo_bodies_set(self.h, abi.ptr(bodies), len(bodies)) == 0
        self.n_bodies = len(bodies)

    def load_scene(self, scene):
        for c in scene.colliders:
            self.add_collider(c.id, c.voxel_size, c.bricks)
        self.set_bodies(scene.bodies)

    def get_bodies(self):
        out = np.zeros(self.n_bodies, dtype=abi.BODY_DTYPE)
        assert L.vxo_bodies_get(self.h, abi.ptr(out), self.n_bodies) == 0
        return out

    def pairs(self, margin=None):
        m = self.pair_margin if margin is None else margin
        n = ctypes.c_uint32(0)
        L.vxo_pairs_find(self.h, np.float32(m), None, 0, ctypes.byref(n))
        out = np.zeros(n.value, dtype=abi.PAIR_DTYPE)
        assert L.vxo_pairs_find(self.h, np.float32(m), abi.ptr(out), len(out), ctypes.byref(n)) == 0
        return out

    def world_aabbs(self):
        """VoxelBody.getWorldAABB of every body: (min, max), each (n, 3) float32."""
        mn = np.zeros((self.n_bodies, 3), dtype=np.float32)
        mx = np.zeros((self.n_bodies, 3), dtype=np.float32)
        assert L.vxo_world_aabbs(self.h, abi.ptr(mn), abi.ptr(mx), self.n_bodies) == 0
        return mn, mx

    def step(self, dt, pairs=None):
        if pairs is None:
            pairs = self.pairs()
        pairs = np.ascontiguousarray(pairs, dtype=abi.PAIR_DTYPE)
        assert L.vxo_step(self.h, np.float32(dt), abi.ptr(pairs), len(pairs)) == 0

    def narrow_phase(self, pairs):
        pairs = np.ascontiguousarray(pairs, dtype=abi.PAIR_DTYPE)
        assert L.vxo_narrow_phase(self.h, abi.ptr(pairs), len(pairs)) == 0

    def narrow_phase_threaded(self, pairs, threads):
        pairs = np.ascontiguousarray(pairs, dtype=abi.PAIR_DTYPE)
        return L.vxo_narrow_phase_threaded(self.h, abi.ptr(pairs), len(pairs), int(threads))

    def step_threaded(self, dt, pairs, threads):
        pairs = np.ascontiguousarray(pairs, dtype=abi.PAIR_DTYPE)
        assert L.vxo_step_threaded(self.h, np.float32(dt), abi.ptr(pairs), len(pairs), int(threads)) == 0

    def solve(self, dt):
        assert L.vxo_solve(self.h, np.float32(dt)) == 0

    def manifolds(self):
        n = ctypes.c_uint32(0)
        L.vxo_manifolds_get(self.h, None, 0, ctypes.byref(n))
        out = np.zeros(n.value, dtype=abi.MANIFOLD_DTYPE)
        L.vxo_manifolds_get(self.h, abi.ptr(out), len(out), ctypes.byref(n))
        return out

    def stats(self):
        s = abi.Stats()
        L.vxo_stats_get(self.h, ctypes.byref(s))
        return s.as_dict()

    def colours(self):
        n = ctypes.c_uint32(0)
        L.vxo_colours_get(self.h, None, 0, ctypes.byref(n))
        out = np.zeros(n.value, dtype=np.uint32)
        overflow = L.vxo_colours_get(self.h, abi.ptr(out), len(out), ctypes.byref(n))
        return out, bool(overflow)

    def set_substep_record(self, on=True):
        L.vxo_set_substep_record(self.h, 1 if on else 0)

    def substeps(self):
        """Body states after each substep of the last step: (substeps, bodies, 13) float32
        (position, rotation, linear velocity, angular velocity)."""
        n = len(self.get_bodies())
        cap = 64 * n * 13
        out = np.zeros(cap, dtype=np.float32)
        ns = ctypes.c_uint32(0)
        L.vxo_substeps_get(self.h, out.ctypes.data, cap, ctypes.byref(ns))
        return out[: ns.value * n * 13].reshape(ns.value, n, 13)

    def set_candidate_dump(self, on=True):
        L.vxo_set_candidate_dump(self.h, 1 if on else 0)

    def candidates(self):
        n = ctypes.c_uint32(0)
        L.vxo_candidates_get(self.h, None, 0, ctypes.byref(n))
        out = np.zeros(n.value, dtype=abi.CANDIDATE_DTYPE)
        L.vxo_candidates_get(self.h, abi.ptr(out), len(out), ctypes.byref(n))
        return out
