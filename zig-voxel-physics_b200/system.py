"""Host-side mirror of the reference's VoxelPhysicsSystem seams over the C ABI.

The reference drives its hot path from VoxelPhysicsSystem.step
(src/system.zig:537-555): narrowPhase() then solve() then
updateSleepStates().  This module keeps that call shape:

    sys = VoxelPhysicsSystem(PhysicsConfig)      # NarrowPhase.init / ContactSolver.init
    sys.add_collider(id, voxel_size, bricks)     # VoxelCollider (recomputeMetadata)
    sys.set_bodies(table)                        # the body slots (VoxelBody)
    sys.update(dt)                               # accumulator loop -> step(fixed_timestep)
    sys.step(dt, pairs)                          # one VoxelPhysicsSystem.step
    sys.narrow_phase(pairs); sys.solve(dt)       # the two halves, for tests

Every call goes to libvxp.so; there is no CPU path.  Errors raise VxpError
with the library's message (the reference swallows most errors with
`catch {}`; here they surface).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import abi


class VxpError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"vxp error {code}: {msg}")
        self.code = code


def _edit_args(coords, values, mode):
    coords = np.ascontiguousarray(coords, dtype=np.int32).reshape(-1, 3)
    values = np.ascontiguousarray(values, dtype=np.uint8).reshape(-1)
    if len(values) != len(coords):
        raise ValueError("one value per voxel")
    mode = {"set": abi.EDIT_SET, "occupancy": abi.EDIT_OCCUPANCY}.get(mode, mode)
    return coords, values, int(mode)


def _read_collider(fn, handle, collider_id):
    info = np.zeros(1, dtype=abi.COLLIDER_INFO_DTYPE)
    n = ctypes.c_uint32(0)
    rc = fn(handle, int(collider_id), abi.ptr(info), None, 0, ctypes.byref(n))
    if rc != 0:
        return rc, None, None
    bricks = np.zeros(n.value, dtype=abi.BRICK_DTYPE)
    rc = fn(handle, int(collider_id), abi.ptr(info), abi.ptr(bricks), len(bricks), ctypes.byref(n))
    return rc, info[0], bricks


class VoxelPhysicsSystem:
    """One simulated world on one GPU."""

    def __init__(self, config: abi.Config | None = None, device: int = 0, pair_margin: float = 0.1, **overrides):
        self.lib = abi.load()
        self.config = config if config is not None else abi.default_config(**overrides)
        h = ctypes.c_void_p()
        rc = self.lib.vxp_create(ctypes.byref(self.config), device, ctypes.byref(h))
        if rc != 0 or not h.value:
            raise VxpError(rc, "vxp_create failed")
        self.ctx = h
        self.pair_margin = float(pair_margin)
        self.accumulated_time = np.float32(0.0)
        self.n_bodies = 0
        self._last_pairs = 0

    # ------------------------------------------------------------------ utils
    def _check(self, rc: int) -> None:
        if rc != 0:
            buf = ctypes.create_string_buffer(512)
            self.lib.vxp_last_error(self.ctx, buf, len(buf))
            raise VxpError(rc, buf.value.decode(errors="replace"))

    def close(self) -> None:
        if getattr(self, "ctx", None) is not None and self.ctx.value:
            self.lib.vxp_destroy(self.ctx)
            self.ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ------------------------------------------------------- scene building
    def add_collider(self, collider_id: int, voxel_size: float, bricks: np.ndarray) -> None:
        bricks = np.ascontiguousarray(bricks, dtype=abi.BRICK_DTYPE)
        self._check(self.lib.vxp_collider_upload(self.ctx, int(collider_id), np.float32(voxel_size),
                                                 abi.ptr(bricks), len(bricks)))

    def edit_collider(self, collider_id: int, coords, values, mode="occupancy") -> None:
        """Writes voxels of an uploaded collider on the device, then recomputes
        its metadata (vxp_collider_edit).  mode "set": values are CollisionVoxel
        bytes, stored as setCollisionVoxel stores them; "occupancy": nonzero
        makes the voxel solid, zero empty, and the written voxels and their
        solid face neighbours are re-typed by classifyFromNeighbors.  Queued
        after the steps already queued."""
        coords, values, mode = _edit_args(coords, values, mode)
        self._check(self.lib.vxp_collider_edit(self.ctx, int(collider_id), abi.ptr(coords), abi.ptr(values),
                                               len(values), mode))

    def read_collider(self, collider_id: int):
        """(info, bricks) of the collider as the device holds it: info is a
        COLLIDER_INFO_DTYPE record, bricks a BRICK_DTYPE array."""
        rc, info, bricks = _read_collider(self.lib.vxp_collider_read, self.ctx, collider_id)
        self._check(rc)
        return info, bricks

    def invalidate_cache_for_body(self, body_id: int) -> int:
        """NarrowPhase.invalidateCacheForBody: drops the body's brick-pair
        cache entries; returns how many there were."""
        n = ctypes.c_uint32(0)
        self._check(self.lib.vxp_invalidate_cache_for_body(self.ctx, int(body_id), ctypes.byref(n)))
        return int(n.value)

    def set_bodies(self, bodies: np.ndarray) -> None:
        bodies = np.ascontiguousarray(bodies, dtype=abi.BODY_DTYPE)
        self._check(self.lib.vxp_bodies_set(self.ctx, abi.ptr(bodies), len(bodies)))
        self.n_bodies = len(bodies)

    def get_bodies(self) -> np.ndarray:
        out = np.zeros(self.n_bodies, dtype=abi.BODY_DTYPE)
        self._check(self.lib.vxp_bodies_get(self.ctx, abi.ptr(out), self.n_bodies))
        return out

    def export_state(self, fields=None, first: int = 0, n: int | None = None) -> dict:
        """Bulk state for a renderer (vxp_bodies_export into host arrays):
        {field: array of shape (n, k)} for the fields asked (default all of
        position, rotation, linear_velocity, angular_velocity, aabb_min,
        aabb_max, sleeping), bodies [first, first + n) in set_bodies order."""
        n = self.n_bodies - first if n is None else n
        out, view = _export_arrays(fields, n)
        self._check(self.lib.vxp_bodies_export(self.ctx, ctypes.byref(view), int(first), int(n), 0, None))
        return out

    def export_state_to_device(self, pointers: dict, first: int = 0, n: int | None = None,
                               consumer_stream: int = 0) -> None:
        """vxp_bodies_export into caller-owned device memory: pointers maps
        field names to device addresses (ints) of arrays laid out as in
        export_state.  Returns without waiting; consumer_stream (a
        cudaStream_t as an int, 0 for none) waits for the export."""
        n = self.n_bodies - first if n is None else n
        view = _device_view(pointers)
        self._check(self.lib.vxp_bodies_export(self.ctx, ctypes.byref(view), int(first), int(n), 1,
                                               ctypes.c_void_p(consumer_stream or None)))

    def load_scene(self, scene) -> None:
        for c in scene.colliders:
            self.add_collider(c.id, c.voxel_size, c.bricks)
        self.set_bodies(scene.bodies)

    # ------------------------------------------------------------- stepping
    def step(self, dt: float, pairs: np.ndarray | None = None) -> None:
        """One VoxelPhysicsSystem.step.  With pairs=None the pair list is built on
        the device from the bodies' inflated AABBs."""
        if pairs is None:
            self._check(self.lib.vxp_step_device_pairs(self.ctx, np.float32(dt), np.float32(self.pair_margin)))
        else:
            pairs = np.ascontiguousarray(pairs, dtype=abi.PAIR_DTYPE)
            self._check(self.lib.vxp_step(self.ctx, np.float32(dt), abi.ptr(pairs), len(pairs)))
            self._last_pairs = len(pairs)

    def update(self, dt: float, pairs_fn=None) -> int:
        """VoxelPhysicsSystem.update (src/system.zig:508-534): fixed-timestep
        accumulator in f32, at most max_substeps (8) steps per call."""
        fixed = np.float32(self.config.fixed_timestep)
        self.accumulated_time = np.float32(self.accumulated_time + np.float32(dt))
        n = 0
        while self.accumulated_time >= fixed and n < 8:
            self.step(fixed, None if pairs_fn is None else pairs_fn())
            self.accumulated_time = np.float32(self.accumulated_time - fixed)
            n += 1
        if self.accumulated_time > np.float32(fixed * np.float32(8)):
            self.accumulated_time = fixed
        return n

    def narrow_phase(self, pairs: np.ndarray) -> None:
        pairs = np.ascontiguousarray(pairs, dtype=abi.PAIR_DTYPE)
        self._check(self.lib.vxp_narrow_phase(self.ctx, abi.ptr(pairs), len(pairs)))

    def solve(self, dt: float) -> None:
        self._check(self.lib.vxp_solve(self.ctx, np.float32(dt)))

    def synchronize(self) -> None:
        self._check(self.lib.vxp_synchronize(self.ctx))

    def set_launch_mode(self, mode: int) -> None:
        self._check(self.lib.vxp_set_launch_mode(self.ctx, int(mode)))

    # -------------------------------------------------------------- outputs
    def set_solver_mode(self, mode: int) -> None:
        """Grid-stepped worlds: 2 sweeps on one thread-block cluster with a
        cluster barrier after every colour batch and the state in shared
        memory (the default where cluster_size() > 0), 1 event-ordered sweeps
        (the default otherwise), 0 a grid barrier after every colour batch.
        Worlds stepped by one CTA use CTA barriers."""
        self._check(self.lib.vxp_set_solver_mode(self.ctx, int(mode)))

    def set_traffic_accounting(self, on: bool = True) -> None:
        """Count the bricks the probed pairs touch (stats bricks_touched; off by
        default, it costs narrow-phase time).  Results do not depend on it."""
        self._check(self.lib.vxp_set_traffic_accounting(self.ctx, 1 if on else 0))

    def set_cluster_constraints(self, on: bool = True) -> None:
        """Solver mode 2: the cluster also builds and colours the constraint
        table, or (default) the grid does that first.  Same results."""
        self._check(self.lib.vxp_set_cluster_constraints(self.ctx, 1 if on else 0))

    def set_cluster_shared_bytes(self, n: int) -> None:
        """Shared memory per CTA the cluster sweeps may keep their state in
        (0: always L2).  Results do not depend on it."""
        self._check(self.lib.vxp_set_cluster_shared_bytes(self.ctx, int(n)))

    def cluster_size(self) -> int:
        """CTAs of the cluster that solver mode 2 runs on (0: not available)."""
        n = ctypes.c_uint32(0)
        self._check(self.lib.vxp_cluster_size(self.ctx, ctypes.byref(n)))
        return int(n.value)

    def set_heavy_pair_voxels(self, n: int) -> None:
        """Pairs with at least n overlap-region voxels are probed by a whole CTA (0: never)."""
        self._check(self.lib.vxp_set_heavy_pair_voxels(self.ctx, int(n)))

    def set_wait_limit_ns(self, ns: int) -> None:
        """Grid-barrier wait limit of grid-launched steps (0: the default, 10 s);
        a step that waits longer fails with VXP_ERR_TIMEOUT."""
        self._check(self.lib.vxp_set_wait_limit_ns(self.ctx, int(ns)))

    def set_probe_tables(self, on: bool = True) -> None:
        """Neighbourhood-mask tables for the narrow phase's probes (on by default)."""
        self._check(self.lib.vxp_set_probe_tables(self.ctx, 1 if on else 0))

    def set_substep_record(self, on: bool = True) -> None:
        self._check(self.lib.vxp_snapshot_substeps(self.ctx, 1 if on else 0))

    def substeps(self) -> np.ndarray:
        """Body states after each substep of the last step: (substeps, bodies, 13)
        float32 (position, rotation, linear velocity, angular velocity)."""
        n = len(self.get_bodies())
        cap = max(1, int(self.config.substeps)) * n * 13
        out = np.zeros(cap, dtype=np.float32)
        ns = ctypes.c_uint32(0)
        self._check(self.lib.vxp_substeps_get(self.ctx, abi.ptr(out), cap, ctypes.byref(ns)))
        return out[: ns.value * n * 13].reshape(ns.value, n, 13)

    def pairs(self, margin: float | None = None) -> np.ndarray:
        m = self.pair_margin if margin is None else margin
        n = ctypes.c_uint32(0)
        rc = self.lib.vxp_pairs_from_bodies(self.ctx, np.float32(m), None, 0, ctypes.byref(n))
        if rc not in (0, abi.VXP_ERR_CAP):
            self._check(rc)
        out = np.zeros(n.value, dtype=abi.PAIR_DTYPE)
        self._check(self.lib.vxp_pairs_from_bodies(self.ctx, np.float32(m), abi.ptr(out), len(out), ctypes.byref(n)))
        return out

    def manifolds(self) -> np.ndarray:
        n = ctypes.c_uint32(0)
        self._check(self.lib.vxp_manifolds_get(self.ctx, None, 0, ctypes.byref(n)))
        out = np.zeros(n.value, dtype=abi.MANIFOLD_DTYPE)
        self._check(self.lib.vxp_manifolds_get(self.ctx, abi.ptr(out), len(out), ctypes.byref(n)))
        return out

    def stats(self) -> dict:
        s = abi.Stats()
        self._check(self.lib.vxp_stats_get(self.ctx, ctypes.byref(s)))
        return s.as_dict()

    def colours(self) -> np.ndarray:
        n = ctypes.c_uint32(0)
        self._check(self.lib.vxp_colours_get(self.ctx, None, 0, ctypes.byref(n)))
        out = np.zeros(n.value, dtype=np.uint32)
        self._check(self.lib.vxp_colours_get(self.ctx, abi.ptr(out), len(out), ctypes.byref(n)))
        return out

    def set_candidate_dump(self, capacity: int) -> None:
        self._check(self.lib.vxp_set_candidate_dump(self.ctx, int(capacity)))

    def candidates(self) -> np.ndarray:
        n = ctypes.c_uint32(0)
        rc = self.lib.vxp_candidates_get(self.ctx, None, 0, ctypes.byref(n))
        if rc not in (0, abi.VXP_ERR_CAP):
            self._check(rc)
        out = np.zeros(n.value, dtype=abi.CANDIDATE_DTYPE)
        self._check(self.lib.vxp_candidates_get(self.ctx, abi.ptr(out), len(out), ctypes.byref(n)))
        return out[: n.value]

    def last_step_ms(self) -> float:
        out = np.zeros(3, dtype=np.float32)
        self._check(self.lib.vxp_last_step_ms(self.ctx, abi.ptr(out)))
        return float(out[2])


class VoxelWorldBatch:
    """Many independent worlds stepped together (one CTA per world, one
    launch per step replayed from a CUDA graph).  Each world's results equal
    VoxelPhysicsSystem.step(dt) on that world alone."""

    def __init__(self, max_worlds: int, config: abi.Config | None = None, device: int = 0, **overrides):
        self.lib = abi.load()
        self.config = config if config is not None else abi.default_config(**overrides)
        h = ctypes.c_void_p()
        rc = self.lib.vxp_batch_create(ctypes.byref(self.config), device, int(max_worlds), ctypes.byref(h))
        if rc != 0 or not h.value:
            raise VxpError(rc, "vxp_batch_create failed")
        self.b = h
        self.max_worlds = int(max_worlds)
        self.sizes = {}

    def _check(self, rc: int) -> None:
        if rc != 0:
            buf = ctypes.create_string_buffer(512)
            self.lib.vxp_batch_last_error(self.b, buf, len(buf))
            raise VxpError(rc, buf.value.decode(errors="replace"))

    def close(self) -> None:
        if getattr(self, "b", None) is not None and self.b.value:
            self.lib.vxp_batch_destroy(self.b)
            self.b = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_collider(self, collider_id: int, voxel_size: float, bricks: np.ndarray) -> None:
        bricks = np.ascontiguousarray(bricks, dtype=abi.BRICK_DTYPE)
        self._check(self.lib.vxp_batch_collider_upload(self.b, int(collider_id), np.float32(voxel_size),
                                                       abi.ptr(bricks), len(bricks)))

    def edit_collider(self, collider_id: int, coords, values, mode="occupancy") -> None:
        """VoxelPhysicsSystem.edit_collider on the batch's shared colliders:
        every world whose bodies use the collider sees the edit."""
        coords, values, mode = _edit_args(coords, values, mode)
        self._check(self.lib.vxp_batch_collider_edit(self.b, int(collider_id), abi.ptr(coords), abi.ptr(values),
                                                     len(values), mode))

    def read_collider(self, collider_id: int):
        rc, info, bricks = _read_collider(self.lib.vxp_batch_collider_read, self.b, collider_id)
        self._check(rc)
        return info, bricks

    def invalidate_cache_for_body(self, world: int, body_id: int) -> int:
        n = ctypes.c_uint32(0)
        self._check(self.lib.vxp_batch_invalidate_cache_for_body(self.b, int(world), int(body_id), ctypes.byref(n)))
        return int(n.value)

    def set_world(self, world: int, bodies: np.ndarray, pair_capacity: int = 0) -> None:
        bodies = np.ascontiguousarray(bodies, dtype=abi.BODY_DTYPE)
        self._check(self.lib.vxp_batch_world_set(self.b, int(world), abi.ptr(bodies), len(bodies), int(pair_capacity)))
        self.sizes[int(world)] = len(bodies)

    def load_scene(self, world: int, scene, collider_offset: int) -> None:
        """Uploads the scene's colliders under ids offset + id and fills the slot."""
        for c in scene.colliders:
            self.add_collider(collider_offset + c.id, c.voxel_size, c.bricks)
        bodies = scene.bodies.copy()
        bodies["collider_id"] = bodies["collider_id"] + collider_offset
        self.set_world(world, bodies)

    def clear_world(self, world: int) -> None:
        """Empties the slot; its device memory stays for the next world set there."""
        self._check(self.lib.vxp_batch_world_clear(self.b, int(world)))
        self.sizes.pop(int(world), None)

    def release_world(self, world: int) -> None:
        """Empties the slot and frees its device memory."""
        self._check(self.lib.vxp_batch_world_release(self.b, int(world)))
        self.sizes.pop(int(world), None)

    def get_world(self, world: int) -> np.ndarray:
        out = np.zeros(self.sizes[int(world)], dtype=abi.BODY_DTYPE)
        self._check(self.lib.vxp_batch_world_get(self.b, int(world), abi.ptr(out), len(out)))
        return out

    def export_world(self, world: int, fields=None, first: int = 0, n: int | None = None) -> dict:
        """export_state for one world of the batch (vxp_batch_world_export)."""
        n = self.sizes[int(world)] - first if n is None else n
        out, view = _export_arrays(fields, n)
        self._check(self.lib.vxp_batch_world_export(self.b, int(world), ctypes.byref(view), int(first), int(n), 0,
                                                    None))
        return out

    def world_stats(self, world: int) -> dict:
        s = abi.Stats()
        self._check(self.lib.vxp_batch_world_stats(self.b, int(world), ctypes.byref(s)))
        return s.as_dict()

    def world_bytes(self, world: int) -> int:
        return int(self.lib.vxp_batch_world_bytes(self.b, int(world)))

    def step(self, dt: float, n_steps: int = 1) -> None:
        self._check(self.lib.vxp_batch_step(self.b, np.float32(dt), int(n_steps)))

    def synchronize(self) -> None:
        self._check(self.lib.vxp_batch_synchronize(self.b))

    def times(self) -> tuple:
        total = ctypes.c_float(0)
        per = np.zeros(self.max_worlds, dtype=np.float32)
        self._check(self.lib.vxp_batch_times(self.b, ctypes.byref(total), abi.ptr(per), self.max_worlds))
        return float(total.value), per

    def set_schedule(self, threads: int, order_mode: int) -> None:
        """One CTA size (256 or 512) for every world; order 0 slot order, 1 longest first."""
        self._check(self.lib.vxp_batch_set_schedule(self.b, int(threads), int(order_mode)))

    def set_tiles(self, min_bodies_512: int, order_mode: int = 1) -> None:
        """Per-world tiles: worlds of at least min_bodies_512 bodies as 512-thread
        CTAs, the rest as 256-thread CTAs, the two launches side by side."""
        self._check(self.lib.vxp_batch_set_tiles(self.b, int(min_bodies_512), int(order_mode)))

    @staticmethod
    def schedule_name(choice: int) -> str:
        """The autotuner's schedule index as text."""
        if choice < 4:
            return f"{256 if choice < 2 else 512}/{'longest-first' if choice & 1 else 'slot-order'}"
        return f"tiles: >= {128 << (choice - 4)} bodies 512, else 256/longest-first"

    def autotune(self, dt: float, trial_steps: int = 3) -> tuple:
        ms = np.zeros(abi.BATCH_SCHEDULES, dtype=np.float32)
        choice = ctypes.c_uint32(0)
        self._check(self.lib.vxp_batch_autotune(self.b, np.float32(dt), int(trial_steps), abi.ptr(ms),
                                                ctypes.byref(choice)))
        return int(choice.value), ms


def _export_arrays(fields, n: int):
    """Host arrays for an export of n bodies and the state view over them."""
    names = list(abi.EXPORT_FIELDS) if fields is None else list(fields)
    out, view = {}, abi.StateView()
    for name in names:
        k, dt = abi.EXPORT_FIELDS[name]
        a = np.zeros((n, k) if k > 1 else n, dtype=dt)
        out[name] = a
        setattr(view, name, a.ctypes.data if a.size else None)
    return out, view


def _device_view(pointers: dict):
    view = abi.StateView()
    for name, addr in pointers.items():
        if name not in abi.EXPORT_FIELDS:
            raise KeyError(f"unknown export field {name!r}")
        setattr(view, name, int(addr) or None)
    return view
