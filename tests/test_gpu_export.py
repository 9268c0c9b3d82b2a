"""Bulk state export (vxp_bodies_export, vxp_batch_world_export): the
per-handle getters of the reference (getPosition, getRotation,
getLinearVelocity, getAngularVelocity, getWorldAABB, isSleeping;
src/system.zig:963-1017) for a range of bodies in one call, into host arrays
or into device memory that a CUDA consumer reads on its own stream."""
import ctypes

import numpy as np
import pytest

import oracle_api as O

pytestmark = pytest.mark.gpu


def _stepped(vxp, steps=40):
    sc = vxp.scenes.config1(mass_fn=O.mass_fn, n_side=3, seed=4)
    g = vxp.VoxelPhysicsSystem()
    g.load_scene(sc)
    r = O.OracleWorld()
    r.load_scene(sc)
    dt = np.float32(sc.dt)
    for _ in range(steps):
        p = r.pairs()
        g.step(dt, p)
        r.step(dt, p)
    assert g.get_bodies().tobytes() == r.get_bodies().tobytes()
    return g, r


def test_export_matches_bodies_and_oracle_aabbs(vxp):
    g, r = _stepped(vxp)
    b = g.get_bodies()
    e = g.export_state()
    assert e["position"].tobytes() == np.ascontiguousarray(b["position"]).tobytes()
    assert e["rotation"].tobytes() == np.ascontiguousarray(b["rotation"]).tobytes()
    assert e["linear_velocity"].tobytes() == np.ascontiguousarray(b["linear_velocity"]).tobytes()
    assert e["angular_velocity"].tobytes() == np.ascontiguousarray(b["angular_velocity"]).tobytes()
    assert (e["sleeping"] == b["is_sleeping"]).all()
    mn, mx = r.world_aabbs()
    assert e["aabb_min"].tobytes() == mn.tobytes()
    assert e["aabb_max"].tobytes() == mx.tobytes()
    # a range, some fields only
    part = g.export_state(fields=("rotation", "aabb_max"), first=5, n=7)
    assert set(part) == {"rotation", "aabb_max"}
    assert part["rotation"].tobytes() == e["rotation"][5:12].tobytes()
    assert part["aabb_max"].tobytes() == mx[5:12].tobytes()
    g.close()
    r.close()


def test_export_into_device_memory_for_a_consumer_stream(vxp):
    import torch

    g, r = _stepped(vxp, steps=25)
    n = g.n_bodies
    dev = {"position": torch.full((n, 3), -1.0, device="cuda:0"), "aabb_min": torch.full((n, 3), -1.0, device="cuda:0"),
           "sleeping": torch.full((n,), 7, dtype=torch.uint8, device="cuda:0")}
    s = torch.cuda.Stream(device="cuda:0")
    g.export_state_to_device({k: v.data_ptr() for k, v in dev.items()}, consumer_stream=s.cuda_stream)
    with torch.cuda.stream(s):
        got = {k: v.clone() for k, v in dev.items()}  # the consumer, ordered after the export
    s.synchronize()
    want = g.export_state(fields=("position", "aabb_min", "sleeping"))
    for k in got:
        assert got[k].cpu().numpy().tobytes() == want[k].tobytes(), k
    g.close()
    r.close()


def test_export_rejects_bad_arguments(vxp):
    g, r = _stepped(vxp, steps=2)
    n = g.n_bodies
    host = np.zeros((n, 3), dtype=np.float32)
    view = vxp.abi.StateView()
    view.position = host.ctypes.data
    # host memory passed as device memory: rejected before any launch
    assert g.lib.vxp_bodies_export(g.ctx, ctypes.byref(view), 0, n, 1, None) == vxp.abi.VXP_ERR_ARG
    # a range past the bodies
    assert g.lib.vxp_bodies_export(g.ctx, ctypes.byref(view), 1, n, 0, None) == vxp.abi.VXP_ERR_ARG
    assert g.lib.vxp_bodies_export(g.ctx, None, 0, n, 0, None) == vxp.abi.VXP_ERR_ARG
    # the context is still usable
    assert g.export_state(fields=("position",))["position"].shape == (n, 3)
    g.close()
    r.close()


def test_batch_world_export(vxp):
    sc = [vxp.scenes.config1(mass_fn=O.mass_fn, n_side=2, seed=s) for s in (1, 2)]
    bt = vxp.VoxelWorldBatch(2)
    for w, scene in enumerate(sc):
        bt.load_scene(w, scene, collider_offset=1000 * w)
    bt.step(np.float32(sc[0].dt), 20)
    for w in range(2):
        b = bt.get_world(w)
        e = bt.export_world(w, fields=("position", "angular_velocity", "sleeping"))
        assert e["position"].tobytes() == np.ascontiguousarray(b["position"]).tobytes()
        assert e["angular_velocity"].tobytes() == np.ascontiguousarray(b["angular_velocity"]).tobytes()
        assert (e["sleeping"] == b["is_sleeping"]).all()
    bt.close()
