"""The allocation-free pair source against the context-owned one.

vxp_pairs_noalloc serves callers that cannot let the library allocate
device memory (a frame thread where cudaMalloc's implicit synchronisation is
not allowed, or an engine that hands out all device memory itself).  It is
called through the C ABI on device buffers the test owns, twice in a row
(the shared static scratch keeps the first call's contents), and each
result must equal vxp_pairs_from_bodies for the same bodies: pair lists are
integers, so the tolerance is exact equality.  This file is collected last
so that a failure here cannot hide any other test.
"""
import ctypes

import numpy as np
import pytest

import oracle_api as O

pytestmark = pytest.mark.gpu


def local_aabbs(scene):
    """Per-collider local AABB as VoxelCollider.recomputeMetadata computes it
    (f32: (brick*8 + cell) * vs, max + vs), merged over bricks."""
    out = {}
    for c in scene.colliders:
        vs = np.float32(c.voxel_size)
        lo = np.full(3, np.inf, dtype=np.float32)
        hi = np.full(3, -np.inf, dtype=np.float32)
        for b in c.bricks:
            idx = np.flatnonzero(b["voxels"] & 7)
            if len(idx) == 0:
                continue
            cell = np.stack([idx % 8, (idx // 8) % 8, idx // 64], axis=1)
            p = (b["pos"][None, :].astype(np.float32) * np.float32(8) + cell.astype(np.float32)) * vs
            lo = np.minimum(lo, p.min(axis=0))
            hi = np.maximum(hi, (p + vs).max(axis=0))
        out[c.id] = (lo, hi)
    return out


def device_inputs(torch, scene, bodies):
    ab = local_aabbs(scene)
    n = len(bodies)
    pos = np.zeros((n, 4), dtype=np.float32)
    pos[:, :3] = bodies["position"]
    rot = np.ascontiguousarray(bodies["rotation"], dtype=np.float32)
    la = np.zeros((n, 8), dtype=np.float32)
    for i, b in enumerate(bodies):
        lo, hi = ab.get(int(b["collider_id"]), (np.ones(3, np.float32), np.zeros(3, np.float32)))
        la[i, :3], la[i, 4:7] = lo, hi
    order = np.argsort(bodies["id"], kind="stable")
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a[order])).cuda()
    return (dev(pos), dev(rot), dev(la), dev(bodies["id"].astype(np.int32)), dev(bodies["body_type"].astype(np.int32)))


def call_noalloc(vxp, torch, ins, n, margin, cap):
    lib = vxp.abi.load()
    out = torch.zeros(cap * 2, dtype=torch.int32, device="cuda")
    count = torch.zeros(1, dtype=torch.int32, device="cuda")
    pos, rot, la, ids, types = ins
    torch.cuda.synchronize()
    rc = lib.vxp_pairs_noalloc(pos.data_ptr(), rot.data_ptr(), la.data_ptr(), ids.data_ptr(), types.data_ptr(), n,
                               np.float32(margin), out.data_ptr(), cap, count.data_ptr(), None)
    assert rc == 0
    torch.cuda.synchronize()
    k = int(count.item())
    got = out.cpu().numpy().view(np.uint32).reshape(-1, 2)[: min(k, cap)]
    res = np.zeros(len(got), dtype=vxp.abi.PAIR_DTYPE)
    res["body_a"], res["body_b"] = got[:, 0], got[:, 1]
    return k, res


@pytest.mark.parametrize("which", ["config1", "config2"])
def test_noalloc_pairs_match_context_pairs_twice(vxp, which):
    torch = pytest.importorskip("torch")
    if which == "config1":
        scene = vxp.scenes.config1(mass_fn=O.mass_fn, seed=21)
    else:
        scene = vxp.scenes.config2(mass_fn=O.mass_fn, n_side=6, seed=22)
    sysm = vxp.VoxelPhysicsSystem(substeps=int(scene.config["substeps"]))
    sysm.load_scene(scene)
    dt = np.float32(scene.dt)
    margin = np.float32(0.1)
    for call in range(2):
        want = sysm.pairs(margin)
        bodies = sysm.get_bodies()
        ins = device_inputs(torch, scene, bodies)
        k, got = call_noalloc(vxp, torch, ins, len(bodies), margin, cap=max(16, 2 * len(want)))
        assert k == len(want), f"call {call}: {k} pairs vs {len(want)}"
        assert got.tobytes() == want.tobytes(), f"call {call}: pair lists differ"
        for _ in range(30):  # move the bodies before the second call
            sysm.step(dt)
    sysm.close()


def test_noalloc_rejects_too_many_bodies(vxp):
    lib = vxp.abi.load()
    c = ctypes.c_void_p(0)
    assert lib.vxp_pairs_noalloc(c, c, c, c, c, 16385, np.float32(0.1), c, 0, c, None) == vxp.abi.VXP_ERR_CAP


def test_noalloc_truncates_at_cap(vxp):
    torch = pytest.importorskip("torch")
    scene = vxp.scenes.config1(mass_fn=O.mass_fn, seed=23)
    sysm = vxp.VoxelPhysicsSystem()
    sysm.load_scene(scene)
    want = sysm.pairs(np.float32(0.1))
    ins = device_inputs(torch, scene, sysm.get_bodies())
    k, got = call_noalloc(vxp, torch, ins, len(scene.bodies), 0.1, cap=5)
    assert k == len(want) and len(got) == 5
    assert got.tobytes() == want[:5].tobytes()
    sysm.close()
