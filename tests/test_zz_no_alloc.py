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


def random_boxes(rng, n):
    """n boxes with identity rotations (their world AABBs are then exact f32
    sums, reproducible in NumPy), ids 1..n, a fifth of them static."""
    pos = np.zeros((n, 4), dtype=np.float32)
    pos[:, :3] = rng.uniform([-20, 0, -20], [20, 10, 20], size=(n, 3)).astype(np.float32)
    rot = np.tile(np.array([0, 0, 0, 1], dtype=np.float32), (n, 1))
    la = np.zeros((n, 8), dtype=np.float32)
    ext = rng.integers(2, 17, size=(n, 3)).astype(np.float32) * np.float32(0.1)
    la[:, 4:7] = ext
    ids = np.arange(1, n + 1, dtype=np.uint32)
    types = np.where(rng.random(n) < 0.2, 0, 2).astype(np.uint32)
    return pos, rot, la, ids, types


def brute_force_pairs(pos, la, ids, types, margin):
    """Every (a, b), a < b, whose margin-inflated world AABBs overlap (<= on
    both sides), static-static excluded, in row order."""
    m = np.float32(margin)
    lo = (pos[:, :3] + la[:, :3]) - m
    hi = (pos[:, :3] + la[:, 4:7]) + m
    n = len(ids)
    out = []
    for r0 in range(0, n, 256):
        r1 = min(n, r0 + 256)
        ov = np.all((lo[r0:r1, None, :] <= hi[None, :, :]) & (hi[r0:r1, None, :] >= lo[None, :, :]), axis=2)
        ov &= np.arange(n)[None, :] > np.arange(r0, r1)[:, None]
        ov &= ~((types[r0:r1, None] == 0) & (types[None, :] == 0))
        i, j = np.nonzero(ov)
        out.append(np.stack([ids[r0 + i], ids[j]], axis=1))
    return np.concatenate(out).astype(np.uint32)


def test_noalloc_on_a_stream_near_the_body_cap(vxp):
    """16000 boxes (near the 16384 cap, where the row sweep has n*32 threads
    and the one-CTA scan its longest loop), queued on a non-default stream,
    twice: the pairs equal a NumPy brute force."""
    torch = pytest.importorskip("torch")
    lib = vxp.abi.load()
    rng = np.random.default_rng(31)
    n = 16000
    pos, rot, la, ids, types = random_boxes(rng, n)
    want = brute_force_pairs(pos, la, ids, types, 0.1)
    assert 10000 < len(want)
    cap = len(want) + 64
    dev = [torch.from_numpy(a.view(np.int32) if a.dtype == np.uint32 else a).cuda() for a in (pos, rot, la, ids, types)]
    stream = torch.cuda.Stream()
    torch.cuda.synchronize()
    for call in range(2):
        with torch.cuda.stream(stream):
            out = torch.zeros(cap * 2, dtype=torch.int32, device="cuda")
            count = torch.zeros(1, dtype=torch.int32, device="cuda")
        stream.synchronize()
        rc = lib.vxp_pairs_noalloc(*(t.data_ptr() for t in dev), n, np.float32(0.1), out.data_ptr(), cap,
                                   count.data_ptr(), ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0
        stream.synchronize()
        k = int(count.item())
        got = out.cpu().numpy().view(np.uint32).reshape(-1, 2)[:k]
        assert k == len(want), f"call {call}: {k} vs {len(want)}"
        assert np.array_equal(got, want), f"call {call}: pair lists differ"


def test_noalloc_unordered_ids_write_nothing(vxp):
    """Ids that are not strictly ascending break the call's precondition: the
    total is 0 and no pair is written (the buffer keeps its fill).  With
    VXP_CHECK_ARGS=1 (a fresh process) the call returns VXP_ERR_ARG."""
    torch = pytest.importorskip("torch")
    lib = vxp.abi.load()
    rng = np.random.default_rng(32)
    n = 300
    pos, rot, la, ids, types = random_boxes(rng, n)
    ids[[10, 11]] = ids[[11, 10]]
    dev = [torch.from_numpy(a.view(np.int32) if a.dtype == np.uint32 else a).cuda() for a in (pos, rot, la, ids, types)]
    out = torch.full((64 * 2,), -1, dtype=torch.int32, device="cuda")
    count = torch.full((1,), 7, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    rc = lib.vxp_pairs_noalloc(*(t.data_ptr() for t in dev), n, np.float32(0.1), out.data_ptr(), 64,
                               count.data_ptr(), None)
    assert rc == 0
    torch.cuda.synchronize()
    assert int(count.item()) == 0
    assert bool((out == -1).all().item())

    import os
    import subprocess
    import sys
    code = (
        "import importlib, sys, ctypes, numpy as np, torch\n"
        f"sys.path.insert(0, {os.path.dirname(os.path.abspath(__file__))!r})\n"
        "import conftest, test_zz_no_alloc as T\n"
        "vxp = conftest.load_package(); lib = vxp.abi.load()\n"
        "pos, rot, la, ids, types = T.random_boxes(np.random.default_rng(32), 300)\n"
        "ids[[10, 11]] = ids[[11, 10]]\n"
        "dev = [torch.from_numpy(a.view(np.int32) if a.dtype == np.uint32 else a).cuda() for a in (pos, rot, la, ids, types)]\n"
        "out = torch.zeros(128, dtype=torch.int32, device='cuda'); cnt = torch.zeros(1, dtype=torch.int32, device='cuda')\n"
        "torch.cuda.synchronize()\n"
        "print(lib.vxp_pairs_noalloc(*(t.data_ptr() for t in dev), 300, np.float32(0.1), out.data_ptr(), 64, cnt.data_ptr(), None))\n"
    )
    env = dict(os.environ, VXP_CHECK_ARGS="1")
    res = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stderr[-2000:]
    assert res.stdout.strip().splitlines()[-1] == str(vxp.abi.VXP_ERR_ARG)
