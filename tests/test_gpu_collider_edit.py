"""Collider edits on the device (vxp_collider_edit), bit for bit with the
oracle's composition of the reference calls (setCollisionVoxel,
classifyFromNeighbors, recomputeMetadata; pinned against a Python
restatement in test_collider_edit_cpu.py):

* edit batches in both modes on a classified block, a brick reached through
  a shared brick hash and a 512 x 512 slab: voxels, brick order and metadata
  equal after every batch, with and without neighbourhood-mask tables;
* a pile that lands on a bin floor, a hole carved in the floor between two
  steps (queued behind the step on the stream), the bin's brick-pair cache
  entries invalidated: bodies, manifolds and counters equal the oracle's
  every step after the edit, for the block and the grid launch;
* a batch of two worlds where one world's ground gets a hole: each world
  equals its oracle;
* re-uploads that leave dead pool ranges until the store reclaims them, and
  edits that place a collider again with new bricks: every collider still
  equals the oracle's.
"""
import numpy as np
import pytest

import oracle_api as O
from test_collider_edit_cpu import _bricks_of, _classified_block, _random_edits, hash_brick
from test_gpu_parity import STAT_KEYS, _first_diff

pytestmark = pytest.mark.gpu

INFO_KEYS = ("voxel_size", "min_bound", "max_bound", "aabb_min", "aabb_max", "solid_count", "n_bricks")


def _same_collider(g, r, cid):
    gi, gb = g.read_collider(cid)
    ri, rb = r.read_collider(cid)
    assert len(gb) == len(rb), f"collider {cid}: {len(gb)} bricks vs {len(rb)}"
    assert gb["pos"].tobytes() == rb["pos"].tobytes(), f"collider {cid}: brick order differs"
    assert gb.tobytes() == rb.tobytes(), f"collider {cid}: voxels differ in {_first_diff(gb, rb)}"
    for k in INFO_KEYS:
        assert np.asarray(gi[k]).tobytes() == np.asarray(ri[k]).tobytes(), f"collider {cid}: {k} {gi[k]} vs {ri[k]}"
    return gi


def _both(vxp, tables=True, **cfg):
    g = vxp.VoxelPhysicsSystem(**cfg)
    g.set_probe_tables(tables)
    return g, O.OracleWorld(**cfg)


def _edit_both(g, r, cid, coords, values, mode):
    g.edit_collider(cid, coords, values, mode)
    r.edit_collider(cid, coords, values, mode)


@pytest.mark.parametrize("tables", [True, False])
def test_edit_batches_equal_the_oracle(vxp, tables):
    rng = np.random.default_rng(11)
    g, r = _both(vxp, tables)
    block = _bricks_of(_classified_block((0, 0, 0), (20, 12, 18)))
    alias = _bricks_of(_classified_block((-16, 0, 24), (-8, 4, 32)))  # brick (-2,0,3)
    assert hash_brick((0, 0, -3)) == hash_brick((-2, 0, 3))
    for cid, bricks in ((3, block), (2, alias)):
        g.add_collider(cid, 0.1, bricks)
        r.add_collider(cid, 0.1, bricks)
    _same_collider(g, r, 3)
    # carving only: the bounds shrink or stay, the table stays
    carve = _random_edits(rng, 500, 0, 20)
    _edit_both(g, r, 3, carve, np.zeros(len(carve), np.uint8), "occupancy")
    info = _same_collider(g, r, 3)
    assert info["has_table"] == (1 if tables else 0)
    for it in range(5):
        coords = _random_edits(rng, 400, -6, 26)  # past the held bricks: new bricks
        values = rng.integers(0, 2, size=len(coords)).astype(np.uint8)
        _edit_both(g, r, 3, coords, values, "occupancy")
        _same_collider(g, r, 3)
        coords = _random_edits(rng, 100, -6, 26)
        values = rng.integers(0, 256, size=len(coords)).astype(np.uint8)
        _edit_both(g, r, 3, coords, values, "set")
        _same_collider(g, r, 3)
    # writes through the shared hash into the held brick (-2,0,3)
    coords = np.array([[3, 1, -20], [4, 1, -20], [3, 2, -22], [-13, 2, 27]], np.int32)
    _edit_both(g, r, 2, coords, np.array([1, 1, 0, 0], np.uint8), "occupancy")
    _same_collider(g, r, 2)
    _edit_both(g, r, 2, coords, np.array([0x1B, 0x0C, 4, 0], np.uint8), "set")
    _same_collider(g, r, 2)
    g.close()
    r.close()


def test_large_slab_edit(vxp):
    """A 512 x 1 x 512 slab (4096 bricks): a disc of ~50k voxels carved, then a
    ring filled back; many CTAs share the metadata pass."""
    sc = vxp.scenes
    g, r = _both(vxp)
    slab = sc.ground_slab(512, 512)
    g.add_collider(1, 0.1, slab)
    r.add_collider(1, 0.1, slab)
    x, z = np.meshgrid(np.arange(512), np.arange(512), indexing="ij")
    d2 = (x - 200) ** 2 + (z - 300) ** 2
    disc = np.stack([x[d2 < 126 ** 2], np.zeros(int((d2 < 126 ** 2).sum()), int), z[d2 < 126 ** 2]], 1)
    _edit_both(g, r, 1, disc, np.zeros(len(disc), np.uint8), "occupancy")
    info = _same_collider(g, r, 1)
    assert info["solid_count"] == 512 * 512 - len(disc)
    ring = (d2 >= 60 ** 2) & (d2 < 70 ** 2)
    fill = np.stack([x[ring], np.zeros(int(ring.sum()), int), z[ring]], 1)
    _edit_both(g, r, 1, fill, np.ones(len(fill), np.uint8), "occupancy")
    _same_collider(g, r, 1)
    g.close()
    r.close()


def _lockstep(g, r, dt, n, check_every=1):
    for s in range(n):
        pairs = r.pairs()
        g.step(dt, pairs)
        r.step(dt, pairs)
        if s % check_every == 0 or s == n - 1:
            gb, rb = g.get_bodies(), r.get_bodies()
            assert gb.tobytes() == rb.tobytes(), f"step {s}: bodies differ in {_first_diff(gb, rb)}"
            gm, rm = g.manifolds(), r.manifolds()
            assert gm.tobytes() == rm.tobytes(), f"step {s}: manifolds differ in {_first_diff(gm, rm)}"
            gs, rs = g.stats(), r.stats()
            for k in STAT_KEYS:
                assert gs[k] == rs[k], f"step {s}: stats[{k}] gpu {gs[k]} oracle {rs[k]}"


@pytest.mark.parametrize("launch", [0, 1])
def test_pile_falls_through_a_carved_floor(vxp, launch):
    """27 boxes land on the bin floor (2 voxels thick, top at 0.2 m) and come
    to rest; a hole of 48 x 48 voxels is carved under the middle column
    between two steps; the bin's cache entries are dropped on both sides (the
    same count); the lowest box of the middle column (body row 6) drops onto
    the ground slab below."""
    sc = vxp.scenes.config2(mass_fn=O.mass_fn, n_side=3, seed=21)
    cfg = dict(substeps=8)
    dt = np.float32(sc.dt)
    g, r = _both(vxp, **cfg)
    g.set_launch_mode(launch)
    g.load_scene(sc)
    r.load_scene(sc)
    _lockstep(g, r, dt, 200, check_every=20)
    before = r.get_bodies()
    xs, zs = np.meshgrid(np.arange(40, 88), np.arange(40, 88), indexing="ij")
    hole = np.concatenate([np.stack([xs.ravel(), np.full(xs.size, y), zs.ravel()], 1) for y in (0, 1)])
    g.edit_collider(0, hole, np.zeros(len(hole), np.uint8), "occupancy")  # queued behind the last step
    r.edit_collider(0, hole, np.zeros(len(hole), np.uint8), "occupancy")
    n_g, n_r = g.invalidate_cache_for_body(1), r.invalidate_cache_for_body(1)
    assert n_g == n_r and n_r > 0, (n_g, n_r)
    _same_collider(g, r, 0)
    _lockstep(g, r, dt, 60)
    after = r.get_bodies()
    assert before["position"][6, 1] - after["position"][6, 1] > 0.1
    g.close()
    r.close()


def test_batch_world_with_a_carved_ground(vxp):
    rng = np.random.default_rng(31)
    scenes = [vxp.scenes.world_for_batch(rng, 27, O.mass_fn, name=f"w{i}") for i in range(2)]
    dt = np.float32(1.0 / 60.0)
    b = vxp.VoxelWorldBatch(2, substeps=4)
    off = [0, len(scenes[0].colliders) + 1]
    for i, s in enumerate(scenes):
        b.load_scene(i, s, collider_offset=off[i])
    rs = []
    for s in scenes:
        r = O.OracleWorld(substeps=4)
        r.load_scene(s)
        rs.append(r)
    b.step(dt, 80)
    for r in rs:
        for _ in range(80):
            r.step(dt)
    xs, zs = np.meshgrid(np.arange(20, 44), np.arange(20, 44), indexing="ij")
    hole = np.stack([xs.ravel(), np.zeros(xs.size, int), zs.ravel()], 1)
    b.edit_collider(off[0] + 0, hole, np.zeros(len(hole), np.uint8), "occupancy")
    rs[0].edit_collider(0, hole, np.zeros(len(hole), np.uint8), "occupancy")
    assert b.invalidate_cache_for_body(0, 1) == rs[0].invalidate_cache_for_body(1)
    b.step(dt, 40)
    b.synchronize()
    for i, r in enumerate(rs):
        for _ in range(40):
            r.step(dt)
        got = b.get_world(i)
        got["collider_id"] -= off[i]
        want = r.get_bodies()
        assert got.tobytes() == want.tobytes(), f"world {i} differs in {_first_diff(got, want)}"
        r.close()
    gi, _ = b.read_collider(off[1])
    assert gi["solid_count"] == 64 * 64  # the other world's ground is whole
    b.close()


def test_reuploads_and_replacements_reclaim_dead_ranges(vxp):
    rng = np.random.default_rng(41)
    g, r = _both(vxp)
    keep = _bricks_of(_classified_block((0, 0, 0), (24, 9, 17)))
    g.add_collider(1, 0.1, keep)
    r.add_collider(1, 0.1, keep)
    for k in range(72):  # 64-brick colliders replaced: the dead bricks outgrow the live ones
        blk = _bricks_of(_classified_block((0, 0, 0), (32, 32, 17 + k % 15)))
        g.add_collider(7, 0.1, blk)
        if k % 9 == 0 or k == 71:
            r.add_collider(7, 0.1, blk)
            for cid in (1, 7):
                _same_collider(g, r, cid)
    # an edit that needs new bricks places collider 1 again
    coords = _random_edits(rng, 300, -10, 34)
    _edit_both(g, r, 1, coords, rng.integers(0, 2, size=len(coords)).astype(np.uint8), "occupancy")
    for cid in (1, 7):
        _same_collider(g, r, cid)
    g.close()
    r.close()
