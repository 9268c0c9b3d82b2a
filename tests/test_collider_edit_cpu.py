"""Collider edits (vxp_collider_edit) in the oracle, pinned against a plain
Python restatement of the reference calls they compose:

* VoxelCollider.setCollisionVoxel / getOrCreateBrick / getCollisionVoxel
  (src/collider.zig:232-273): bricks keyed by hashBrickPos alone, a new
  zeroed brick appended when the hash is new, so a voxel whose brick position
  shares a hash with a held brick is written into that brick;
* classifyFromNeighbors / classifyVoxel / computeNormalIndex
  (src/collision_voxel.zig:103-130, 194-235): type by the count of empty
  faces, normal the NORMAL_LUT entry equal to the sum of the empty faces'
  directions, else entry 0;
* recomputeMetadata (src/collider.zig:90-133, 283-333) in float32.

Small colliders only; the device path is compared with the oracle in
test_gpu_collider_edit.py.
"""
import numpy as np

import oracle_api as O
from oracle_api import abi

M64 = (1 << 64) - 1
NORMAL_LUT = [(1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1),
              (1, 1, 0), (1, -1, 0), (-1, 1, 0), (-1, -1, 0), (1, 0, 1), (1, 0, -1), (-1, 0, 1), (-1, 0, -1),
              (0, 1, 1), (0, 1, -1), (0, -1, 1), (0, -1, -1),
              (1, 1, 1), (1, 1, -1), (1, -1, 1), (1, -1, -1), (-1, 1, 1), (-1, 1, -1), (-1, -1, 1), (-1, -1, -1)]
FACES = [(-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0), (0, 0, -1), (0, 0, 1)]


def hash_brick(p):
    x, y, z = (int(v) & M64 for v in p)
    return (x ^ ((y * 0x517cc1b727220a95) & M64) ^ ((z * 0x9e3779b97f4a7c15) & M64)) & M64


class Model:
    """A VoxelCollider as the reference stores it: bricks in creation order."""

    def __init__(self, vs, bricks):
        self.vs = np.float32(vs)
        self.pos = [tuple(int(v) for v in b["pos"]) for b in bricks]
        self.vox = [b["voxels"].copy() for b in bricks]
        self.by_hash = {hash_brick(p): i for i, p in enumerate(self.pos)}

    def _slot(self, v, create):
        bp = tuple(c // 8 for c in v)
        h = hash_brick(bp)
        if h not in self.by_hash:
            if not create:
                return None
            self.by_hash[h] = len(self.pos)
            self.pos.append(bp)
            self.vox.append(np.zeros(512, np.uint8))
        return self.by_hash[h], (v[0] % 8) + 8 * (v[1] % 8) + 64 * (v[2] % 8)

    def get(self, v):
        s = self._slot(v, False)
        return 0 if s is None else int(self.vox[s[0]][s[1]])

    def set(self, v, val):
        b, i = self._slot(v, True)
        self.vox[b][i] = val

    def solid(self, v):
        return (self.get(v) & 7) != 0

    def classify(self, v):
        empty = [not self.solid((v[0] + d[0], v[1] + d[1], v[2] + d[2])) for d in FACES]
        n = sum(empty)
        vtype = 4 if n == 0 else 3 if n == 1 else 2 if n == 2 else 1
        s = tuple(sum(d[k] for d, e in zip(FACES, empty) if e) for k in range(3))
        normal = NORMAL_LUT.index(s) if s in NORMAL_LUT else 0
        return vtype | (normal << 3)

    def edit(self, coords, values, mode):
        for v, val in zip(coords, values):
            v = tuple(int(c) for c in v)
            if mode == "set":
                self.set(v, int(val))
            elif not val:
                self.set(v, 0)
            else:
                self.set(v, self.get(v) if self.solid(v) else 4)
        if mode == "occupancy":
            for v in coords:
                for d in [(0, 0, 0)] + FACES:
                    u = (int(v[0]) + d[0], int(v[1]) + d[1], int(v[2]) + d[2])
                    if self.solid(u):
                        self.set(u, self.classify(u))

    def metadata(self):
        f = np.float32
        inf = f(np.inf)
        mn, mx = [None] * 3, [None] * 3
        amn, amx = [inf] * 3, [-inf] * 3
        solid = 0
        for p, v in zip(self.pos, self.vox):
            idx = np.nonzero(v & 7)[0]
            if len(idx) == 0:
                continue
            solid += len(idx)
            c = np.stack([idx % 8, (idx // 8) % 8, idx // 64], 1)
            for k in range(3):
                vc = p[k] * 8 + c[:, k]
                mn[k] = vc.min() if mn[k] is None else min(mn[k], vc.min())
                mx[k] = vc.max() + 1 if mx[k] is None else max(mx[k], vc.max() + 1)
                lp = (f(p[k]) * f(8.0) + c[:, k].astype(f)) * self.vs
                amn[k] = min(amn[k], lp.min())
                amx[k] = max(amx[k], (lp + self.vs).max())
        if solid == 0:
            mn, mx = [0] * 3, [0] * 3
        return dict(min_bound=mn, max_bound=mx, aabb_min=amn, aabb_max=amx, solid_count=solid)


def _classified_block(lo, hi):
    """Bricks of a solid box of voxels [lo, hi) typed by classifyFromNeighbors."""
    m = Model(0.1, np.zeros(0, abi.BRICK_DTYPE))
    pts = [(x, y, z) for x in range(lo[0], hi[0]) for y in range(lo[1], hi[1]) for z in range(lo[2], hi[2])]
    for p in pts:
        m.set(p, 4)
    for p in pts:
        m.set(p, m.classify(p))
    return m


def _bricks_of(m):
    b = np.zeros(len(m.pos), abi.BRICK_DTYPE)
    for i, (p, v) in enumerate(zip(m.pos, m.vox)):
        b[i]["pos"] = p
        b[i]["voxels"] = v
    return b


def _oracle_with(cid, vs, bricks):
    r = O.OracleWorld()
    r.add_collider(cid, vs, bricks)
    return r


def _assert_same(r, cid, m):
    info, bricks = r.read_collider(cid)
    assert [tuple(p) for p in bricks["pos"]] == m.pos
    for i, v in enumerate(m.vox):
        assert bricks[i]["voxels"].tobytes() == v.tobytes(), f"brick {m.pos[i]}"
    want = m.metadata()
    for k in ("min_bound", "max_bound"):
        assert list(info[k]) == list(want[k]), k
    for k in ("aabb_min", "aabb_max"):
        assert np.asarray(info[k], np.float32).tobytes() == np.asarray(want[k], np.float32).tobytes(), k
    assert info["solid_count"] == want["solid_count"]
    assert info["n_bricks"] == len(m.pos)


def _random_edits(rng, n, lo, hi):
    coords = rng.integers(lo, hi, size=(n, 3)).astype(np.int32)
    coords[n // 2:] = coords[: n - n // 2]  # every other voxel written twice
    rng.shuffle(coords)
    return coords


def test_occupancy_edits_equal_the_reference_calls():
    rng = np.random.default_rng(5)
    m = _classified_block((0, 0, 0), (12, 6, 10))
    bricks = _bricks_of(m)
    r = _oracle_with(3, 0.1, bricks)
    m = Model(0.1, bricks)
    for it in range(6):
        coords = _random_edits(rng, 300, -4, 18)  # reaches past the held bricks
        values = rng.integers(0, 2, size=len(coords)).astype(np.uint8)
        m.edit(coords, values, "occupancy")
        r.edit_collider(3, coords, values, "occupancy")
        _assert_same(r, 3, m)
    assert len(m.pos) > len(bricks)  # edits created bricks
    r.close()


def test_set_edits_equal_the_reference_calls():
    rng = np.random.default_rng(6)
    m = _classified_block((-9, 0, -9), (9, 3, 9))
    bricks = _bricks_of(m)
    r = _oracle_with(1, 0.25, bricks)
    m = Model(0.25, bricks)
    for it in range(4):
        coords = _random_edits(rng, 200, -12, 12)
        values = rng.integers(0, 256, size=len(coords)).astype(np.uint8)
        values[values % 3 == 0] = 0
        m.edit(coords, values, "set")
        r.edit_collider(1, coords, values, "set")
        _assert_same(r, 1, m)
    r.close()


def test_edit_into_a_brick_that_shares_a_hash():
    """(0,0,-3) and (-2,0,3) share hashBrickPos: a voxel written in brick
    (0,0,-3) lands in the held brick (-2,0,3), at the same local coordinate."""
    assert hash_brick((0, 0, -3)) == hash_brick((-2, 0, 3))
    m = _classified_block((-16, 0, 24), (-8, 4, 32))
    bricks = _bricks_of(m)
    assert [tuple(p) for p in bricks["pos"]] == [(-2, 0, 3)]
    r = _oracle_with(2, 0.1, bricks)
    m = Model(0.1, bricks)
    coords = np.array([[3, 5, -20], [4, 5, -20], [3, 1, -22]], np.int32)  # bricks (0,0,-3)
    for mode, values in (("occupancy", np.array([1, 1, 0], np.uint8)), ("set", np.array([9, 0, 17], np.uint8))):
        m.edit(coords, values, mode)
        r.edit_collider(2, coords, values, mode)
        _assert_same(r, 2, m)
    assert len(m.pos) == 1
    # the written voxels show at the held brick's own position
    assert m.get((-16 + 3, 5, 24 + 4)) == r.read_collider(2)[1][0]["voxels"][3 + 8 * 5 + 64 * 4]
    r.close()


def test_occupancy_edits_keep_a_classified_shape_classified():
    """A shape typed by classifyFromNeighbors stays so under occupancy edits:
    every solid voxel equals classifyFromNeighbors of the final occupancy.
    The edits stay within bricks [0, 3)^3, whose hashes are distinct (a voxel
    written through a shared hash shows at another position, which no
    occupancy rule keeps consistent)."""
    cells = {hash_brick((x, y, z)) for x in range(3) for y in range(3) for z in range(3)}
    assert len(cells) == 27
    rng = np.random.default_rng(7)
    m = _classified_block((1, 1, 1), (16, 8, 16))
    for _ in range(3):
        coords = _random_edits(rng, 400, 0, 24)
        m.edit(coords, rng.integers(0, 2, size=len(coords)).astype(np.uint8), "occupancy")
    for p, v in zip(m.pos, m.vox):
        for i in np.nonzero(v & 7)[0]:
            u = (p[0] * 8 + i % 8, p[1] * 8 + (i // 8) % 8, p[2] * 8 + i // 64)
            assert v[i] == m.classify(u), u


def test_carving_everything_leaves_zero_bounds():
    m = _classified_block((0, 0, 0), (4, 4, 4))
    bricks = _bricks_of(m)
    r = _oracle_with(4, 0.1, bricks)
    coords = np.array([(x, y, z) for x in range(4) for y in range(4) for z in range(4)], np.int32)
    r.edit_collider(4, coords, np.zeros(len(coords), np.uint8), "occupancy")
    info, b = r.read_collider(4)
    assert info["solid_count"] == 0 and list(info["min_bound"]) == [0, 0, 0] and list(info["max_bound"]) == [0, 0, 0]
    assert np.isinf(info["aabb_min"]).all() and len(b) == 1
    r.close()
