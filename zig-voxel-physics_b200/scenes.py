"""Seeded synthetic scenes for the five benchmark configurations.

Every scene is a list of colliders (sparse 8x8x8 bricks of CollisionVoxel
bytes) plus a body table, in the layouts of include/vxp.h.  The same arrays
feed the CUDA library, the CPU oracle and the CPU baseline, so all three run
on identical inputs.

Voxel classification follows the reference:
  * classify_from_neighbors: classifyFromNeighbors / classifyVoxel /
    computeNormalIndex (src/collision_voxel.zig:103-235);
  * readme_box: the cube classification of the README quick start
    (README.md:84-116) with the boundary test at the cube's first and last
    voxel;
  * example_ground / ground_slab: the ground-slab convention of
    examples/basic.zig:91-122 (face voxels with a +y normal, edge rims,
    corner corners);
  * example_box: the 3x3x3 box of examples/basic.zig:125-156.

Two rules of the reference decide how a one-voxel-thick ground slab must be
built for its bodies to rest on it:
  * the brick map is keyed by hashBrickPos alone (src/collider.zig:153,
    187-192, 232-238), and that hash collides for small brick positions of
    mixed sign, e.g. (-4,0,1) and (2,0,-1): the second brick's voxels are
    written into the first, which keeps its own position.  A 64x64 slab at
    voxels [-32,32) keeps only 40 of its 64 bricks and loses the strip
    z >= 1.6 m (local), AABB included.  Slabs here therefore sit at
    non-negative voxel coordinates (no merges up to 512x512), and the body
    is placed to centre them;
  * classifyFromNeighbors (src/collision_voxel.zig:103-130, 194-235) types a
    voxel with two empty faces as an edge and sums the empty faces'
    directions; a one-voxel slab's +y and -y cancel to (0,0,0), which
    findClosestNormalIndex (src/collision_voxel.zig:85-99) maps to index 0,
    +x.  Contacts on such a slab get a horizontal normal whenever the
    voxel pair's direction leans towards +x (generateContact,
    src/narrow_phase.zig:860-922), and boxes sink through it.  Ground slabs
    therefore use the example's explicit classification.

Boxes are placed by their centres and rotated about them
(origin_for_centre): the body position is the collider's voxel origin, a
corner of the box, so a rotation applied there could put a box into the
ground before the first step, and only corner voxels ever meet the ground's
face voxels (src/narrow_phase.zig:701-709).

One rule is the reference's and no scene avoids it: Quat.toMat3
(src/math.zig:350-372) is the transpose of the rotation Quat.rotate applies,
so the world inverse inertia (src/body.zig:386-392, src/solver.zig:351-354)
is R^T I^-1 R.  Cubes do not notice; a long box's contacts can get a normal
mass an order of magnitude too small, so long boxes under load in the pile
sink slowly into the ground.

Bodies are VoxelBody records (src/body.zig:177-263): dynamic bodies get
BodyProperties.default damping (0.3 / 0.5) and the mass properties of
computeMassProperties (src/body.zig:462-519); static bodies get static_props
and start asleep (initStatic, src/body.zig:226-243).  Friction and
restitution are PhysicsConfig's defaults 0.6 / 0.2 (src/system.zig:64-65).
"""
from __future__ import annotations

import dataclasses
import math
from typing import Callable

import numpy as np

from . import abi

# NORMAL_LUT (src/collision_voxel.zig:47-76)
NORMAL_LUT = np.array(
    [
        (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1),
        (1, 1, 0), (1, -1, 0), (-1, 1, 0), (-1, -1, 0), (1, 0, 1), (1, 0, -1),
        (-1, 0, 1), (-1, 0, -1), (0, 1, 1), (0, 1, -1), (0, -1, 1), (0, -1, -1),
        (1, 1, 1), (1, 1, -1), (1, -1, 1), (1, -1, -1), (-1, 1, 1), (-1, 1, -1),
        (-1, -1, 1), (-1, -1, -1),
    ],
    dtype=np.int32,
)
T_EMPTY, T_CORNER, T_EDGE, T_FACE, T_INSIDE = 0, 1, 2, 3, 4


def _normal_index_table() -> np.ndarray:
    """computeNormalIndex for all 64 empty-neighbour masks.  Every non-zero
    (dx, dy, dz) in {-1,0,1}^3 is in NORMAL_LUT; (0,0,0) falls back to
    findClosestNormalIndex, whose dot products are all zero, i.e. index 0."""
    lut = {tuple(v): i for i, v in enumerate(NORMAL_LUT.tolist())}
    out = np.zeros(64, dtype=np.uint8)
    for m in range(64):
        if m == 0:
            continue
        dx = (1 if m & 2 else 0) - (1 if m & 1 else 0)
        dy = (1 if m & 8 else 0) - (1 if m & 4 else 0)
        dz = (1 if m & 32 else 0) - (1 if m & 16 else 0)
        out[m] = lut.get((dx, dy, dz), 0)
    return out


NORMAL_INDEX = _normal_index_table()
_POP = np.array([bin(m).count("1") for m in range(64)], dtype=np.uint8)
_TYPE_OF_POP = np.array([T_INSIDE, T_FACE, T_EDGE, T_CORNER, T_CORNER, T_CORNER, T_CORNER], dtype=np.uint8)


def voxel_byte(vtype, normal):
    """CollisionVoxel packed byte: type in bits 0-2, normal index in bits 3-7."""
    return (np.asarray(vtype, dtype=np.uint8) & 7) | (np.asarray(normal, dtype=np.uint8) << 3)


def classify_from_neighbors(solid: np.ndarray) -> np.ndarray:
    """Per-voxel CollisionVoxel bytes of a dense occupancy grid indexed [x, y, z];
    voxels outside the grid count as empty."""
    s = np.pad(solid.astype(bool), 1)
    c = s[1:-1, 1:-1, 1:-1]
    mask = np.zeros(c.shape, dtype=np.uint8)
    mask |= (~s[:-2, 1:-1, 1:-1]).astype(np.uint8) * 1
    mask |= (~s[2:, 1:-1, 1:-1]).astype(np.uint8) * 2
    mask |= (~s[1:-1, :-2, 1:-1]).astype(np.uint8) * 4
    mask |= (~s[1:-1, 2:, 1:-1]).astype(np.uint8) * 8
    mask |= (~s[1:-1, 1:-1, :-2]).astype(np.uint8) * 16
    mask |= (~s[1:-1, 1:-1, 2:]).astype(np.uint8) * 32
    out = voxel_byte(_TYPE_OF_POP[_POP[mask]], NORMAL_INDEX[mask])
    out[~c] = 0
    return out


_K1 = np.uint64(0x517CC1B727220A95)
_K2 = np.uint64(0x9E3779B97F4A7C15)


def hash_brick_pos(bx, by, bz) -> np.ndarray:
    """VoxelCollider.hashBrickPos (src/collider.zig:187-192), wrapping u64."""
    ux = np.asarray(bx, dtype=np.int64).astype(np.uint64)
    uy = np.asarray(by, dtype=np.int64).astype(np.uint64)
    uz = np.asarray(bz, dtype=np.int64).astype(np.uint64)
    with np.errstate(over="ignore"):
        return ux ^ (uy * _K1) ^ (uz * _K2)


def bricks_from_calls(coords: np.ndarray, values: np.ndarray) -> np.ndarray:
    """The bricks a VoxelCollider holds after setCollisionVoxel(coords[i],
    values[i]) is called for every i in order (src/collider.zig:232-273).

    The brick map is keyed by hashBrickPos, which collides for some small
    brick positions (e.g. (0,0,-3) and (-2,0,3)): a voxel whose brick hashes
    like an existing brick is written into that brick (getOrCreateBrick finds
    it), which keeps the position it was created with.  The result lists one
    brick per distinct hash, in creation order, with the last value written to
    each of its 512 cells."""
    coords = np.asarray(coords, dtype=np.int64).reshape(-1, 3)
    values = np.asarray(values, dtype=np.uint8).reshape(-1)
    if len(coords) == 0:
        return np.zeros(0, dtype=abi.BRICK_DTYPE)
    bpos = coords >> 3
    local = (coords[:, 0] & 7) + 8 * (coords[:, 1] & 7) + 64 * (coords[:, 2] & 7)
    h = hash_brick_pos(bpos[:, 0], bpos[:, 1], bpos[:, 2])
    uniq, first, inv = np.unique(h, return_index=True, return_inverse=True)
    order = np.argsort(first, kind="stable")  # creation order of the bricks
    rank = np.empty(len(order), dtype=np.int64)
    rank[order] = np.arange(len(order))
    brick_of = rank[inv.reshape(-1)]
    out = np.zeros(len(order), dtype=abi.BRICK_DTYPE)
    out["pos"] = bpos[first[order]]
    # the last write of each (brick, cell) wins
    key = brick_of * 512 + local
    rev_key = key[::-1]
    _, last_rev = np.unique(rev_key, return_index=True)
    last = len(key) - 1 - last_rev
    vox = np.zeros((len(order), 512), dtype=np.uint8)
    vox[brick_of[last], local[last]] = values[last]
    out["voxels"] = vox
    return out


def dense_to_bricks(vox: np.ndarray, origin=(0, 0, 0)) -> np.ndarray:
    """Bricks of a collider built from a dense voxel-byte grid [x, y, z] whose
    [0,0,0] sits at voxel coordinate `origin`: setCollisionVoxel is called for
    every non-empty voxel in z, y, x loop order (z outermost), as the
    reference's examples build their colliders."""
    ox, oy, oz = (int(v) for v in origin)
    zyx = np.argwhere((np.transpose(vox, (2, 1, 0)) & 7) != 0)  # rows (z, y, x), z-major order
    if len(zyx) == 0:
        return np.zeros(0, dtype=abi.BRICK_DTYPE)
    coords = np.stack([zyx[:, 2] + ox, zyx[:, 1] + oy, zyx[:, 0] + oz], axis=1)
    values = vox[zyx[:, 2], zyx[:, 1], zyx[:, 0]]
    return bricks_from_calls(coords, values)


def readme_box(n: int = 8) -> np.ndarray:
    """n^3 cube at voxels (0..n-1)^3, classified as in the README example."""
    idx = np.arange(n)
    x, y, z = np.meshgrid(idx, idx, idx, indexing="ij")
    on_x = (x == 0) | (x == n - 1)
    on_y = (y == 0) | (y == n - 1)
    on_z = (z == 0) | (z == n - 1)
    edges = on_x.astype(np.uint8) + on_y + on_z
    vtype = np.select([edges == 3, edges == 2, edges == 1], [T_CORNER, T_EDGE, T_FACE], T_INSIDE)
    normal = np.full(x.shape, 2, dtype=np.uint8)
    normal[on_x & (x == n - 1)] = 0
    normal[on_x & (x == 0)] = 1
    normal[on_y & (y == n - 1)] = 2
    normal[on_y & (y == 0)] = 3
    normal[on_z & (z == n - 1)] = 4
    normal[on_z & (z == 0)] = 5
    return dense_to_bricks(voxel_byte(vtype, normal))


def _ground_voxels(nx: int, nz: int) -> np.ndarray:
    """Voxel bytes [x, 1, z] of an nx x 1 x nz ground slab classified as in
    examples/basic.zig:91-122: face with the +y normal (2) inside, edge rims
    with the outward-and-up normals (-x: 8, +x: 6, -z: 15, +z: 14), corner
    corners (-x-z: 23, +x-z: 19, -x+z: 22, +x+z: 18)."""
    i = np.arange(nx)[:, None]
    k = np.arange(nz)[None, :]
    lo_x, hi_x = i == 0, i == nx - 1
    lo_z, hi_z = k == 0, k == nz - 1
    on_x, on_z = lo_x | hi_x, lo_z | hi_z
    shape = (nx, nz)
    vtype = np.full(shape, T_FACE, dtype=np.uint8)
    normal = np.full(shape, 2, dtype=np.uint8)
    corner = on_x & on_z
    vtype[corner] = T_CORNER
    normal[corner & lo_x & lo_z] = 23
    normal[corner & hi_x & lo_z] = 19
    normal[corner & lo_x & hi_z] = 22
    normal[corner & hi_x & hi_z] = 18
    ex = on_x & ~on_z
    vtype[ex] = T_EDGE
    normal[ex] = np.broadcast_to(np.where(lo_x, 8, 6), shape)[ex]
    ez = on_z & ~on_x
    vtype[ez] = T_EDGE
    normal[ez] = np.broadcast_to(np.where(lo_z, 15, 14), shape)[ez]
    return voxel_byte(vtype, normal)[:, None, :]


def example_ground(size: int) -> np.ndarray:
    """size x 1 x size slab at x, z in [-size/2, size/2), y = 0, exactly as
    examples/basic.zig:91-122 builds it (its loops run z then x).  At size 64
    the brick hash merges 24 of its 64 bricks (see the module docstring);
    the reference's own example uses size 16, which merges none."""
    half = size // 2
    return dense_to_bricks(_ground_voxels(size, size), origin=(-half, 0, -half))


def ground_slab(nx: int, nz: int) -> np.ndarray:
    """nx x 1 x nz ground slab at voxels [0,nx) x 0 x [0,nz), classified as in
    examples/basic.zig:91-122; non-negative brick positions keep every brick
    distinct under hashBrickPos."""
    return dense_to_bricks(_ground_voxels(nx, nz))


def example_box() -> np.ndarray:
    """The 3x3x3 box of examples/basic.zig:125-156: voxels (-1..1)^3 written in
    z, y, x order, typed by the count of boundary axes, normal 0 unless a
    boundary axis overrides it (x, then y, then z)."""
    idx = np.arange(-1, 2)
    x, y, z = np.meshgrid(idx, idx, idx, indexing="ij")
    on_x, on_y, on_z = x != 0, y != 0, z != 0
    edges = on_x.astype(np.uint8) + on_y + on_z
    vtype = np.select([edges == 3, edges == 2, edges == 1], [T_CORNER, T_EDGE, T_FACE], T_INSIDE)
    normal = np.zeros(x.shape, dtype=np.uint8)
    normal[on_x & (x > 0)] = 0
    normal[on_x & (x < 0)] = 1
    normal[on_y & (y > 0)] = 2
    normal[on_y & (y < 0)] = 3
    normal[on_z & (z > 0)] = 4
    normal[on_z & (z < 0)] = 5
    return dense_to_bricks(voxel_byte(vtype, normal), origin=(-1, -1, -1))


def solid_box(ex: int, ey: int, ez: int) -> np.ndarray:
    """ex x ey x ez solid box at the voxel origin, classified from neighbours."""
    return dense_to_bricks(classify_from_neighbors(np.ones((ex, ey, ez), dtype=bool)))


def walled_bin(nx: int, ny: int, nz: int, wall: int = 2) -> np.ndarray:
    """Static bin: floor `wall` voxels thick and four walls, classified from
    neighbours, at voxels [0,nx) x [0,ny) x [0,nz)."""
    s = np.zeros((nx, ny, nz), dtype=bool)
    s[:, :wall, :] = True
    s[:wall, :, :] = True
    s[-wall:, :, :] = True
    s[:, :, :wall] = True
    s[:, :, -wall:] = True
    return dense_to_bricks(classify_from_neighbors(s))


def value_noise_solid(rng: np.random.Generator, n: int = 64, lattice: int = 8, threshold: float = 0.5) -> np.ndarray:
    """Occupancy of trilinear value noise (lattice^3 of U[0,1)) sampled at the
    n^3 voxel centres, thresholded."""
    g = rng.random((lattice + 1, lattice + 1, lattice + 1))
    t = (np.arange(n) + 0.5) * (lattice / n)
    i0 = np.floor(t).astype(int)
    f = t - i0
    i1 = i0 + 1
    fx, fy, fz = f[:, None, None], f[None, :, None], f[None, None, :]
    a, b = i0, i1
    c000 = g[a][:, a][:, :, a]
    c100 = g[b][:, a][:, :, a]
    c010 = g[a][:, b][:, :, a]
    c110 = g[b][:, b][:, :, a]
    c001 = g[a][:, a][:, :, b]
    c101 = g[b][:, a][:, :, b]
    c011 = g[a][:, b][:, :, b]
    c111 = g[b][:, b][:, :, b]
    v = (
        c000 * (1 - fx) * (1 - fy) * (1 - fz)
        + c100 * fx * (1 - fy) * (1 - fz)
        + c010 * (1 - fx) * fy * (1 - fz)
        + c110 * fx * fy * (1 - fz)
        + c001 * (1 - fx) * (1 - fy) * fz
        + c101 * fx * (1 - fy) * fz
        + c011 * (1 - fx) * fy * fz
        + c111 * fx * fy * fz
    )
    return v >= threshold


def shoemake_quat(rng: np.random.Generator, n: int) -> np.ndarray:
    """Uniform random unit quaternions (x, y, z, w), Shoemake's method, as f32."""
    u1, u2, u3 = rng.random(n), rng.random(n), rng.random(n)
    a, b = np.sqrt(1 - u1), np.sqrt(u1)
    q = np.stack(
        [a * np.sin(2 * np.pi * u2), a * np.cos(2 * np.pi * u2), b * np.sin(2 * np.pi * u3), b * np.cos(2 * np.pi * u3)],
        axis=1,
    )
    return q.astype(np.float32)


def origin_for_centre(centre: np.ndarray, rot: np.ndarray, half: np.ndarray) -> np.ndarray:
    """Body positions (the collider's voxel origin, src/body.zig:177-203) that
    put each box's centre `half` (local) at `centre` (world) under rotation
    `rot` (x, y, z, w): position = centre - R(rot) half.  Rotating about the
    centre keeps a box inside the sphere of radius |half| around its lattice
    point, so a lattice whose lowest centres sit that far above the ground
    starts with no box in the ground."""
    q = np.asarray(rot, dtype=np.float64)
    u, w = q[:, :3], q[:, 3:4]
    v = np.broadcast_to(np.asarray(half, dtype=np.float64), u.shape)
    t = 2.0 * np.cross(u, v)
    r = v + w * t + np.cross(u, t)
    return (np.asarray(centre, dtype=np.float64) - r).astype(np.float32)


# ---------------------------------------------------------------------------
@dataclasses.dataclass
class Collider:
    id: int
    voxel_size: float
    bricks: np.ndarray


@dataclasses.dataclass
class Scene:
    name: str
    colliders: list
    bodies: np.ndarray
    dt: float
    steps: int
    config: dict
    pair_margin: float = 0.1
    notes: str = ""

    @property
    def dynamic_count(self) -> int:
        return int((self.bodies["body_type"] == abi.BODY_DYNAMIC).sum())


MassFn = Callable[[float, np.ndarray, float], tuple]


def default_mass_fn() -> MassFn:
    """computeMassProperties through the library's host entry point."""
    import ctypes

    lib = abi.load()

    def fn(vs: float, bricks: np.ndarray, density: float):
        im = ctypes.c_float(0.0)
        inv = np.zeros(9, dtype=np.float32)
        rc = lib.vxp_mass_properties(np.float32(vs), abi.ptr(bricks), len(bricks), np.float32(density),
                                     ctypes.byref(im), abi.ptr(inv))
        if rc != 0:
            raise RuntimeError(f"vxp_mass_properties failed: {rc}")
        return np.float32(im.value), inv

    return fn


def _static_body(bid: int, cid: int, pos) -> np.ndarray:
    """A one-row body table holding a static body."""
    b = np.zeros(1, dtype=abi.BODY_DTYPE)
    b["id"] = bid
    b["body_type"] = abi.BODY_STATIC
    b["collider_id"] = cid
    b["is_sleeping"] = 1
    b["position"] = pos
    b["rotation"] = (0, 0, 0, 1)
    b["inv_mass"] = 0.0
    b["friction"] = 0.6
    b["restitution"] = 0.2
    return b


def _dynamic_bodies(ids, cids, pos, rot, mass_of: dict) -> np.ndarray:
    n = len(ids)
    b = np.zeros(n, dtype=abi.BODY_DTYPE)
    b["id"] = ids
    b["body_type"] = abi.BODY_DYNAMIC
    b["collider_id"] = cids
    b["position"] = np.asarray(pos, dtype=np.float32)
    b["rotation"] = np.asarray(rot, dtype=np.float32)
    for i, c in enumerate(cids):
        im, inv = mass_of[int(c)]
        b["inv_mass"][i] = im
        b["inv_inertia_local"][i] = inv
    b["friction"] = 0.6
    b["restitution"] = 0.2
    b["linear_damping"] = 0.3
    b["angular_damping"] = 0.5
    return b


def config1(mass_fn: MassFn | None = None, n_side: int = 4, seed: int = 1, steps: int = 300) -> Scene:
    """64 solid 8^3 cubes (one brick each, vs 0.2, 1 kg per voxel), centres on
    a 4x4x4 lattice at 2 m spacing, lowest layer 3 m up, over a static 64x1x64 slab at
    y = 0 spanning x, z in [-6.4, 6.4) m (created first, so it is body A of
    every ground pair; its voxels sit at [0,64) and the body at x = z = -6.4 so
    that no brick is merged by the brick hash); +-0.1 m position jitter,
    uniform random orientations about the cube's centre; dt 1/60, 4
    substeps, 300 steps."""
    mass_fn = mass_fn or default_mass_fn()
    rng = np.random.default_rng(seed)
    vs = 0.2
    ground = Collider(0, vs, ground_slab(64, 64))
    box = Collider(1, vs, readme_box(8))
    density = 1.0 / (vs ** 3)
    mass = {1: mass_fn(vs, box.bricks, np.float32(density))}
    n = n_side ** 3
    grid = np.array([(i, j, k) for j in range(n_side) for k in range(n_side) for i in range(n_side)], dtype=np.float64)
    off = (n_side - 1) / 2.0
    centre = np.stack([(grid[:, 0] - off) * 2.0, 3.0 + grid[:, 1] * 2.0, (grid[:, 2] - off) * 2.0], axis=1)
    centre += rng.uniform(-0.1, 0.1, size=centre.shape)
    rot = shoemake_quat(rng, n)
    pos = origin_for_centre(centre, rot, np.full(3, 8 * vs * 0.5))
    bodies = np.concatenate(
        [_static_body(1, 0, (-6.4, -vs * 0.5, -6.4)),
         _dynamic_bodies(np.arange(2, n + 2), np.ones(n, int), pos, rot, mass)]
    )
    return Scene("config1_small", [ground, box], bodies, 1.0 / 60.0, steps, dict(substeps=4), 0.1,
                 notes=f"{n} cubes 8^3 vs0.2 on 64x1x64 slab, seed {seed}")


def basic_example(mass_fn: MassFn | None = None, centred_ground: bool = True) -> Scene:
    """The scene of examples/basic.zig:16-90: a static 16x1x16 ground slab
    (vs 0.2) at (0, -0.1, 0) created first, then the 3x3x3 box at (0, 3, 0)
    with density 1.0 (createDynamicBody, src/system.zig:294-320: 1 kg per m^3,
    i.e. 0.008 kg per voxel); gravity -9.81, dt 1/60, 4 substeps, 2 velocity
    and 4 position iterations, warm starting and sleeping on, at most 600
    frames.  `centred_ground=False` builds the same slab at voxels [0,16)
    placed at (-1.6, -0.1, -1.6)."""
    mass_fn = mass_fn or default_mass_fn()
    vs = 0.2
    if centred_ground:
        ground, gpos = Collider(0, vs, example_ground(16)), (0.0, -vs * 0.5, 0.0)
    else:
        ground, gpos = Collider(0, vs, ground_slab(16, 16)), (-1.6, -vs * 0.5, -1.6)
    box = Collider(1, vs, example_box())
    mass = {1: mass_fn(vs, box.bricks, np.float32(1.0))}
    bodies = np.concatenate([_static_body(1, 0, gpos),
                             _dynamic_bodies([2], [1], [(0.0, 3.0, 0.0)], [(0.0, 0.0, 0.0, 1.0)], mass)])
    return Scene("basic_example", [ground, box], bodies, 1.0 / 60.0, 600,
                 dict(substeps=4, velocity_iterations=2, position_iterations=4), 0.1,
                 notes="examples/basic.zig: 3x3x3 box dropped from 3 m onto a 16x1x16 slab")


_BOX_CACHE: dict = {}


def _box(key, vs, mass_fn):
    """Bricks and mass properties of one solid box shape (cached by extents)."""
    k = (key, float(vs), id(mass_fn))
    if k not in _BOX_CACHE:
        br = solid_box(*key)
        _BOX_CACHE[k] = (br, mass_fn(vs, br, np.float32(1.0 / (vs ** 3))))
    return _BOX_CACHE[k]


def _random_box_colliders(rng, n, first_cid, vs, mass_fn, lo=2, hi=16):
    ext = rng.integers(lo, hi + 1, size=(n, 3))
    cols, mass = [], {}
    for i in range(n):
        key = tuple(int(v) for v in ext[i])
        br, m = _box(key, vs, mass_fn)
        cid = first_cid + i
        cols.append(Collider(cid, vs, br))
        mass[cid] = m
    return cols, mass, ext


def box_shape_id(ex: int, ey: int, ez: int, lo: int = 2, hi: int = 16) -> int:
    """Id of a box shape in the shared shape library (1 + index of the extents)."""
    span = hi - lo + 1
    return 1 + ((ex - lo) * span + (ey - lo)) * span + (ez - lo)


def shape_library(mass_fn=None, vs: float = 0.1, lo: int = 2, hi: int = 16) -> list:
    """Every config-2 box shape once, ids box_shape_id(...), plus the 64x1x64
    ground slab as id 0: a server uploads these once and jobs refer to them."""
    mass_fn = mass_fn or default_mass_fn()
    out = [Collider(0, vs, ground_slab(64, 64))]
    for ex in range(lo, hi + 1):
        for ey in range(lo, hi + 1):
            for ez in range(lo, hi + 1):
                br, _ = _box((ex, ey, ez), vs, mass_fn)
                out.append(Collider(box_shape_id(ex, ey, ez, lo, hi), vs, br))
    return out


def job_bodies(job: dict, mass_fn=None, vs: float = 0.1) -> np.ndarray:
    """Body table of a served job, its colliders given as shape-library ids."""
    mass_fn = mass_fn or default_mass_fn()
    rng = np.random.default_rng(job["seed"])
    n = job["bodies"]
    ext = rng.integers(2, 17, size=(n, 3))
    mass = {}
    cids = np.zeros(n, dtype=np.int64)
    for i in range(n):
        key = tuple(int(v) for v in ext[i])
        cids[i] = box_shape_id(*key)
        mass[int(cids[i])] = _box(key, vs, mass_fn)[1]
    k = np.arange(n)
    layer, cell = np.divmod(k, 9)
    cx, cz = np.divmod(cell, 3)
    half = ext * vs * 0.5
    centre = np.stack([(cx - 1) * 2.2, 1.6 + layer * 2.8, (cz - 1) * 2.2], axis=1).astype(np.float64)
    centre += rng.uniform(-0.1, 0.1, size=centre.shape)
    rot = shoemake_quat(rng, n)
    pos = origin_for_centre(centre, rot, half)
    return np.concatenate([_static_body(1, 0, (-3.2, -vs, -3.2)),
                           _dynamic_bodies(np.arange(2, n + 2), cids, pos, rot, mass)])


def config2(mass_fn: MassFn | None = None, n_side: int = 16, seed: int = 2, steps: int = 600) -> Scene:
    """4096 seeded random boxes (per-axis extents U{2..16} voxels, vs 0.1, sparse
    bricks, classified from neighbours, 1 kg per voxel) dropped with their
    centres on a 16^3 jittered lattice (2.8 m spacing, lowest layer 1.7 m up,
    so no box, whatever its rotation about its jittered centre, starts below
    the bin floor's top at 0.2 m) over a static 128x8x128 walled bin (floor and walls 2 voxels thick) that
    sits on a static 512x1x512 ground slab; dt 1/120, 8 substeps, 600 steps."""
    mass_fn = mass_fn or default_mass_fn()
    rng = np.random.default_rng(seed)
    vs = 0.1
    bin_c = Collider(0, vs, walled_bin(128, 8, 128))
    ground = Collider(1, vs, ground_slab(512, 512))
    n = n_side ** 3
    cols, mass, ext = _random_box_colliders(rng, n, 2, vs, mass_fn)
    sp = 2.8
    grid = np.array([(i, j, k) for j in range(n_side) for k in range(n_side) for i in range(n_side)], dtype=np.float64)
    off = (n_side - 1) / 2.0
    half = ext * vs * 0.5
    centre = np.stack([(grid[:, 0] - off) * sp, 1.7 + grid[:, 1] * sp, (grid[:, 2] - off) * sp], axis=1)
    centre += rng.uniform(-0.1, 0.1, size=centre.shape)
    rot = shoemake_quat(rng, n)
    pos = origin_for_centre(centre, rot, half)
    bodies = np.concatenate(
        [
            _static_body(1, 0, (-6.4, 0.0, -6.4)),
            _static_body(2, 1, (-25.6, -vs, -25.6)),
            _dynamic_bodies(np.arange(3, n + 3), np.arange(2, n + 2), pos, rot, mass),
        ]
    )
    return Scene("config2_pile", [bin_c, ground] + cols, bodies, 1.0 / 120.0, steps, dict(substeps=8), 0.1,
                 notes=f"{n} random boxes, 2.8 m lattice centred over a 12.8 m bin on a 51.2 m slab, seed {seed}")


def world_for_batch(rng, n_bodies: int, mass_fn: MassFn, vs: float = 0.1, steps: int = 300, name="world") -> Scene:
    """One world of the batched / served mixes: n bodies shaped as in config 2
    (random boxes U{2..16} voxels) in columns over the world's own static
    64x1x64 slab (vs 0.1): box centres in 3x3 columns at 2.2 m spacing, 2.8 m
    per layer from 1.6 m up, random orientations about the centre."""
    ground = Collider(0, vs, ground_slab(64, 64))
    cols, mass, ext = _random_box_colliders(rng, n_bodies, 1, vs, mass_fn)
    k = np.arange(n_bodies)
    layer, cell = np.divmod(k, 9)
    cx, cz = np.divmod(cell, 3)
    half = ext * vs * 0.5
    centre = np.stack([(cx - 1) * 2.2, 1.6 + layer * 2.8, (cz - 1) * 2.2], axis=1).astype(np.float64)
    centre += rng.uniform(-0.1, 0.1, size=centre.shape)
    rot = shoemake_quat(rng, n_bodies)
    pos = origin_for_centre(centre, rot, half)
    bodies = np.concatenate(
        [
            _static_body(1, 0, (-3.2, -vs, -3.2)),
            _dynamic_bodies(np.arange(2, n_bodies + 2), np.arange(1, n_bodies + 1), pos, rot, mass),
        ]
    )
    return Scene(name, [ground] + cols, bodies, 1.0 / 60.0, steps, dict(substeps=4), 0.1)


def config3(mass_fn: MassFn | None = None, n_worlds: int = 256, seed: int = 3, steps: int = 300) -> list:
    """256 independent worlds, bodies per world floor(exp(U(ln 8, ln 2048))),
    config-2 shapes, each world with its own 64x1x64 slab; dt 1/60, 4 substeps."""
    mass_fn = mass_fn or default_mass_fn()
    rng = np.random.default_rng(seed)
    sizes = np.floor(np.exp(rng.uniform(math.log(8), math.log(2048), size=n_worlds))).astype(int)
    return [world_for_batch(rng, int(s), mass_fn, steps=steps, name=f"world{w}") for w, s in enumerate(sizes)]


def config4(mass_fn: MassFn | None = None, n_side: int = 8, size: int = 64, seed: int = 4, steps: int = 120) -> Scene:
    """512 colliders of 64^3 voxels (512 bricks each, vs 0.1) filled by
    thresholding seeded 3-D value noise at 0.5 (about half full) and
    reclassified from neighbours, stacked 8x8x8 with 10% overlap inside a
    static walled bin; dt 1/60, 4 substeps, 120 steps."""
    mass_fn = mass_fn or default_mass_fn()
    rng = np.random.default_rng(seed)
    vs = 0.1
    n = n_side ** 3
    sp = 0.9 * size * vs
    span = n_side * sp + size * vs
    nb = int(math.ceil(span / vs)) + 8
    bin_c = Collider(0, vs, walled_bin(nb, 16, nb))
    cols, mass = [], {}
    density = np.float32(1.0 / (vs ** 3))
    for i in range(n):
        solid = value_noise_solid(rng, size)
        br = dense_to_bricks(classify_from_neighbors(solid))
        cols.append(Collider(i + 1, vs, br))
        mass[i + 1] = mass_fn(vs, br, density)
    grid = np.array([(i, j, k) for j in range(n_side) for k in range(n_side) for i in range(n_side)], dtype=np.float64)
    pos = np.stack([4 * vs + grid[:, 0] * sp, 2 * vs + grid[:, 1] * sp, 4 * vs + grid[:, 2] * sp], axis=1)
    rot = np.tile(np.array([0, 0, 0, 1], dtype=np.float32), (n, 1))
    bodies = np.concatenate(
        [_static_body(1, 0, (0.0, 0.0, 0.0)), _dynamic_bodies(np.arange(2, n + 2), np.arange(1, n + 1), pos, rot, mass)]
    )
    return Scene("config4_stress", [bin_c] + cols, bodies, 1.0 / 60.0, steps, dict(substeps=4), 0.1,
                 notes=f"{n} noise bodies {size}^3, 10% overlap lattice in a walled bin, seed {seed}")


def serving_jobs(n_jobs: int, seed: int = 5, rate: float = 200.0, lo: int = 16, hi: int = 4096,
                 steps_lo: int = 60, steps_hi: int = 600):
    """Poisson arrivals (mean `rate` jobs/s) of jobs: (arrival time s, bodies
    log-uniform [lo, hi], steps uniform {steps_lo..steps_hi}, world seed)."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, size=n_jobs))
    sizes = np.floor(np.exp(rng.uniform(math.log(lo), math.log(hi), size=n_jobs))).astype(int)
    steps = rng.integers(steps_lo, steps_hi + 1, size=n_jobs)
    seeds = rng.integers(0, 2 ** 31, size=n_jobs)
    return [dict(arrival=float(t[i]), bodies=int(sizes[i]), steps=int(steps[i]), seed=int(seeds[i])) for i in range(n_jobs)]


def job_world(job: dict, mass_fn: MassFn | None = None) -> Scene:
    mass_fn = mass_fn or default_mass_fn()
    rng = np.random.default_rng(job["seed"])
    return world_for_batch(rng, job["bodies"], mass_fn, steps=job["steps"], name=f"job{job['seed']}")
