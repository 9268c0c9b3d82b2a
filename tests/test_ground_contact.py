"""Bodies on a one-voxel ground slab, checked on the CPU oracle.

Three rules of the reference decide whether a box stays on a ground slab
one voxel thick, and the scene builder is written around them:

* the brick map is keyed by `hashBrickPos` alone (src/collider.zig:153,
  187-192, 232-238); the hash collides for small brick positions of mixed
  sign, so a 64x64 slab at voxels [-32, 32) keeps 40 of its 64 bricks and
  its collider ends at z = 1.6 m (local);
* `classifyFromNeighbors` (src/collision_voxel.zig:103-130, 194-235) types
  a voxel with empty +y and -y faces as an edge whose normal directions
  cancel to (0,0,0), which `findClosestNormalIndex`
  (src/collision_voxel.zig:85-99) maps to index 0, +x: contacts on such a
  slab can get a horizontal normal (src/narrow_phase.zig:860-922);
* only corner voxels meet a slab's face voxels (`shouldCheckCollision`,
  src/narrow_phase.zig:701-709), so a box whose corner starts below the
  slab is never pushed back.

The reference's own example (examples/basic.zig:16-90) is replayed as the
known-good case."""
import ctypes

import numpy as np

import oracle_api as O


def _metadata(vxp, vs, bricks):
    """VoxelCollider bounds and local AABB after recomputeMetadata."""
    bounds = np.zeros(6, np.int32)
    aabb = np.zeros(6, np.float32)
    solid = ctypes.c_uint32()
    rc = O.L.vxo_collider_metadata(np.float32(vs), vxp.abi.ptr(bricks), len(bricks), bounds.ctypes.data,
                                   aabb.ctypes.data, ctypes.byref(solid))
    assert rc == 0
    return bounds, aabb, solid.value


def _rotate(q, v):
    u, w = q[..., :3].astype(np.float64), q[..., 3:4].astype(np.float64)
    t = 2.0 * np.cross(u, v)
    return v + w * t + np.cross(u, t)


def _local_centres(vxp, scene):
    """Centre of each body's collider AABB in body coordinates."""
    cid = {c.id: c for c in scene.colliders}
    half = np.zeros((len(scene.bodies), 3))
    for i, b in enumerate(scene.bodies):
        c = cid[int(b["collider_id"])]
        _, aabb, _ = _metadata(vxp, c.voxel_size, c.bricks)
        half[i] = (aabb[:3].astype(np.float64) + aabb[3:]) * 0.5
    return half


def _centres(half, bodies):
    return bodies["position"] + _rotate(bodies["rotation"], half)


def _lowest_corner(vxp, scene):
    cid = {c.id: c for c in scene.colliders}
    out = np.zeros(len(scene.bodies))
    for i, b in enumerate(scene.bodies):
        c = cid[int(b["collider_id"])]
        _, aabb, _ = _metadata(vxp, c.voxel_size, c.bricks)
        corners = np.array([[x, y, z] for x in aabb[0::3] for y in aabb[1::3] for z in aabb[2::3]], np.float64)
        out[i] = (b["position"][1] + _rotate(np.broadcast_to(b["rotation"], (8, 4)), corners)[:, 1]).min()
    return out


def test_reference_example_box_rests_and_sleeps(vxp):
    """examples/basic.zig: the 3x3x3 box dropped from 3 m comes to rest on
    the 16x1x16 slab (its bottom, 0.2 m below its origin, on the slab top at
    y = 0.1) and falls asleep at frame 77; the slab placed at non-negative
    voxel coordinates gives the same frame and height."""
    results = []
    for centred in (True, False):
        sc = vxp.scenes.basic_example(O.mass_fn, centred_ground=centred)
        w = O.OracleWorld(**sc.config)
        w.load_scene(sc)
        frame = None
        for f in range(sc.steps):
            w.step(np.float32(sc.dt))
            box = w.get_bodies()[1]
            if box["is_sleeping"]:
                frame = f
                break
        w.close()
        assert frame == 77, frame
        bottom = float(box["position"][1]) - 0.2
        assert abs(bottom - 0.1) < 0.005, bottom
        assert np.all(box["linear_velocity"] == 0)
        results.append(box["position"].copy())
    assert np.allclose(results[0], results[1], atol=1e-5)


def test_mixed_sign_brick_positions_merge_and_cut_the_slab(vxp):
    """A 64x64 slab at voxels [-32, 32) keeps 40 bricks and its collider
    stops at z = 1.6 m; the same slab at [0, 64) keeps all 64 bricks."""
    sc = vxp.scenes
    centred = sc.example_ground(64)
    assert len(centred) == 40
    _, aabb, solid = _metadata(vxp, 0.2, centred)
    assert solid == 40 * 64
    assert aabb[5] == np.float32(1.6)
    shifted = sc.ground_slab(64, 64)
    assert len(shifted) == 64
    h = sc.hash_brick_pos(shifted["pos"][:, 0], shifted["pos"][:, 1], shifted["pos"][:, 2])
    assert len(np.unique(h)) == 64
    _, aabb, solid = _metadata(vxp, 0.2, shifted)
    assert solid == 64 * 64
    assert tuple(aabb) == (0.0, 0.0, 0.0, np.float32(12.8), np.float32(0.2), np.float32(12.8))
    # the 512x512 slab of the pile keeps every brick too
    big = sc.ground_slab(512, 512)
    assert len(big) == 64 * 64


def test_one_voxel_slab_from_neighbours_has_x_normals(vxp):
    """classifyFromNeighbors on a voxel with only +y and -y empty: an edge
    with normal index 0 (+x); the ground slab of the example is a face with
    the +y normal (index 2) instead."""
    sc = vxp.scenes
    # solid, -x, +x, -y, +y, -z, +z neighbours solid?
    byte = O.L.vxo_classify_from_neighbors(1, 1, 1, 0, 0, 1, 1)
    assert byte == int(sc.voxel_byte(sc.T_EDGE, 0))
    thin = sc.classify_from_neighbors(np.ones((8, 1, 8), dtype=bool))
    assert np.all(thin[1:-1, 0, 1:-1] == sc.voxel_byte(sc.T_EDGE, 0))
    ground = sc._ground_voxels(8, 8)
    assert np.all(ground[1:-1, 0, 1:-1] == sc.voxel_byte(sc.T_FACE, 2))
    assert ground[0, 0, 0] == sc.voxel_byte(sc.T_CORNER, 23)
    assert ground[7, 0, 3] == sc.voxel_byte(sc.T_EDGE, 6)


def test_lattice_boxes_start_above_the_ground(vxp):
    """Boxes are rotated about their centres, so none starts in the ground:
    config 1 over its slab top (y = 0.1), a batched world over its slab top
    (y = 0), a 6x6x6 pile over the bin floor (y = 0.2)."""
    sc = vxp.scenes
    s1 = sc.config1(mass_fn=O.mass_fn)
    assert _lowest_corner(vxp, s1)[1:].min() > 0.1 + 1.0
    w = sc.world_for_batch(np.random.default_rng(9), 96, O.mass_fn)
    assert _lowest_corner(vxp, w)[1:].min() > 0.0
    s2 = sc.config2(mass_fn=O.mass_fn, n_side=6)
    assert _lowest_corner(vxp, s2)[2:].min() > 0.2


def _leave_points(half, w, dt, steps, below):
    """Step a world and return, for each body whose centre drops below
    `below`, the centre where it first did."""
    gone = {}
    for _ in range(steps):
        w.step(np.float32(dt))
        c = _centres(half, w.get_bodies())
        for i in np.nonzero(c[1:, 1] < below)[0] + 1:
            gone.setdefault(int(i), c[i].copy())
    return gone


def test_config1_keeps_every_cube_on_the_slab(vxp):
    """300 steps of config 1: no cube's centre goes below the slab top
    (y = 0.1) inside the slab's 12.8 m footprint (cubes thrown apart by the
    lattice's initial overlaps may roll off its edge) and some fall asleep.
    The same scene over the centred slab of 40 bricks loses the cubes above
    the missing strip, inside the nominal footprint."""
    sc = vxp.scenes
    s = sc.config1(mass_fn=O.mass_fn)
    half = _local_centres(vxp, s)
    w = O.OracleWorld(substeps=4)
    w.load_scene(s)
    gone = _leave_points(half, w, s.dt, 300, 0.1)
    asleep = int(w.get_bodies()["is_sleeping"][1:].sum())
    w.close()
    assert all(abs(c[0]) > 6.4 or abs(c[2]) > 6.4 for c in gone.values()), gone
    assert len(gone) <= 8
    assert asleep >= 10

    s.colliders[0] = sc.Collider(0, 0.2, sc.example_ground(64))
    s.bodies["position"][0] = (0.0, -0.1, 0.0)
    w = O.OracleWorld(substeps=4)
    w.load_scene(s)
    gone = _leave_points(half, w, s.dt, 300, 0.1)
    w.close()
    through = [c for c in gone.values() if abs(c[0]) < 6.4 and abs(c[2]) < 6.4]
    assert len(through) >= 10
    # they went down over the strip z >= 1.6 m that the merged bricks left empty
    assert all(c[2] > 1.6 - 0.8 for c in through), through


def test_thin_slab_world_keeps_boxes_that_land_on_it(vxp):
    """A 48-box world (config-3 shapes) over the example-classified slab:
    no box passes through inside the slab's footprint in 200 steps (boxes
    that leave roll off its 6.4 m edge).  Classified from neighbours, the
    same slab lets several through."""
    sc = vxp.scenes

    def through(old):
        s = sc.world_for_batch(np.random.default_rng(3), 48, O.mass_fn, steps=200)
        if old:
            s.colliders[0] = sc.Collider(0, 0.1, sc.dense_to_bricks(
                sc.classify_from_neighbors(np.ones((64, 1, 64), dtype=bool))))
        w = O.OracleWorld(**s.config)
        w.load_scene(s)
        gone = _leave_points(_local_centres(vxp, s), w, s.dt, 200, -0.3)
        w.close()
        return sum(1 for c in gone.values() if abs(c[0]) < 3.2 and abs(c[2]) < 3.2)

    assert through(old=False) == 0
    assert through(old=True) >= 3


def test_world_inverse_inertia_is_rotated_by_the_transpose(vxp):
    """Quat.toMat3 (src/math.zig:350-372) is the transpose of the rotation
    Quat.rotate applies (src/math.zig:267-283), and Mat3.mulVec
    (src/math.zig:446-452) multiplies row by vector, so
    VoxelBody.getWorldInvInertia (src/body.zig:386-392), and the solver's copy
    of it after every integration (src/solver.zig:351-354), is
    R^T I^-1 R instead of R I^-1 R^T.  Only bodies whose inertia is not
    isotropic notice: a cube's is the same either way."""
    q = np.array([0, 0, np.sin(np.pi / 12), np.cos(np.pi / 12)], dtype=np.float32)  # 30 degrees about +z
    inv_local = np.diag(np.array([1.0, 2.0, 3.0], dtype=np.float32)).astype(np.float32)
    out = np.zeros(9, dtype=np.float32)
    O.L.vxo_world_inv_inertia(q.ctypes.data, inv_local.ctypes.data, out.ctypes.data)
    rot = np.zeros((3, 3))
    for j in range(3):
        e = np.zeros(3, dtype=np.float32)
        e[j] = 1
        col = np.zeros(3, dtype=np.float32)
        O.L.vxo_quat_rotate(q.ctypes.data, e.ctypes.data, col.ctypes.data)
        rot[:, j] = col
    got = out.reshape(3, 3)
    assert np.allclose(got, rot.T @ inv_local @ rot, atol=1e-6)
    assert not np.allclose(got, rot @ inv_local @ rot.T, atol=1e-3)
    iso = np.eye(3, dtype=np.float32) * np.float32(0.25)
    O.L.vxo_world_inv_inertia(q.ctypes.data, iso.ctypes.data, out.ctypes.data)
    assert np.allclose(out.reshape(3, 3), iso, atol=1e-7)


def test_long_box_contact_mass_uses_the_transposed_inertia(vxp):
    """A tilted 2x16x3 box (96 voxels, 96 kg) touching a floor two voxels
    thick: every contact point's normal mass after one step is
    1 / (1/m + (r x n) . R^T I^-1 R . (r x n)) (src/solver.zig:640-645 with
    the world inertia above), about half a kilogram, where the correctly
    rotated inertia would give more than ten times as much.  Impulses that small spin such a box
    instead of stopping it, which is how long boxes under load sink into
    the ground in the pile."""
    sc = vxp.scenes
    vs = 0.1
    ext = (2, 16, 3)
    floor = sc.Collider(0, vs, sc.dense_to_bricks(sc.classify_from_neighbors(np.ones((64, 2, 64), dtype=bool))))
    box = sc.Collider(1, vs, sc.solid_box(*ext))
    im, inv_local = O.mass_fn(vs, box.bricks, np.float32(1.0 / vs ** 3))
    half = np.array(ext, dtype=np.float64) * vs * 0.5
    axis = np.array([-1.28, 0.63, 0.58]) / np.linalg.norm([-1.28, 0.63, 0.58])
    rot = np.array([[*(axis * np.sin(0.98)), np.cos(0.98)]], dtype=np.float32)
    corners = np.array([[x, y, z] for x in (-1, 1) for y in (-1, 1) for z in (-1, 1)], np.float64) * half
    lowest = _rotate(np.broadcast_to(rot[0], (8, 4)), corners)[:, 1].min()
    centre = np.array([[0.0, 0.0 - lowest - 0.03, 0.0]])  # lowest corner 3 cm into the floor top (y = 0)
    pos = sc.origin_for_centre(centre, rot, half)
    bodies = np.concatenate([sc._static_body(1, 0, (-3.2, -0.2, -3.2)),
                             sc._dynamic_bodies([2], [1], pos, rot, {1: (im, inv_local)})])
    s = sc.Scene("tilted", [floor, box], bodies, 1.0 / 120.0, 1, dict(substeps=8), 0.1)
    w = O.OracleWorld(**s.config)
    w.load_scene(s)
    w.step(np.float32(s.dt))
    b = w.get_bodies()[1]
    man = w.manifolds()
    w.close()
    assert len(man) == 1 and man[0]["contact_count"] >= 1
    cols = np.zeros((3, 3))
    for j in range(3):
        e = np.zeros(3, dtype=np.float32)
        e[j] = 1
        col = np.zeros(3, dtype=np.float32)
        O.L.vxo_quat_rotate(b["rotation"].ctypes.data, e.ctypes.data, col.ctypes.data)
        cols[:, j] = col
    inv_i = inv_local.reshape(3, 3).astype(np.float64)
    for c in man[0]["contacts"][: man[0]["contact_count"]]:
        r = cols @ c["local_anchor_b"].astype(np.float64)
        rn = np.cross(r, c["normal"].astype(np.float64))
        as_reference = 1.0 / (im + rn @ (cols.T @ inv_i @ cols) @ rn)
        rotated = 1.0 / (im + rn @ (cols @ inv_i @ cols.T) @ rn)
        assert abs(c["normal_mass"] - as_reference) < 0.05 * as_reference, (c["normal_mass"], as_reference)
        assert rotated > 10.0 * as_reference, (rotated, as_reference)
