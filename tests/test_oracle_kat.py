"""The reference's own unit tests, restated against the CPU oracle.

Each test cites the Zig test block it follows.  These are the only
known-answer vectors the reference holds for the hot path; they pin the
oracle's type filter, classification, normal table, feature ids, SAT,
manifold replacement, warm-start transfer, cache keys, soft parameters,
computeOrthogonal, integrateRotationSmall and the sleep timer.
"""
import ctypes
import math

import numpy as np
import pytest

import oracle_api as O

L = O.L
EMPTY, CORNER, EDGE, FACE, INSIDE = 0, 1, 2, 3, 4


def f3(*v):
    return np.array(v, dtype=np.float32)


# ---------------------------------------------------------- collision_voxel.zig
def test_collision_rules_matrix():
    # collision_voxel.zig:247-271 and narrow_phase.zig:1736-1753
    yes = {(CORNER, CORNER), (CORNER, EDGE), (CORNER, FACE), (CORNER, INSIDE), (EDGE, CORNER), (EDGE, EDGE),
           (FACE, CORNER), (INSIDE, CORNER)}
    for a in range(5):
        for b in range(5):
            assert bool(L.vxo_should_collide(a, b)) == ((a, b) in yes), (a, b)


@pytest.mark.parametrize("mask,vtype", [(0b000111, CORNER), (0b000011, EDGE), (0b000001, FACE), (0b000000, INSIDE)])
def test_classify(mask, vtype):
    # collision_voxel.zig:273-292
    assert L.vxo_classify(1, mask) & 7 == vtype


def test_classify_empty():
    # collision_voxel.zig:294-298
    assert L.vxo_classify(0, 0b111111) == 0


def test_normal_lut():
    # collision_voxel.zig:300-322
    out = np.zeros(3, dtype=np.float32)
    L.vxo_normal_vec(0, out.ctypes.data)
    assert np.allclose(out, [1, 0, 0], atol=1e-6)
    L.vxo_normal_vec(3, out.ctypes.data)
    assert np.allclose(out, [0, -1, 0], atol=1e-6)
    for idx in (6, 18):
        L.vxo_normal_vec(idx, out.ctypes.data)
        assert abs(float(np.linalg.norm(out)) - 1.0) < 1e-6


def test_compute_normal_index():
    # collision_voxel.zig:324-337
    assert L.vxo_compute_normal_index(0b000010) == 0
    assert L.vxo_compute_normal_index(0b001010) == 6
    assert L.vxo_find_closest_normal(1.0, 0.1, -0.1) == 0


# ------------------------------------------------------------------ collider.zig
def test_brick_coordinates():
    # collider.zig:466-486
    b = np.zeros(3, dtype=np.int32)
    l = np.zeros(3, dtype=np.int32)
    for v, eb in [((15, 20, 25), (1, 2, 3)), ((-1, -10, -20), (-1, -2, -3))]:
        vv = np.array(v, dtype=np.int32)
        L.vxo_brick_coords(vv.ctypes.data, b.ctypes.data, l.ctypes.data)
        assert tuple(b) == eb
    vv = np.array((13, 18, 23), dtype=np.int32)
    L.vxo_brick_coords(vv.ctypes.data, b.ctypes.data, l.ctypes.data)
    assert tuple(l) == (5, 2, 7)


def test_collider_metadata_two_voxels(vxp):
    # collider.zig:488-499: two voxels far apart -> solid_count 2
    sc = vxp.scenes
    coords = np.array([[0, 0, 0], [10, 10, 10]])
    vals = np.array([sc.voxel_byte(CORNER, 0), sc.voxel_byte(EDGE, 1)])
    bricks = sc.bricks_from_calls(coords, vals)
    b6 = np.zeros(6, dtype=np.int32)
    a6 = np.zeros(6, dtype=np.float32)
    solid = ctypes.c_uint32(0)
    assert L.vxo_collider_metadata(np.float32(0.1), bricks.ctypes.data, len(bricks), b6.ctypes.data, a6.ctypes.data,
                                   ctypes.byref(solid)) == 0
    assert solid.value == 2
    assert tuple(b6) == (0, 0, 0, 11, 11, 11)


# -------------------------------------------------------------- narrow_phase.zig
def test_feature_id():
    # narrow_phase.zig:1635-1651
    def fid(a, b):
        aa, bb = np.array(a, dtype=np.int32), np.array(b, dtype=np.int32)
        return L.vxo_feature_id(aa.ctypes.data, bb.ctypes.data)

    assert fid((1, 2, 3), (4, 5, 6)) == fid((1, 2, 3), (4, 5, 6))
    assert fid((1, 2, 3), (4, 5, 6)) != fid((1, 2, 4), (4, 5, 6))
    # field layout: a.x | a.y<<16 | a.z<<32 | (b.x&15)<<48 | (b.y&15)<<52 | (b.z&15)<<56
    assert fid((1, 2, 3), (4, 5, 6)) == 1 | 2 << 16 | 3 << 32 | 4 << 48 | 5 << 52 | 6 << 56
    assert fid((-1, 0, 0), (-1, 0, 0)) == 0xFFFF | 0xF << 48


def obb(c, h, q=(0, 0, 0, 1)):
    return np.array([*c, *h, *q], dtype=np.float32)


def test_sat_separated():
    # narrow_phase.zig:1653-1666
    a, b = obb((0, 0, 0), (1, 1, 1)), obb((5, 0, 0), (1, 1, 1))
    assert L.vxo_sat_early_out(a.ctypes.data, b.ctypes.data) == 1


def test_sat_overlapping():
    # narrow_phase.zig:1668-1681
    a, b = obb((0, 0, 0), (1, 1, 1)), obb((1.5, 0, 0), (1, 1, 1))
    assert L.vxo_sat_early_out(a.ctypes.data, b.ctypes.data) == 0


def test_sat_with_penetration():
    # narrow_phase.zig:1683-1718
    d = ctypes.c_float(0)
    ax = np.zeros(3, dtype=np.float32)
    a, b = obb((0, 0, 0), (1, 1, 1)), obb((1.5, 0, 0), (1, 1, 1))
    assert L.vxo_sat_with_penetration(a.ctypes.data, b.ctypes.data, ctypes.byref(d), ax.ctypes.data) == 1
    assert d.value > 0 and abs(d.value - 0.5) <= 0.01
    c = obb((5, 0, 0), (1, 1, 1))
    assert L.vxo_sat_with_penetration(a.ctypes.data, c.ctypes.data, ctypes.byref(d), ax.ctypes.data) == 0


def test_sat_rotated():
    # narrow_phase.zig:1720-1734: B rotated 45 degrees about y, 2 m away: overlap
    q = np.zeros(4, dtype=np.float32)
    axis = f3(0, 1, 0)
    L.vxo_from_axis_angle(axis.ctypes.data, np.float32(math.pi / 4.0), q.ctypes.data)
    a, b = obb((0, 0, 0), (1, 1, 1)), obb((2, 0, 0), (1, 1, 1), q)
    assert L.vxo_sat_early_out(a.ctypes.data, b.ctypes.data) == 0


def test_manifold_keeps_deepest():
    # narrow_phase.zig:1755-1794: four contacts of penetration 0.1*i, then a
    # fifth of 10.0 replaces the shallowest.
    pens = np.array([np.float32(0.1) * np.float32(i) for i in range(4)] + [10.0], dtype=np.float32)
    fids = np.array([1, 2, 3, 4, 999], dtype=np.uint64)
    slots = np.zeros(4, dtype=np.uint32)
    n = ctypes.c_uint32(0)
    L.vxo_manifold_replay(pens.ctypes.data, fids.ctypes.data, 5, slots.ctypes.data, ctypes.byref(n))
    assert n.value == 4
    assert 4 in slots.tolist()  # the deep contact is held
    assert slots.tolist() == [4, 1, 2, 3]  # it took slot 0 (penetration 0.0)


def test_manifold_tie_keeps_earlier_slot():
    # strict "<" in addContact (narrow_phase.zig:471-476): equal penetrations
    # never replace, and the first minimum slot is the one replaced.
    pens = np.array([1, 1, 2, 2, 1, 3], dtype=np.float32)
    fids = np.arange(1, 7, dtype=np.uint64)
    slots = np.zeros(4, dtype=np.uint32)
    n = ctypes.c_uint32(0)
    L.vxo_manifold_replay(pens.ctypes.data, fids.ctypes.data, 6, slots.ctypes.data, ctypes.byref(n))
    assert slots.tolist() == [5, 1, 2, 3]


def test_contact_manager_warm_start():
    # narrow_phase.zig:1796-1825
    assert abs(L.vxo_contact_manager_warm(12345, np.float32(50.0), 12345) - 50.0) < 1e-3
    assert L.vxo_contact_manager_warm(12345, np.float32(50.0), 12346) == 0.0


def test_cache_basic_operations():
    # narrow_phase.zig:1884-1912 (capacity 64)
    c = L.vxo_cache_create(64)
    try:
        ids = np.array([1, 2], dtype=np.uint32)
        rp = f3(1, 0, 0)
        rr = np.array([0, 0, 0, 1], dtype=np.float32)
        cnt = ctypes.c_uint32(0)
        assert L.vxo_cache_get(c, ids.ctypes.data, rp.ctypes.data, rr.ctypes.data, ctypes.byref(cnt)) == 0
        st = np.zeros(4, dtype=np.uint64)
        L.vxo_cache_stats(c, st.ctypes.data)
        assert st[1] == 1 and st[0] == 0
        L.vxo_cache_put(c, ids.ctypes.data, rp.ctypes.data, rr.ctypes.data, 1, 1)
        assert L.vxo_cache_get(c, ids.ctypes.data, rp.ctypes.data, rr.ctypes.data, ctypes.byref(cnt)) == 2
        assert cnt.value == 1
        L.vxo_cache_stats(c, st.ctypes.data)
        assert st[0] == 1
    finally:
        L.vxo_cache_destroy(c)


def test_cache_invalidation():
    # narrow_phase.zig:1914-1937
    c = L.vxo_cache_create(64)
    try:
        z = f3(0, 0, 0)
        q = np.array([0, 0, 0, 1], dtype=np.float32)
        keys = [np.array(k, dtype=np.uint32) for k in ((1, 2), (1, 3), (2, 3))]
        for k in keys:
            L.vxo_cache_put(c, k.ctypes.data, z.ctypes.data, q.ctypes.data, 0, 0)
        cnt = ctypes.c_uint32(0)
        for k in keys:
            assert L.vxo_cache_get(c, k.ctypes.data, z.ctypes.data, q.ctypes.data, ctypes.byref(cnt)) != 0
        L.vxo_cache_invalidate(c, 1)
        assert L.vxo_cache_get(c, keys[0].ctypes.data, z.ctypes.data, q.ctypes.data, ctypes.byref(cnt)) == 0
        assert L.vxo_cache_get(c, keys[1].ctypes.data, z.ctypes.data, q.ctypes.data, ctypes.byref(cnt)) == 0
        assert L.vxo_cache_get(c, keys[2].ctypes.data, z.ctypes.data, q.ctypes.data, ctypes.byref(cnt)) != 0
    finally:
        L.vxo_cache_destroy(c)


def test_cache_key_transform_sensitivity():
    # narrow_phase.zig:1939-1969
    ids = np.array([1, 2], dtype=np.uint32)
    q = np.array([0, 0, 0, 1], dtype=np.float32)
    a, b = f3(0, 0, 0), f3(0.1, 0, 0)
    assert L.vxo_cache_key_eq(ids.ctypes.data, a.ctypes.data, q.ctypes.data, ids.ctypes.data, b.ctypes.data,
                              q.ctypes.data) == 0
    assert L.vxo_cache_key_eq(ids.ctypes.data, a.ctypes.data, q.ctypes.data, ids.ctypes.data, a.ctypes.data,
                              q.ctypes.data) == 1
    # 1 cm truncation: 0.004 and 0.006 both quantise to 0
    c = f3(0.004, 0, 0)
    d = f3(0.006, 0, 0)
    assert L.vxo_cache_key_eq(ids.ctypes.data, c.ctypes.data, q.ctypes.data, ids.ctypes.data, d.ctypes.data,
                              q.ctypes.data) == 1


# -------------------------------------------------------------------- solver.zig
def test_soft_params():
    # solver.zig:1007-1023
    out = np.zeros(3, dtype=np.float32)
    L.vxo_soft_params(np.float32(30.0), np.float32(1.0), np.float32(1.0 / 240.0), out.ctypes.data)
    assert out[0] > 0 and 0 < out[1] < 1 and 0 < out[2] < 1
    L.vxo_soft_params(np.float32(0.0), np.float32(1.0), np.float32(1.0 / 60.0), out.ctypes.data)
    assert tuple(out) == (0.0, 1.0, 1.0)


def test_compute_orthogonal():
    # solver.zig:1025-1041
    out = np.zeros(3, dtype=np.float32)
    for v in ((1, 0, 0), (0, 1, 0), (0, 0, 1), tuple(np.array([1, 1, 1]) / math.sqrt(3))):
        vv = f3(*v)
        L.vxo_compute_orthogonal(vv.ctypes.data, out.ctypes.data)
        assert abs(float(np.dot(vv, out))) < 1e-6


def test_integrate_rotation_small_identity():
    # solver.zig:1043-1051
    q = np.array([0, 0, 0, 1], dtype=np.float32)
    out = np.zeros(4, dtype=np.float32)
    z = f3(0, 0, 0)
    L.vxo_integrate_rotation_small(q.ctypes.data, z.ctypes.data, out.ctypes.data)
    assert np.all(np.abs(out - q) < 1e-6)


def test_solver_config_defaults(vxp):
    # solver.zig:1061-1072
    c = vxp.abi.default_config()
    assert (c.substeps, c.velocity_iterations, c.position_iterations) == (4, 1, 2)
    assert c.hertz == 30.0 and c.damping_ratio == 1.0
    assert c.warm_starting and c.enable_friction and c.enable_restitution


# -------------------------------------------------------------------- body.zig
def test_sleep_after_sixty_frames():
    # body.zig:570-586: a resting body sleeps within 60 frames of 1/60 s
    assert L.vxo_sleep_after(60, np.float32(1.0 / 60.0)) == 1
    assert L.vxo_sleep_after(29, np.float32(1.0 / 60.0)) == 0


# ------------------------------------------------------------------- islands.zig
def test_graph_colouring_basic():
    # islands.zig:818-846: a triangle of manifolds needs <= 3 colours and no
    # two manifolds sharing a body share a colour.
    ab = np.array([0, 1, 1, 2, 2, 0], dtype=np.uint32)
    col = np.zeros(3, dtype=np.uint8)
    n = L.vxo_graph_colouring(ab.ctypes.data, 3, col.ctypes.data)
    assert n <= 3
    assert len(set(col.tolist())) == 3


# --------------------------------------------------------------------- math.zig
def test_quat_90_degree_rotation():
    # math.zig:816-824
    q = np.zeros(4, dtype=np.float32)
    axis, v = f3(0, 0, 1), f3(1, 0, 0)
    L.vxo_from_axis_angle(axis.ctypes.data, np.float32(math.pi / 2.0), q.ctypes.data)
    out = np.zeros(3, dtype=np.float32)
    L.vxo_quat_rotate(q.ctypes.data, v.ctypes.data, out.ctypes.data)
    assert np.all(np.abs(out - f3(0, 1, 0)) <= 1e-6)


def test_mat3_inverse():
    # math.zig:835-846
    m = np.array([1, 2, 3, 0, 1, 4, 5, 6, 0], dtype=np.float32)
    inv = np.zeros(9, dtype=np.float32)
    L.vxo_mat3_inverse(m.ctypes.data, inv.ctypes.data)
    prod = m.reshape(3, 3).astype(np.float64) @ inv.reshape(3, 3).astype(np.float64)
    assert np.allclose(prod, np.eye(3), atol=1e-4)


def test_transform_round_trip():
    # math.zig:848-858
    q = np.zeros(4, dtype=np.float32)
    axis, p = f3(0, 1, 0), f3(1, 2, 3)
    L.vxo_from_axis_angle(axis.ctypes.data, np.float32(math.pi / 4.0), q.ctypes.data)
    pos = f3(10, 20, 30)
    w = np.zeros(3, dtype=np.float32)
    back = np.zeros(3, dtype=np.float32)
    L.vxo_transform_point(pos.ctypes.data, q.ctypes.data, p.ctypes.data, w.ctypes.data)
    L.vxo_inverse_transform_point(pos.ctypes.data, q.ctypes.data, w.ctypes.data, back.ctypes.data)
    assert np.all(np.abs(back - f3(1, 2, 3)) <= 1e-4)


def test_sin_cos_correctly_rounded():
    # @sin/@cos (math.zig:230-240): the oracle's f32 sin/cos is the double
    # value rounded once; compare with numpy's double sin rounded to f32.
    rng = np.random.default_rng(0)
    xs = np.concatenate([rng.uniform(-4, 4, 20000), rng.uniform(-0.5, 0.5, 20000),
                         rng.uniform(-300, 300, 5000)]).astype(np.float32)
    s = np.array([L.vxo_sinf(x) for x in xs], dtype=np.float32)
    c = np.array([L.vxo_cosf(x) for x in xs], dtype=np.float32)
    rs = np.sin(xs.astype(np.float64)).astype(np.float32)
    rc = np.cos(xs.astype(np.float64)).astype(np.float32)
    assert (s != rs).sum() <= 2 and (c != rc).sum() <= 2
    ulp = np.abs(s.view(np.int32).astype(np.int64) - rs.view(np.int32).astype(np.int64))
    assert ulp.max() <= 1
