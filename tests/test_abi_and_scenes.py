"""CPU checks of the C ABI library (loads, exports what include/vxp.h
declares, struct layouts, host-side helpers) and of the scene builder."""
import ctypes
import os

import numpy as np
import pytest

import oracle_api as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_every_header_symbol(vxp):
    lib = vxp.abi.load()
    names = vxp.abi.declared_symbols(os.path.join(ROOT, "include", "vxp.h"))
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) <= set(vxp.abi.SIGNATURES), set(names) - set(vxp.abi.SIGNATURES)
    assert lib.vxp_abi_version() == 2


def test_config_default_matches_reference(vxp):
    lib = vxp.abi.load()
    c = vxp.abi.Config()
    lib.vxp_config_default(ctypes.byref(c))
    d = vxp.abi.default_config()
    assert bytes(c) == bytes(d)


def test_struct_sizes(vxp):
    a = vxp.abi
    assert a.BODY_DTYPE.itemsize == 128
    assert a.BRICK_DTYPE.itemsize == 524
    assert a.MANIFOLD_DTYPE.itemsize == 376
    assert a.CONTACT_DTYPE.itemsize == 88
    assert ctypes.sizeof(a.Config) == 4 * 27
    assert ctypes.sizeof(a.Stats) == 4 * 24


def test_classification_matches_reference(vxp):
    """classify_from_neighbors against the oracle's classifyFromNeighbors for
    every neighbour pattern (collision_voxel.zig:213-235)."""
    sc = vxp.scenes
    for m in range(64):
        solid = np.zeros((3, 3, 3), dtype=bool)
        solid[1, 1, 1] = True
        nb = {0: (0, 1, 1), 1: (2, 1, 1), 2: (1, 0, 1), 3: (1, 2, 1), 4: (1, 1, 0), 5: (1, 1, 2)}
        for bit, idx in nb.items():
            if not (m >> bit) & 1:  # bit set = neighbour empty
                solid[idx] = True
        got = int(sc.classify_from_neighbors(solid)[1, 1, 1])
        flags = [bool(solid[nb[b]]) for b in range(6)]
        want = O.L.vxo_classify_from_neighbors(1, *[int(f) for f in flags])
        assert got == want, (m, got, want)


def test_brick_hash_collisions_merge_like_reference(vxp):
    """hashBrickPos collides for (0,0,-3) and (-2,0,3): the second brick's
    voxels land in the first one, which keeps its position."""
    sc = vxp.scenes
    h = sc.hash_brick_pos([0, -2], [0, 0], [-3, 3])
    assert h[0] == h[1]
    coords = np.array([[0, 0, -24], [-16, 0, 24]])
    vals = np.array([sc.voxel_byte(1, 0), sc.voxel_byte(2, 5)])
    b = sc.bricks_from_calls(coords, vals)
    assert len(b) == 1
    assert tuple(b["pos"][0]) == (0, 0, -3)
    assert b["voxels"][0][0] == vals[1]  # cell (0,0,0) written last by the second call
    g = sc.example_ground(64)
    assert len(g) == 40  # 64 bricks fold into 40 hash-distinct bricks


def test_host_mass_properties_match_oracle(vxp):
    """vxp_mass_properties (host code of the library) equals the oracle's
    computeMassProperties bit for bit."""
    fn = vxp.scenes.default_mass_fn()
    rng = np.random.default_rng(7)
    cases = [(0.2, vxp.scenes.readme_box(8), 125.0), (0.1, vxp.scenes.solid_box(5, 11, 3), 1000.0)]
    for _ in range(3):
        cases.append((0.1, vxp.scenes.dense_to_bricks(vxp.scenes.classify_from_neighbors(
            vxp.scenes.value_noise_solid(rng, 16))), 1000.0))
    for vs, bricks, dens in cases:
        a = fn(vs, bricks, np.float32(dens))
        b = O.mass_fn(vs, bricks, np.float32(dens))
        assert a[0] == b[0]
        assert a[1].tobytes() == b[1].tobytes()


def test_scene_shapes(vxp):
    sc = vxp.scenes
    s1 = sc.config1(mass_fn=O.mass_fn)
    assert len(s1.bodies) == 65 and s1.dynamic_count == 64
    assert s1.bodies["id"][0] == 1 and s1.bodies["body_type"][0] == 0 and s1.bodies["is_sleeping"][0] == 1
    # 1 kg per voxel: 512 voxels
    assert abs(1.0 / s1.bodies["inv_mass"][1] - 512.0) < 1e-2
    s2 = sc.config2(mass_fn=O.mass_fn, n_side=3)
    assert s2.dynamic_count == 27 and len(s2.colliders) == 29
    jobs = sc.serving_jobs(50)
    assert all(16 <= j["bodies"] <= 4096 and 60 <= j["steps"] <= 600 for j in jobs)
    assert all(jobs[i]["arrival"] < jobs[i + 1]["arrival"] for i in range(49))


def test_scene_determinism(vxp):
    a = vxp.scenes.config1(mass_fn=O.mass_fn, seed=5)
    b = vxp.scenes.config1(mass_fn=O.mass_fn, seed=5)
    assert a.bodies.tobytes() == b.bodies.tobytes()


def test_product_package_has_no_oracle_imports():
    """The product neither imports, links nor includes anything under oracle/."""
    pkg = os.path.join(ROOT, "zig-voxel-physics_b200")
    banned = ("oracle_api", "liboracle", "vxp_oracle", "import oracle", "from oracle", "oracle_capi")
    for dirpath, _, files in os.walk(pkg):
        for f in files:
            if f.endswith((".py", ".cu", ".cuh", ".h", ".cpp")):
                src = open(os.path.join(dirpath, f)).read()
                assert not any(b in src for b in banned), f


def test_tuning_setters_reject_a_null_context(vxp):
    """Every tuning setter checks its context before touching the device, so
    a null context is an argument error on any machine."""
    lib = vxp.abi.load()
    calls = {
        "vxp_set_candidate_dump": (0,),
        "vxp_set_traffic_accounting": (1,),
        "vxp_set_cluster_constraints": (1,),
        "vxp_set_cluster_shared_bytes": (0,),
        "vxp_set_launch_mode": (0,),
        "vxp_set_solver_blocks_divisor": (128,),
        "vxp_set_heavy_pair_voxels": (768,),
        "vxp_set_wait_limit_ns": (0,),
        "vxp_set_probe_tables": (0,),
        "vxp_set_solver_mode": (0,),
        "vxp_synchronize": (),
    }
    for name, args in calls.items():
        assert getattr(lib, name)(None, *args) == vxp.abi.VXP_ERR_ARG, name
    n = ctypes.c_uint32(7)
    assert lib.vxp_cluster_size(None, ctypes.byref(n)) == vxp.abi.VXP_ERR_ARG
