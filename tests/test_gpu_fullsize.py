"""Parity at the benchmark sizes, through the C ABI, bit for bit with the
sequential CPU oracle (the reference's own order of work).

* The 4096-box pile (config 2): the device steps it 360 steps to the state
  the benchmark times; a fresh context and a fresh oracle then start from
  those bodies and step 5 steps together: bodies, every manifold and the
  narrow-phase / solver counters compared after each.
* The narrow-phase stress scene at full size (config 4: 512 bodies of 64^3
  voxels, 10 % overlap): 2 steps from the start, ~2.6e8 voxel probes a step,
  with the neighbourhood-mask tables and with the 27-lookup path.
* The 256-world batch (config 3): all 256 worlds in one batch for the
  configuration's 300 steps; the three largest worlds (>= 1024 bodies each,
  9 columns of boxes whose lower layers have landed by then) equal the oracle
  stepping each of them alone.
"""
import numpy as np
import pytest

import oracle_api as O
from test_gpu_parity import STAT_KEYS, _first_diff

pytestmark = pytest.mark.gpu


def _compare(g, r, s):
    gm, rm = g.manifolds(), r.manifolds()
    assert len(gm) == len(rm), f"step {s}: {len(gm)} manifolds vs {len(rm)}"
    assert gm.tobytes() == rm.tobytes(), f"step {s}: manifolds differ in {_first_diff(gm, rm)}"
    gs, rs = g.stats(), r.stats()
    for k in STAT_KEYS:
        assert gs[k] == rs[k], f"step {s}: stats[{k}] gpu {gs[k]} oracle {rs[k]}"
    gb, rb = g.get_bodies(), r.get_bodies()
    assert gb.tobytes() == rb.tobytes(), f"step {s}: bodies differ in {_first_diff(gb, rb)}"
    return rs


def test_full_pile_from_the_benchmarked_state(vxp):
    sc = vxp.scenes.config2(mass_fn=O.mass_fn)
    cfg = dict(substeps=8, fixed_timestep=np.float32(1.0 / 120.0), reference_caps=0)
    dt = np.float32(sc.dt)
    g = vxp.VoxelPhysicsSystem(max_pairs=65536, max_bodies=len(sc.bodies), **cfg)
    g.load_scene(sc)
    for i in range(360):
        g.step(dt)
        if i % 32 == 31:
            g.synchronize()
    settled = g.get_bodies()
    g.close()

    g = vxp.VoxelPhysicsSystem(max_pairs=65536, max_bodies=len(sc.bodies), **cfg)
    g.load_scene(sc)
    g.set_bodies(settled)
    r = O.OracleWorld(**cfg)
    r.load_scene(sc)
    r.set_bodies(settled)
    points = []
    for s in range(5):
        pairs = r.pairs()
        g.step(dt, pairs)
        r.step(dt, pairs)
        points.append(_compare(g, r, s)["contact_points"])
        # the sweeps keep their state on the cluster (rows that do not fit
        # in shared memory spill to global memory), never the all-L2 path
        assert g.stats()["sweep_path"] in (1, 2)
    g.close()
    r.close()
    assert min(points) > 10000, points  # a settled pile, not a free fall


def test_stress_scene_full_size(vxp):
    """Both probe paths at full size: one context builds the neighbourhood-mask
    tables (2.4 GB for the 512 colliders), the other probes with 27 voxel
    lookups per centre; each equals the oracle."""
    sc = vxp.scenes.config4(mass_fn=O.mass_fn)
    cfg = dict(substeps=4, reference_caps=0)
    dt = np.float32(sc.dt)
    gs = []
    for tables in (True, False):
        g = vxp.VoxelPhysicsSystem(**cfg)
        g.set_probe_tables(tables)
        g.load_scene(sc)
        gs.append(g)
    r = O.OracleWorld(**cfg)
    r.load_scene(sc)
    probes = []
    for s in range(2):
        pairs = r.pairs()
        for g in gs:
            g.step(dt, pairs)
        r.step(dt, pairs)
        for g in gs:
            probes.append(_compare(g, r, s)["voxels_checked"])
    for g in gs:
        g.close()
    r.close()
    assert min(probes) > 10 ** 8, probes


def test_largest_batched_worlds_equal_the_oracle(vxp):
    scenes = vxp.scenes.config3(mass_fn=O.mass_fn)
    dt = np.float32(1.0 / 60.0)
    steps = 300
    b = vxp.VoxelWorldBatch(len(scenes), substeps=4)
    off = []
    o = 0
    for i, sc in enumerate(scenes):
        b.load_scene(i, sc, collider_offset=o)
        off.append(o)
        o += len(sc.colliders) + 1
    b.step(dt, steps)
    b.synchronize()
    big = sorted(range(len(scenes)), key=lambda i: -scenes[i].dynamic_count)[:3]
    assert min(scenes[i].dynamic_count for i in big) >= 1024
    for i in big:
        got = b.get_world(i)
        got["collider_id"] -= off[i]
        r = O.OracleWorld(substeps=4)
        r.load_scene(scenes[i])
        for _ in range(steps):
            r.step(dt)
        want = r.get_bodies()
        assert r.stats()["contact_points"] > 1000
        r.close()
        assert got.tobytes() == want.tobytes(), f"world {i} ({scenes[i].dynamic_count} bodies) differs"
    b.close()
