"""Batched worlds: each world of a batch must give exactly the results of the
same world stepped alone (single-world context, and the CPU oracle), under
any schedule, with worlds joining and leaving between steps."""
import numpy as np
import pytest

import oracle_api as O

pytestmark = pytest.mark.gpu


def small_mix(vxp, sizes, seed=7):
    rng = np.random.default_rng(seed)
    return [vxp.scenes.world_for_batch(rng, int(n), O.mass_fn, name=f"w{i}") for i, n in enumerate(sizes)]


def run_alone(vxp, scene, steps, dt):
    s = vxp.VoxelPhysicsSystem(substeps=4)
    s.load_scene(scene)
    for _ in range(steps):
        s.step(dt)
    out = s.get_bodies()
    s.close()
    return out


def run_oracle(scene, steps, dt):
    r = O.OracleWorld(substeps=4)
    r.load_scene(scene)
    for _ in range(steps):
        r.step(dt)
    out = r.get_bodies()
    r.close()
    return out


ISLAND_KEYS = ("island_count", "active_islands", "sleeping_islands", "largest_island_size")


def test_batch_world_islands_equal_the_oracle(vxp):
    """The island pass runs in every batch world (one CTA): after each of 200
    steps every world's IslandManager statistics equal the oracle's for that
    world alone.  Islands of the 12-box world sleep from step ~183, those of
    the reference's example scene from step 76 (its box sleeps soon after and
    every later step is skipped)."""
    scenes = small_mix(vxp, [12, 40, 25], seed=21) + [vxp.scenes.basic_example(O.mass_fn)]
    dt = np.float32(1.0 / 60.0)
    b = vxp.VoxelWorldBatch(len(scenes), substeps=4)
    rs = []
    for i, sc in enumerate(scenes):
        b.load_scene(i, sc, collider_offset=1000 * (i + 1))
        r = O.OracleWorld(substeps=4)
        r.load_scene(sc)
        rs.append(r)
    slept = 0
    for s in range(200):
        b.step(dt)
        b.synchronize()
        for i, r in enumerate(rs):
            r.step(dt)
            got, want = b.world_stats(i), r.stats()
            assert {k: got[k] for k in ISLAND_KEYS} == {k: want[k] for k in ISLAND_KEYS}, (s, i)
            slept += want["sleeping_islands"]
    for r in rs:
        r.close()
    b.close()
    assert slept > 0


def test_batch_equals_alone_and_oracle(vxp):
    scenes = small_mix(vxp, [8, 30, 90, 17, 60])
    dt = np.float32(1.0 / 60.0)
    b = vxp.VoxelWorldBatch(len(scenes), substeps=4)
    for i, sc in enumerate(scenes):
        b.load_scene(i, sc, collider_offset=10000 * (i + 1))
    steps = 80
    b.step(dt, steps)
    b.synchronize()
    for i, sc in enumerate(scenes):
        got = b.get_world(i)
        alone = run_alone(vxp, sc, steps, dt)
        got_cmp = got.copy()
        got_cmp["collider_id"] -= 10000 * (i + 1)
        assert got_cmp.tobytes() == alone.tobytes(), f"world {i} differs from the same world alone"
        if i < 3:
            ref = run_oracle(sc, steps, dt)
            assert got_cmp.tobytes() == ref.tobytes(), f"world {i} differs from the oracle"
    b.close()


@pytest.mark.parametrize("threads,order", [(256, 0), (256, 1), (512, 0), (512, 1), ("tiles", 30), ("tiles", 50)])
def test_schedule_does_not_change_results(vxp, threads, order):
    """Every schedule, per-world tiles included (order = the body count from
    which a world steps as a 512-thread CTA), gives each world its results
    alone."""
    scenes = small_mix(vxp, [40, 12, 70], seed=8)
    dt = np.float32(1.0 / 60.0)
    b = vxp.VoxelWorldBatch(3, substeps=4)
    for i, sc in enumerate(scenes):
        b.load_scene(i, sc, collider_offset=1000 * (i + 1))
    if threads == "tiles":
        b.set_tiles(order)
    else:
        b.set_schedule(threads, order)
    b.step(dt, 40)
    b.synchronize()
    for i, sc in enumerate(scenes):
        got = b.get_world(i)
        got["collider_id"] -= 1000 * (i + 1)
        assert got.tobytes() == run_alone(vxp, sc, 40, dt).tobytes()
    b.close()


def test_autotune_keeps_results(vxp):
    scenes = small_mix(vxp, [50, 20, 8, 35], seed=9)
    dt = np.float32(1.0 / 60.0)
    b = vxp.VoxelWorldBatch(4, substeps=4)
    for i, sc in enumerate(scenes):
        b.load_scene(i, sc, collider_offset=1000 * (i + 1))
    choice, ms = b.autotune(dt, trial_steps=2)  # every schedule: 1 + 2 real steps
    assert 0 <= choice < vxp.abi.BATCH_SCHEDULES and len(ms) == vxp.abi.BATCH_SCHEDULES and np.all(ms > 0)
    b.step(dt, 8)
    b.synchronize()
    steps = vxp.abi.BATCH_SCHEDULES * 3 + 8
    for i, sc in enumerate(scenes):
        got = b.get_world(i)
        got["collider_id"] -= 1000 * (i + 1)
        assert got.tobytes() == run_alone(vxp, sc, steps, dt).tobytes()
    b.close()


def test_worlds_join_and_leave(vxp):
    """Continuous batching: a slot is emptied and refilled between steps; the
    new world's result equals the world alone, the others are undisturbed."""
    scenes = small_mix(vxp, [25, 40, 15, 33], seed=10)
    dt = np.float32(1.0 / 60.0)
    b = vxp.VoxelWorldBatch(3, substeps=4)
    for i in range(3):
        b.load_scene(i, scenes[i], collider_offset=1000 * (i + 1))
    b.step(dt, 20)
    b.synchronize()
    b.clear_world(1)
    b.step(dt, 10)  # slot 1 empty
    b.load_scene(1, scenes[3], collider_offset=5000)
    b.step(dt, 30)
    b.synchronize()
    got0 = b.get_world(0)
    got0["collider_id"] -= 1000
    assert got0.tobytes() == run_alone(vxp, scenes[0], 60, dt).tobytes()
    got1 = b.get_world(1)
    got1["collider_id"] -= 5000
    assert got1.tobytes() == run_alone(vxp, scenes[3], 30, dt).tobytes()
    b.close()


def test_reused_slot_matches_new_slot(vxp):
    """A cleared slot keeps its device buffers: a small world set into a slot
    that held a larger one (larger pair and body capacities, a used contact
    manager and cache) steps exactly as the small world alone; so does one
    set after the slot's memory was released."""
    scenes = small_mix(vxp, [120, 20, 30], seed=11)
    dt = np.float32(1.0 / 60.0)
    b = vxp.VoxelWorldBatch(1, substeps=4)
    b.load_scene(0, scenes[0], collider_offset=1000)
    b.step(dt, 15)
    b.synchronize()
    held = b.world_bytes(0)
    b.clear_world(0)
    assert b.world_bytes(0) == held
    b.load_scene(0, scenes[1], collider_offset=3000)
    assert b.world_bytes(0) == held
    b.step(dt, 25)
    b.synchronize()
    got = b.get_world(0)
    got["collider_id"] -= 3000
    assert got.tobytes() == run_alone(vxp, scenes[1], 25, dt).tobytes()
    b.release_world(0)
    assert b.world_bytes(0) == 0
    b.load_scene(0, scenes[2], collider_offset=5000)
    b.step(dt, 10)
    b.synchronize()
    got = b.get_world(0)
    got["collider_id"] -= 5000
    assert got.tobytes() == run_alone(vxp, scenes[2], 10, dt).tobytes()
    b.close()
