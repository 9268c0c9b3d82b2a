"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

Both sides get the same scene and, each step, the same pair list, and are
compared bit for bit: bodies (pose, velocities, sleep state), every manifold
(points, normals, depths, anchors, feature ids, impulses, masses, slot order)
and the narrow-phase / solver counters.  The two implementations use the same
colour-major sweep order and the same correctly rounded sin/cos, so the
tolerance is zero; the 1e-5 relative bound of the task is checked as well for
the record.
"""
import numpy as np
import pytest

import oracle_api as O

pytestmark = pytest.mark.gpu

STAT_KEYS = ("pairs_tested", "pairs_colliding", "voxels_checked", "contacts_generated", "pairs_skipped_sleeping",
             "cache_hits", "cache_misses", "cache_evictions", "manifolds", "constraints", "contact_points", "colours",
             "position_iterations_run", "step_skipped", "max_penetration", "candidates", "island_count",
             "active_islands", "sleeping_islands", "largest_island_size")


def _first_diff(g, r):
    if g.dtype.names:
        return [n for n in g.dtype.names if g[n].tobytes() != r[n].tobytes()]
    return ["raw"]


def lockstep(vxp, scene, steps, mode=-1, own_pairs=False, check_every=1, solver=None, cluster_smem=None,
             cluster_cons=None, probe_tables=None, **cfg):
    """Steps GPU and oracle together; returns the GPU system (open).
    solver: the grid solver mode (0 grid barriers, 1 event order, 2 cluster);
    cluster_smem: shared memory the cluster sweeps may use (0: state in L2);
    cluster_cons: 1 to build and colour the constraint table on the cluster too;
    probe_tables: False to probe without the neighbourhood-mask tables."""
    g = vxp.VoxelPhysicsSystem(**cfg)
    g.load_scene(scene)
    g.set_launch_mode(mode)
    if solver is not None:
        g.set_solver_mode(solver)
    if cluster_smem is not None:
        g.set_cluster_shared_bytes(cluster_smem)
    if cluster_cons is not None:
        g.set_cluster_constraints(bool(cluster_cons))
    if probe_tables is not None:
        g.set_probe_tables(bool(probe_tables))
    r = O.OracleWorld(**cfg)
    r.load_scene(scene)
    dt = np.float32(scene.dt)
    touching = 0
    for s in range(steps):
        pairs = r.pairs()
        if own_pairs:
            gp = g.pairs()
            assert gp.tobytes() == pairs.tobytes(), f"step {s}: device pair source differs"
            g.step(dt, None)
        else:
            g.step(dt, pairs)
        r.step(dt, pairs)
        touching += r.stats()["manifolds"] > 0
        if s % check_every and s != steps - 1:
            continue
        gm, rm = g.manifolds(), r.manifolds()
        assert len(gm) == len(rm), f"step {s}: {len(gm)} manifolds vs {len(rm)}"
        assert gm.tobytes() == rm.tobytes(), f"step {s}: manifolds differ in {_first_diff(gm, rm)}"
        gs, rs = g.stats(), r.stats()
        for k in STAT_KEYS:
            assert gs[k] == rs[k], f"step {s}: stats[{k}] gpu {gs[k]} oracle {rs[k]}"
        gb, rb = g.get_bodies(), r.get_bodies()
        assert gb.tobytes() == rb.tobytes(), f"step {s}: bodies differ in {_first_diff(gb, rb)}"
    r.close()
    # a run of 20 steps or more must have compared some contacts, not only free fall
    assert steps < 20 or touching >= 5, f"only {touching} of {steps} steps had a manifold"
    return g


@pytest.mark.parametrize("mode", [0, 1])
def test_islands_sleep_like_the_oracle(vxp, mode):
    """IslandManager statistics (system.zig:705-760) on the reference's
    example scene: islands appear when the box lands and one sleeps once the
    contact graph has not changed for 0.5 s; the lockstep compares every
    statistic each step, in block and grid launch."""
    sc = vxp.scenes.basic_example(O.mass_fn)
    g = lockstep(vxp, sc, 78, mode=mode)  # the body itself sleeps after step 78: later steps are skipped
    assert g.stats()["sleeping_islands"] >= 1
    g.close()


@pytest.mark.parametrize("mode", [0, 1])
def test_config1_trajectory_bit_exact(vxp, mode):
    """The 64-cube scene, 300 steps (the full run), block and grid launch."""
    sc = vxp.scenes.config1(mass_fn=O.mass_fn)
    lockstep(vxp, sc, 300 if mode == 0 else 120, mode=mode).close()


def test_pile_subset_device_pair_source_on_the_grid(vxp):
    """The grid step's own broad phase (its count pass tiled through shared
    memory, 512 boxes a tile: two tiles for the 514 bodies here) on 512 boxes
    of the pile: every step's results equal the oracle's on the oracle's pair
    list."""
    sc = vxp.scenes.config2(mass_fn=O.mass_fn, n_side=8, seed=2)
    lockstep(vxp, sc, 100, mode=1, own_pairs=True, check_every=10, substeps=8).close()


def test_config1_device_pair_source(vxp):
    sc = vxp.scenes.config1(mass_fn=O.mass_fn, seed=9)
    lockstep(vxp, sc, 150, own_pairs=True).close()


@pytest.mark.parametrize("cfg", [dict(colouring=1), dict(use_brick_pair_cache=0), dict(reference_caps=1),
                                 dict(enable_sleeping=0), dict(enable_warm_starting=0, warm_starting=0),
                                 dict(use_brick_sat=0), dict(velocity_iterations=2, position_iterations=4)])
def test_config1_modes(vxp, cfg):
    sc = vxp.scenes.config1(mass_fn=O.mass_fn, seed=3)
    lockstep(vxp, sc, 90, **cfg).close()


@pytest.mark.parametrize("solver,smem,cons", [(0, None, None), (1, None, None), (2, None, None), (2, 0, None),
                                              (2, 4096, None), (2, None, 1)])
def test_config2_pile_subset(vxp, solver, smem, cons):
    """216 boxes of the config-2 pile, 8 substeps at 1/120 s, grid launch,
    each grid solver mode (the cluster one with its state in shared memory,
    with 4 KiB of shared memory a CTA so that most constraint rows spill to
    global memory, and in L2; with the colouring on the cluster and on the
    grid).  The last step's stats say which sweep path ran."""
    sc = vxp.scenes.config2(mass_fn=O.mass_fn, n_side=6, seed=2)
    g = lockstep(vxp, sc, 200, mode=1, check_every=10, solver=solver, cluster_smem=smem, cluster_cons=cons,
                 substeps=8)
    want = {None: 1, 4096: 2, 0: 3}[smem] if solver == 2 else 0
    assert g.stats()["sweep_path"] == want
    g.close()


def test_cluster_available(vxp):
    """The B200 schedules a cluster for the sweeps (16 CTAs, or 8)."""
    g = vxp.VoxelPhysicsSystem()
    assert g.cluster_size() in (8, 16)
    g.close()


@pytest.mark.parametrize("solver", [0, 1, 2])
@pytest.mark.parametrize("cfg", [dict(), dict(colouring=1), dict(velocity_iterations=2, position_iterations=4),
                                 dict(enable_warm_starting=0, warm_starting=0)])
def test_config1_grid_solver_modes(vxp, solver, cfg):
    """The 64-cube scene on the grid with each solver mode."""
    sc = vxp.scenes.config1(mass_fn=O.mass_fn, seed=5)
    lockstep(vxp, sc, 90, mode=1, solver=solver, **cfg).close()


@pytest.mark.parametrize("mode", [0, 1])
def test_probes_without_tables(vxp, mode):
    """The narrow phase's 27 voxel lookups per probe centre (the path of
    colliders too large for a neighbourhood-mask table), on one CTA and on
    the grid, bit-exact against the oracle."""
    sc = vxp.scenes.config2(mass_fn=O.mass_fn, n_side=6, seed=3)
    lockstep(vxp, sc, 40, mode=mode, substeps=8, probe_tables=False).close()


def test_config4_noise_subset(vxp):
    """8 value-noise bodies (32^3 voxels) stacked with 10% overlap."""
    sc = vxp.scenes.config4(mass_fn=O.mass_fn, n_side=2, size=32, seed=4)
    lockstep(vxp, sc, 20, mode=1).close()


def test_candidate_set_bit_exact(vxp):
    """Every type-filter-passing voxel pair (A voxel, B voxel, distance^2,
    pass flag) of the narrow phase equals the oracle's, as a set."""
    sc = vxp.scenes.config1(mass_fn=O.mass_fn, seed=1)
    g = vxp.VoxelPhysicsSystem()
    g.load_scene(sc)
    g.set_candidate_dump(1 << 20)
    r = O.OracleWorld()
    r.load_scene(sc)
    r.set_candidate_dump(True)
    dt = np.float32(sc.dt)
    for s in range(40):
        pairs = r.pairs()
        g.step(dt, pairs)
        r.step(dt, pairs)
        gc, rc = g.candidates(), r.candidates()
        key = lambda c: np.lexsort([c["b"][:, 2], c["b"][:, 1], c["b"][:, 0], c["a"][:, 2], c["a"][:, 1],
                                    c["a"][:, 0], c["pair_index"]])
        gc, rc = gc[key(gc)], rc[key(rc)]
        assert len(gc) == len(rc), f"step {s}: {len(gc)} vs {len(rc)} candidates"
        assert gc.tobytes() == rc.tobytes(), f"step {s}: candidate sets differ"
    g.close()


def test_narrow_then_solve_split(vxp):
    """vxp_narrow_phase + vxp_solve equal narrowPhase() + solve() of the oracle."""
    sc = vxp.scenes.config1(mass_fn=O.mass_fn, n_side=3, seed=4)
    g = vxp.VoxelPhysicsSystem()
    g.load_scene(sc)
    r = O.OracleWorld()
    r.load_scene(sc)
    dt = np.float32(sc.dt)
    for s in range(30):
        pairs = r.pairs()
        g.narrow_phase(pairs)
        r.narrow_phase(pairs)
        assert g.manifolds().tobytes() == r.manifolds().tobytes(), f"step {s}: narrow phase"
        g.solve(dt)
        r.solve(dt)
        assert g.get_bodies().tobytes() == r.get_bodies().tobytes(), f"step {s}: solve"
    g.close()


# ----------------------------------------------------------------- edge cases
def test_empty_pair_list(vxp):
    sc = vxp.scenes.config1(mass_fn=O.mass_fn, n_side=2)
    g = lockstep(vxp, sc, 1)
    dt = np.float32(sc.dt)
    r = O.OracleWorld()
    r.load_scene(sc)
    r.step(dt, r.pairs())
    empty = np.zeros(0, dtype=vxp.abi.PAIR_DTYPE)
    g.step(dt, empty)
    r.step(dt, empty)
    assert g.get_bodies().tobytes() == r.get_bodies().tobytes()
    assert len(g.manifolds()) == 0
    g.close()


def test_all_sleeping_step_is_skipped(vxp):
    sc = vxp.scenes.config1(mass_fn=O.mass_fn, n_side=2)
    b = sc.bodies.copy()
    b["is_sleeping"] = 1
    sc.bodies = b
    g = lockstep(vxp, sc, 3)
    assert g.stats()["step_skipped"] == 1
    g.close()


def test_unknown_ids_and_missing_collider(vxp):
    """Pairs naming absent bodies are skipped; a body without a collider
    takes part in no contact (processPair returns early)."""
    sc = vxp.scenes.config1(mass_fn=O.mass_fn, n_side=2)
    b = sc.bodies.copy()
    b["collider_id"][2] = 77  # no such collider
    sc.bodies = b
    g = vxp.VoxelPhysicsSystem()
    g.load_scene(sc)
    r = O.OracleWorld()
    r.load_scene(sc)
    dt = np.float32(sc.dt)
    for s in range(10):
        pairs = r.pairs()
        extra = np.array([(900, 901), (1, 999)], dtype=vxp.abi.PAIR_DTYPE)
        pairs = np.concatenate([pairs, extra])
        g.step(dt, pairs)
        r.step(dt, pairs)
        assert g.get_bodies().tobytes() == r.get_bodies().tobytes()
        assert g.manifolds().tobytes() == r.manifolds().tobytes()
    g.close()


def test_kinematic_body(vxp):
    """A kinematic body moves with its own velocity and pushes dynamic ones."""
    sc = vxp.scenes.config1(mass_fn=O.mass_fn, n_side=2)
    b = sc.bodies.copy()
    b["body_type"][1] = vxp.abi.BODY_KINEMATIC
    b["inv_mass"][1] = 0.0
    b["inv_inertia_local"][1] = 0.0
    b["linear_velocity"][1] = (0.0, -2.0, 0.0)
    sc.bodies = b
    lockstep(vxp, sc, 60).close()


def test_pair_capacity_growth_keeps_warm_start(vxp):
    """A pair list larger than the initial device capacity grows the buffers
    between steps without losing the previous frame's manifolds."""
    sc = vxp.scenes.config1(mass_fn=O.mass_fn)
    g = vxp.VoxelPhysicsSystem(max_pairs=16)
    g.load_scene(sc)
    r = O.OracleWorld()
    r.load_scene(sc)
    dt = np.float32(sc.dt)
    for s in range(20):
        pairs = r.pairs()
        if s >= 10:  # pad with duplicates of absent ids to force growth
            pad = np.zeros(2000 * (s - 9), dtype=vxp.abi.PAIR_DTYPE)
            pad["body_a"] = 5000
            pad["body_b"] = 5001 + np.arange(len(pad))
            pairs = np.concatenate([pairs, pad])
        g.step(dt, pairs)
        r.step(dt, pairs)
        assert g.get_bodies().tobytes() == r.get_bodies().tobytes(), f"step {s}"
        assert g.manifolds().tobytes() == r.manifolds().tobytes(), f"step {s}"
    g.close()


def test_tolerance_bound_recorded(vxp):
    """The stated float tolerance (1e-5 relative on body state) holds trivially
    when the results are bit-identical; this records it on a short run."""
    sc = vxp.scenes.config1(mass_fn=O.mass_fn, n_side=2)
    g = lockstep(vxp, sc, 30)
    r = O.OracleWorld()
    r.load_scene(sc)
    dt = np.float32(sc.dt)
    for _ in range(30):
        r.step(dt, r.pairs())
    gb, rb = g.get_bodies(), r.get_bodies()
    for f in ("position", "rotation", "linear_velocity", "angular_velocity"):
        a, b = gb[f].astype(np.float64), rb[f].astype(np.float64)
        assert np.all(np.abs(a - b) <= 1e-5 * np.maximum(np.abs(b), 1e-3))
    g.close()


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("heavy", [0, 1, 200])
def test_heavy_pair_split_keeps_results(vxp, mode, heavy):
    """Pairs probed by a whole CTA (every pair at heavy=1, those with >= 200
    region voxels at heavy=200, none at 0) give the oracle's manifolds,
    counters and bodies bit for bit, and so does the candidate set."""
    sc = vxp.scenes.config1(mass_fn=O.mass_fn)
    g = vxp.VoxelPhysicsSystem(substeps=4)
    g.load_scene(sc)
    g.set_launch_mode(mode)
    g.set_heavy_pair_voxels(heavy)
    g.set_candidate_dump(1 << 20)
    r = O.OracleWorld(substeps=4)
    r.load_scene(sc)
    r.set_candidate_dump(True)
    dt = np.float32(sc.dt)
    key = lambda c: np.lexsort([c["b"][:, 2], c["b"][:, 1], c["b"][:, 0], c["a"][:, 2], c["a"][:, 1],
                                c["a"][:, 0], c["pair_index"]])
    for s in range(60):
        pairs = r.pairs()
        g.step(dt, pairs)
        r.step(dt, pairs)
        gm, rm = g.manifolds(), r.manifolds()
        assert gm.tobytes() == rm.tobytes(), f"step {s}: manifolds differ"
        gs, rs = g.stats(), r.stats()
        for k in STAT_KEYS:
            assert gs[k] == rs[k], f"step {s}: stats[{k}] gpu {gs[k]} oracle {rs[k]}"
        gc, rc = g.candidates(), r.candidates()
        gc, rc = gc[key(gc)], rc[key(rc)]
        assert gc.tobytes() == rc.tobytes(), f"step {s}: candidate sets differ"
        assert g.get_bodies().tobytes() == r.get_bodies().tobytes(), f"step {s}: bodies differ"
    g.close()
    r.close()


@pytest.mark.parametrize("heavy", [0, 1024])
def test_traffic_accounting_changes_only_the_brick_count(vxp, heavy):
    """With traffic accounting on, every step counts the bricks its probed
    pairs touch; the manifolds, counters and bodies stay those of the run
    without it (and the count reads 0 there)."""
    sc = vxp.scenes.config2(mass_fn=O.mass_fn, n_side=6, seed=2)
    runs = []
    for on in (False, True):
        g = vxp.VoxelPhysicsSystem(substeps=8)
        g.load_scene(sc)
        g.set_launch_mode(1)
        g.set_heavy_pair_voxels(heavy)
        g.set_traffic_accounting(on)
        dt = np.float32(sc.dt)
        rows = []
        for _ in range(40):
            g.step(dt)
            st = g.stats()
            rows.append((g.manifolds().tobytes(), g.get_bodies().tobytes(), st["bricks_touched"],
                         tuple(st[k] for k in STAT_KEYS)))
        runs.append(rows)
        g.close()
    for s, (off, on) in enumerate(zip(*runs)):
        assert off[0] == on[0] and off[1] == on[1] and off[3] == on[3], f"step {s}: results differ"
        assert off[2] == 0, f"step {s}: bricks counted with accounting off"
    assert sum(r[2] for r in runs[1]) > 0


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("cache", [32, 48, 64, 200])
def test_small_brick_pair_cache(vxp, mode, cache):
    """A brick-pair cache of a few dozen slots: nearly every lookup evicts and
    consecutive lookups' 16-slot windows often overlap, so the device replay
    of the lookups (in rounds of lookups whose windows are disjoint) is checked
    against the oracle's sequential one through the hit / miss / eviction
    counters and the manifolds, every step.  Tables this small compare the
    windows of the pending lookups pairwise (larger ones by table
    sixty-fourths)."""
    sc = vxp.scenes.config2(mass_fn=O.mass_fn, n_side=6, seed=2)
    lockstep(vxp, sc, 60, mode=mode, brick_pair_cache_size=cache, substeps=8).close()
