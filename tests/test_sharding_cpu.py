"""Sharding of independent worlds (config 3) and served jobs (config 5) over
ranks, on the CPU: every world or job lands on exactly one rank, the
estimated cost is balanced, every rank computes the same assignment without
talking to the others, and a world's result does not depend on the rank
that steps it (gloo, world size 2, each rank stepping its share on the
oracle)."""
import os
import socket
import sys

import numpy as np
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TESTS = os.path.dirname(os.path.abspath(__file__))


def _sizes():
    import math
    rng = np.random.default_rng(3)
    return np.floor(np.exp(rng.uniform(math.log(8), math.log(2048), size=256))).astype(int)


def test_partition_covers_every_world_once_and_balances(vxp):
    sh = vxp.sharding
    costs = [sh.world_cost(int(n)) for n in _sizes()]
    for ranks in (1, 2, 4, 8):
        parts = sh.partition(costs, ranks)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        assert sh.imbalance(costs, parts) < 1.02, (ranks, sh.imbalance(costs, parts))
        assert parts == sh.partition(list(costs), ranks)  # deterministic


def test_partition_with_one_dominant_world(vxp):
    """A world costlier than all others together gets a rank to itself."""
    sh = vxp.sharding
    parts = sh.partition([100.0, 1.0, 1.0, 1.0, 1.0], 2)
    assert [0] in parts and sorted(i for p in parts for i in p) == [0, 1, 2, 3, 4]


def test_jobs_assigned_once_and_balanced(vxp):
    sh = vxp.sharding
    jobs = vxp.scenes.serving_jobs(300, seed=5)
    for ranks in (2, 8):
        r = sh.assign_jobs(jobs, ranks)
        assert len(r) == len(jobs) and set(r) <= set(range(ranks))
        load = np.zeros(ranks)
        for j, k in zip(jobs, r):
            load[k] += sh.job_cost(j["bodies"], j["steps"])
        assert load.max() / load.mean() < 1.25, load
        assert r == sh.assign_jobs(list(jobs), ranks)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _world_mix():
    import importlib
    sys.path.insert(0, ROOT)
    sys.path.insert(0, TESTS)
    import oracle_api as O
    vxp = importlib.import_module("zig-voxel-physics_b200")
    rng = np.random.default_rng(17)
    return vxp, O, [vxp.scenes.world_for_batch(rng, int(n), O.mass_fn, name=f"w{i}")
                    for i, n in enumerate([30, 9, 45, 12, 20, 60])]


def _step_alone(O, scene, steps):
    r = O.OracleWorld(substeps=4)
    r.load_scene(scene)
    for _ in range(steps):
        r.step(np.float32(scene.dt))
    out = r.get_bodies().tobytes()
    r.close()
    return out


def _rank(rank, world, port, out):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    vxp, O, scenes = _world_mix()
    parts = vxp.sharding.partition([vxp.sharding.world_cost(s.dynamic_count) for s in scenes], world)
    mine = {i: _step_alone(O, scenes[i], 25) for i in parts[rank]}
    got = [None] * world
    dist.all_gather_object(got, (parts, mine))  # the check only; stepping needed no exchange
    if rank == 0:
        out["parts"] = [g[0] for g in got]
        out["results"] = {i: b for g in got for i, b in g[1].items()}
        out["owners"] = {i: r for r, g in enumerate(got) for i in g[1]}
    dist.destroy_process_group()


def test_two_gloo_ranks_step_their_worlds_unchanged():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(300)
            assert p.exitcode == 0
        parts, results, owners = out["parts"], dict(out["results"]), dict(out["owners"])
    assert parts[0] == parts[1]  # both ranks computed the same partition
    vxp, O, scenes = _world_mix()
    assert sorted(owners) == list(range(len(scenes)))  # every world exactly once
    assert len(set(owners.values())) == 2
    for i, sc in enumerate(scenes):
        assert results[i] == _step_alone(O, sc, 25), f"world {i} differs when stepped on rank {owners[i]}"
