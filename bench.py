#!/usr/bin/env python
"""Benchmark: body-substeps/s of the voxel contact + TGS-soft step on B200.

Workload (N=1): the 4096-body pile (seeded random boxes, per-axis extents
2..16 voxels at 0.1 m, dropped from a 16^3 lattice into a walled bin on a
ground slab; dt 1/120, 8 substeps).  The scene is first advanced `--settle`
steps (default 360: the lower layers have landed and the pile holds ~2x10^4
contact points), then `--warmup` steps, then `--steps` timed steps.  A "step"
is one VoxelPhysicsSystem.step: the device pair source, the narrow phase and
the solver with its 8 substeps.

value: device time (CUDA events on the library's stream) of each step with
its inputs resident; the L2 is flushed (a 256 MiB write) between timed steps.
e2e: the same steps through the public C ABI with host buffers in pinned
memory: every step copies the pair list host->device (vxp_step) and reads the
pair list and the body table back (vxp_pairs_from_bodies, vxp_bodies_get),
timed by the host clock.

The pile's line also carries compact runs of the batched and served
comparisons, on the same box: "batched" (the 256-world mix under the
autotuned schedule against the plain single-world path, 10 timed steps) and
"serving" (150 Poisson-arriving jobs through the continuous-batching server,
step and job latency percentiles); --no-extras leaves them out.

--workload stress: the narrow-phase stress scene (512 bodies of 64^3 voxels
filled by value noise, 10 % overlap in a walled bin; dt 1/60, 4 substeps),
timed from its first step; the same value / roofline / e2e / CPU baseline.
--workload batched / serving: the full versions of the two summaries.

--impl reference times the reference's CPU path (the CPU restatement of the
reference, with its thread-pooled narrow phase on every host core and the
single-threaded solver) on the same scene (pile or stress).

Multi-GPU: a single world does not shard; N ranks run N independent replicas
("replicas only", weak scaling) and value is the sum of their work over the
slowest rank's time.
"""
from __future__ import annotations

import argparse
import ctypes
import importlib
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

L2_FLUSH_BYTES = 256 << 20
SOLVER_V, SOLVER_Q = 1, 2


# DRAM bytes (read + write) per launch of each step kernel, keyed by
# (workload, kernel), from one ncu capture of the same workload (the pile's
# state after 360 steps; the stress scene's first steps): the bytes, the
# profile file that summarises the capture, and the commit whose kernel was
# captured; to be captured again whenever a kernel changes.  The bench line
# carries the commit next to the figure.
_PILE_PROFILE = "profiles/k_step_grid_k_solve_grid_k_solve_cluster_config2_pile.md"
PROFILED_TRAFFIC = {
    ("config2_pile_4096", "k_step_grid"): (54_253_312, _PILE_PROFILE, "d08c536"),
    ("config2_pile_4096", "k_solve_grid"): (7_303_680, _PILE_PROFILE, "d08c536"),
    ("config2_pile_4096", "k_solve_cluster"): (4_125_184, _PILE_PROFILE, "8a7312f"),
    ("config4_stress_512", "k_step_grid"): (755_527_680, "profiles/k_step_grid_config4_stress.md", "d08c536"),
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--settle", type=int, default=360)
    ap.add_argument("--n-side", type=int, default=16)
    ap.add_argument("--cpu-sample-s", type=float, default=12.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--launch-mode", type=int, default=-1)
    ap.add_argument("--solver", type=int, default=-1, help="grid solver mode (-1: the library default)")
    ap.add_argument("--workload", default="pile", choices=["pile", "small", "stress", "batched", "serving"],
                    help="pile: the 4096-body pile (the headline); small: the 64 cubes of config 1 (100 steps "
                         "in); stress: 512 bodies of 64^3 voxels (narrow-phase stress); "
                         "batched: 256 independent worlds; "
                         "serving: Poisson-arriving jobs through the continuous-batching server")
    ap.add_argument("--no-extras", action="store_true",
                    help="pile only: skip the batched and serving summaries the pile line carries")
    ap.add_argument("--jobs", type=int, default=300)
    ap.add_argument("--state-out", default=None, help="save the body table after settling (npy)")
    ap.add_argument("--state-in", default=None, help="start from a saved body table instead of settling")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--slots", type=int, default=512)
    ap.add_argument("--worlds", type=int, default=256)
    ap.add_argument("--batch-settle", type=int, default=150,
                    help="batched: untimed steps before the autotuner and the timed steps (mid-run state)")
    return ap.parse_args()


# --------------------------------------------------------------------------
def dist_setup(args):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if ws > 1:
        import datetime

        import torch
        import torch.distributed as dist

        backend = "nccl" if args.impl == "ours" else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
        pg = dist
    return ws, rank, local, pg


def max_over_ranks(pg, x: float, device: str) -> float:
    """The largest x over all ranks (the job's time is its slowest rank's);
    x itself without a process group."""
    if not pg:
        return float(x)
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


class Clocks:
    """nvidia-smi clock / throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() in ("active", "1"):
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def alg_bytes(st: dict, substeps: int, n_dyn_awake: int, n_nonstatic: int) -> tuple:
    """Algorithmic bytes of one step (stats of that step; bricks_touched from
    a replay of it with traffic accounting on), counting each f32 or byte field the
    reference reads or writes once per operation: narrow phase per pair
    2x28 + 2x8, per brick touched 512, per contact 60, per manifold 16;
    solver per contact point prepare 308 x S, velocity sweep 316 x V x S,
    relax 316 x S, warm start 248, position sweep 232 x Q, storeImpulses 20;
    per dynamic body gravity + integrate 208 x S, write-back 104."""
    narrow = st["pairs_tested"] * 72 + st["bricks_touched"] * 512 + st["contacts_generated"] * 60 + st["manifolds"] * 16
    pts = st["contact_points"]
    solver = pts * (308 * substeps + 316 * SOLVER_V * substeps + 316 * substeps + 248 +
                    232 * max(1, st["position_iterations_run"]) + 20)
    solver += n_dyn_awake * 208 * substeps + n_nonstatic * 104
    return narrow, solver


def peaks() -> tuple:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# --------------------------------------------------------------------------
def single_world_workload(vxp, args, mass_fn=None):
    """(scene, substeps, settle steps, workload name) of a single-world run:
    the 4096-box pile (config 2, 8 substeps at dt 1/120, settled before the
    timed steps), the 64 cubes (config 1, 4 substeps at dt 1/60, from step
    100) or the narrow-phase stress scene (config 4, 4 substeps at dt 1/60,
    timed from its start)."""
    if args.workload == "stress":
        scene = vxp.scenes.config4(mass_fn=mass_fn)
        return scene, 4, 0, f"config4_stress_{scene.dynamic_count}"
    if args.workload == "small":
        scene = vxp.scenes.config1(mass_fn=mass_fn)
        return scene, 4, 100, f"config1_small_{scene.dynamic_count}"
    scene = vxp.scenes.config2(mass_fn=mass_fn, n_side=args.n_side)
    return scene, 8, args.settle, f"config2_pile_{scene.dynamic_count}"


def run_cpu(scene, oracle, args, body_state=None, steps=None, budget_s=None, threads=None, substeps=8):
    """Times the reference's CPU step (threaded narrow phase on every host core,
    single-threaded solver).  Returns (body_substeps_per_s, steps_timed, threads, per-step s)."""
    threads = threads or os.cpu_count() or 1
    w = oracle.OracleWorld(substeps=substeps, fixed_timestep=np.float32(scene.dt), reference_caps=0)
    w.load_scene(scene)
    if body_state is not None:
        w.set_bodies(body_state)
    dt = np.float32(scene.dt)
    n_dyn = scene.dynamic_count
    times = []
    t_start = time.perf_counter()
    k = 0
    while True:
        pairs = w.pairs()
        t0 = time.perf_counter()
        w.step_threaded(dt, pairs, threads)
        times.append(time.perf_counter() - t0)
        k += 1
        if steps is not None and k >= steps:
            break
        if budget_s is not None and time.perf_counter() - t_start > budget_s and k >= 2:
            break
    w.close()
    return n_dyn * substeps * k / sum(times), k, threads, times


def reference_arm(args):
    ws, rank, local, pg = dist_setup(args)
    if rank != 0:
        if pg:
            pg.destroy_process_group()
        return 0
    vxp = importlib.import_module("zig-voxel-physics_b200")
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_api

    scene, substeps, settle, workload = single_world_workload(vxp, args, oracle_api.mass_fn)
    threads = os.cpu_count() or 1
    w = oracle_api.OracleWorld(substeps=substeps, fixed_timestep=np.float32(scene.dt), reference_caps=0)
    w.load_scene(scene)
    dt = np.float32(scene.dt)
    for _ in range(settle + args.warmup):
        w.step_threaded(dt, w.pairs(), threads)
    times = []
    for _ in range(args.steps):
        pairs = w.pairs()
        t0 = time.perf_counter()
        w.step_threaded(dt, pairs, threads)
        times.append(time.perf_counter() - t0)
    n_dyn = scene.dynamic_count
    value = n_dyn * substeps * len(times) / sum(times)
    line = {
        "impl": "reference", "metric": "body_substeps_per_s", "value": value, "unit": "body-substeps/s",
        "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": workload, "bodies": n_dyn, "substeps": substeps,
                   "dt": "1/120" if substeps == 8 else "1/60", "settle_steps": settle},
        "cpu_baseline": {"value": value, "unit": "body-substeps/s", "cores": threads, "kind": "port",
                         "sample": f"{len(times)} steps after {settle + args.warmup} settle/warm-up steps; "
                                   "threaded narrow phase (reference partitioning) + single-threaded solver"},
        "e2e": {"value": value, "unit": "body-substeps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------------------------
def ours(args):
    ws, rank, local, pg = dist_setup(args)
    import torch

    torch.cuda.set_device(local)
    vxp = importlib.import_module("zig-voxel-physics_b200")
    abi = vxp.abi
    scene, substeps, settle, workload = single_world_workload(vxp, args)
    n_dyn = scene.dynamic_count
    n_nonstatic = int((scene.bodies["body_type"] != abi.BODY_STATIC).sum())
    sysm = vxp.VoxelPhysicsSystem(device=local, substeps=substeps, fixed_timestep=np.float32(scene.dt),
                                  reference_caps=0, max_pairs=max(1024, 16 * n_dyn), max_bodies=len(scene.bodies))
    sysm.load_scene(scene)
    sysm.set_launch_mode(args.launch_mode)
    if args.solver >= 0:
        sysm.set_solver_mode(args.solver)
    dt = np.float32(scene.dt)
    if args.state_in:
        sysm.set_bodies(np.load(args.state_in))
    else:
        for i in range(settle):
            sysm.step(dt)
            if i % 32 == 31:
                sysm.synchronize()
    sysm.synchronize()
    if args.state_out:
        np.save(args.state_out, sysm.get_bodies())
    for _ in range(args.warmup):
        sysm.step(dt)
        sysm.synchronize()
    # the e2e loop below replays the same steps from this state
    start_state = sysm.get_bodies()
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=f"cuda:{local}")
    clocks = Clocks(local)
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    clocks.start()
    step_ms, kern_ms, pair_ms, stats, part_ms, split_ms = [], [], [], [], [], []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        sysm.step(dt)
        out = np.zeros(3, dtype=np.float32)
        sysm._check(sysm.lib.vxp_last_step_ms(sysm.ctx, abi.ptr(out)))
        pair_ms.append(float(out[0]))
        kern_ms.append(float(out[1]))
        step_ms.append(float(out[2]))
        parts = np.zeros(2, dtype=np.float32)
        sysm._check(sysm.lib.vxp_last_kernel_ms(sysm.ctx, abi.ptr(parts)))
        part_ms.append((float(parts[0]), float(parts[1])))
        split = np.zeros(2, dtype=np.float32)
        sysm._check(sysm.lib.vxp_last_solve_split_ms(sysm.ctx, abi.ptr(split)))
        split_ms.append((float(split[0]), float(split[1])))
        stats.append(sysm.stats())
    torch.cuda.synchronize()
    clk = clocks.stop()
    total_s = sum(step_ms) / 1e3
    total_s = max_over_ranks(pg, total_s, f"cuda:{local}")
    value = ws * n_dyn * substeps * args.steps / total_s
    pts = [s["contact_points"] for s in stats]
    contacts_per_s = ws * sum(pts) * substeps / total_s
    bodies = sysm.get_bodies()
    n_dyn_awake = int(((bodies["body_type"] == abi.BODY_DYNAMIC) & (bodies["is_sleeping"] == 0)).sum())
    # the bricks each step's probed pairs touch (the narrow phase's per-brick
    # bytes) are counted on an untimed replay of the same steps: counting
    # them costs narrow-phase time and is no part of the step
    sysm.set_bodies(start_state)
    sysm.set_traffic_accounting(True)
    for st in stats:
        sysm.step(dt)
        st["bricks_touched"] = sysm.stats()["bricks_touched"]
    sysm.set_traffic_accounting(False)
    nb = [sum(alg_bytes(s, substeps, n_dyn_awake, n_nonstatic)) for s in stats]
    peak, peak_kind = peaks()
    achieved = sum(nb) / (sum(kern_ms) / 1e3) / 1e9
    # per kernel of the step, each its algorithmic bytes over its own event
    # time: narrow part (k_step_grid), then the solve part: one grid kernel
    # (k_solve_grid), or the cluster kernel (k_solve_cluster: the solver's
    # bytes), after the grid's constraint table and colouring when those do
    # not run on the cluster (k_solve_grid: no per-unit byte count, time only)
    nb_parts = [alg_bytes(s, substeps, n_dyn_awake, n_nonstatic) for s in stats]
    grid = n_dyn >= 512
    cluster = grid and all(x[1] > 0.0 for x in split_ms)
    kernels = {}
    if grid:
        names = [("k_step_grid", [x[0] for x in part_ms], [x[0] for x in nb_parts])]
        if cluster:
            if statistics.mean(x[0] for x in split_ms) > 0.005:
                names += [("k_solve_grid", [x[0] for x in split_ms], None)]
            names += [("k_solve_cluster", [x[1] for x in split_ms], [x[1] for x in nb_parts])]
        else:
            names += [("k_solve_grid", [x[1] for x in part_ms], [x[1] for x in nb_parts])]
        for name, tl, bl in names:
            t = sum(tl) / 1e3
            kernels[name] = {"ms_mean": 1e3 * t / len(tl)}
            if bl is None:
                kernels[name].update({"alg_bytes_per_launch": None, "achieved": None, "frac": None})
            else:
                b = sum(bl)
                kernels[name].update({"alg_bytes_per_launch": b / len(bl), "achieved": b / t / 1e9,
                                      "frac": b / t / 1e9 / peak})
        dominant = max((k for k in kernels if kernels[k]["achieved"] is not None), key=lambda k: kernels[k]["ms_mean"])
    else:
        dominant = "k_step_block"
        kernels[dominant] = {"ms_mean": statistics.mean(kern_ms), "alg_bytes_per_launch": statistics.mean(nb),
                             "achieved": achieved, "frac": achieved / peak}

    # ---- e2e through the public API with pinned host buffers
    cap = max(1024, 16 * n_dyn)
    pin_pairs = torch.empty(cap * 8, dtype=torch.uint8).pin_memory().numpy().view(abi.PAIR_DTYPE)
    pin_bodies = torch.empty(len(scene.bodies) * 128, dtype=torch.uint8).pin_memory().numpy().view(abi.BODY_DTYPE)
    h2d = d2h = 0

    def e2e_step():
        n = ctypes.c_uint32(0)
        sysm._check(sysm.lib.vxp_pairs_from_bodies(sysm.ctx, np.float32(sysm.pair_margin), abi.ptr(pin_pairs), cap,
                                                    ctypes.byref(n)))
        sysm._check(sysm.lib.vxp_step(sysm.ctx, dt, abi.ptr(pin_pairs), n.value))
        sysm._check(sysm.lib.vxp_bodies_get(sysm.ctx, abi.ptr(pin_bodies), len(pin_bodies)))
        return n.value

    # untimed warm-up of this path too (first launches of the pair-source
    # kernels load their code, its buffers are allocated once); then the
    # timed loop steps the same bodies as the device-timed loop (the pile is
    # still settling: every step adds pairs)
    if not args.no_e2e:
        sysm.set_bodies(start_state)
        for _ in range(args.warmup):
            e2e_step()
        sysm.set_bodies(start_state)
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(0 if args.no_e2e else args.steps):
        n = e2e_step()
        h2d += 8 * n
        d2h += 8 * n + 128 * len(pin_bodies)
    e2e_s = max(time.perf_counter() - t0, 1e-9)
    e2e_s = max_over_ranks(pg, e2e_s, f"cuda:{local}")
    e2e_value = None if args.no_e2e else ws * n_dyn * substeps * args.steps / e2e_s

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import oracle_api

        state = sysm.get_bodies()
        v, k, threads, _ = run_cpu(scene, oracle_api, args, body_state=state, budget_s=args.cpu_sample_s,
                                   substeps=substeps)
        cpu = {"value": v, "unit": "body-substeps/s", "cores": threads, "kind": "port",
               "sample": f"{k} steps of the same scene from the GPU's state after {settle + args.warmup + args.steps} "
                         "steps; threaded narrow phase (reference partitioning) + single-threaded solver"}
    sysm.close()
    extras = {}
    if rank == 0 and ws == 1 and args.workload == "pile" and not args.no_extras:
        # the batched and served comparisons, measured on the same box in the same run
        # (compact versions of --workload batched / serving)
        bl = batched(args, steps=10, warmup=3, emit=False)
        extras["batched"] = {k: bl[k] for k in ("value", "unit", "ms_per_step", "plain_single_world",
                                                "batched_over_plain", "world_step_latency_ms", "clocks")}
        extras["batched"]["config"] = bl["config"]
        sl = serving(args, jobs=150, emit=False)
        so = sl["serving"]
        extras["serving"] = {"value": sl["value"], "unit": sl["unit"], "config": sl["config"], "clocks": sl["clocks"],
                             **{k: so[k] for k in ("step_ms_p50", "step_ms_p99", "job_latency_s_p50",
                                                   "job_latency_s_p99", "jobs_finished", "wall_s",
                                                   "mean_active_jobs")}}
    if rank == 0:
        ms = statistics.mean(step_ms)
        line = {
            "metric": "body_substeps_per_s", "value": value, "unit": "body-substeps/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": workload, "bodies": n_dyn, "substeps": substeps,
                       "dt": "1/120" if substeps == 8 else "1/60",
                       "settle_steps": settle, "l2": "flushed (256 MiB write) between timed steps",
                       "parallelism": f"replicas x{ws}" if ws > 1 else "single world",
                       "contact_points_mean": statistics.mean(pts), "pairs_mean": statistics.mean(
                           [s["pairs_tested"] for s in stats]),
                       # 1: constraint rows in the cluster's shared memory; 2: the
                       # rows that do not fit spilled to global memory; 3: all in L2
                       "sweep_paths": sorted({int(s["sweep_path"]) for s in stats})},
            "contacts_per_s": contacts_per_s,
            "step_latency_ms": {"p50": float(np.percentile(step_ms, 50)), "p99": float(np.percentile(step_ms, 99)),
                                "kernel_mean": statistics.mean(kern_ms), "pairs_mean": statistics.mean(pair_ms)},
            "roofline": {"bound": "hbm", "achieved": kernels[dominant]["achieved"], "peak": peak, "unit": "GB/s",
                         "frac": kernels[dominant]["frac"],
                         "traffic": PROFILED_TRAFFIC.get((workload, dominant), (None,))[0],
                         "traffic_source": PROFILED_TRAFFIC.get((workload, dominant), (None, None))[1],
                         "traffic_captured_at": PROFILED_TRAFFIC.get((workload, dominant), (None, None, None))[2],
                         "peak_kind": peak_kind, "kernel": dominant,
                         "alg_bytes_per_launch": kernels[dominant]["alg_bytes_per_launch"],
                         "step": {"achieved": achieved, "frac": achieved / peak,
                                  "alg_bytes_per_step": statistics.mean(nb)},
                         "kernels": {k: dict(v, traffic=PROFILED_TRAFFIC.get((workload, k), (None,))[0])
                                     for k, v in kernels.items()}},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "body-substeps/s", "h2d_bytes_per_step": h2d // max(1, args.steps),
                    "d2h_bytes_per_step": d2h // max(1, args.steps)},
            "clocks": clk,
            "gpu_launches": args.steps * (len(kernels) if grid else 1),
            **extras,
        }
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return 0


def batched(args, steps=None, warmup=None, emit=True, dist_ctx=(1, 0, 0, None)):
    """256 independent worlds (bodies per world floor(exp(U(ln 8, ln 2048))),
    config-2 shapes, own 64x1x64 slab, dt 1/60, 4 substeps) stepped by one
    graph-replayed launch per step under the autotuned schedule, against the
    plain single-world path stepping the same worlds one after another.
    With N ranks the worlds are sharded by estimated cost (sharding.partition,
    the same on every rank, no exchange); times are the slowest rank's and the
    plain path's time is the sum over ranks (one GPU stepping every world).
    Returns the line (printed on rank 0 when emit)."""
    import torch

    ws, rank, local, pg = dist_ctx
    steps = args.steps if steps is None else steps
    warmup = args.warmup if warmup is None else warmup
    vxp = importlib.import_module("zig-voxel-physics_b200")
    all_scenes = vxp.scenes.config3(n_worlds=args.worlds)
    n_dyn = sum(sc.dynamic_count for sc in all_scenes)
    parts = vxp.sharding.partition([vxp.sharding.world_cost(sc.dynamic_count) for sc in all_scenes], ws)
    scenes = [all_scenes[i] for i in parts[rank]]
    dt = np.float32(1.0 / 60.0)
    b = vxp.VoxelWorldBatch(len(scenes), substeps=4, device=local)
    off, offs = 0, []
    for i, sc in enumerate(scenes):
        b.load_scene(i, sc, collider_offset=off)
        offs.append(off)
        off += len(sc.colliders) + 1
    # half-way through the configuration's 300 steps: the lower layers of
    # every world have landed, so the timed steps carry contacts
    if args.batch_settle:
        b.step(dt, args.batch_settle)
        b.synchronize()
    choice, tune_ms = b.autotune(dt, trial_steps=2)
    for _ in range(warmup):
        b.step(dt)
        b.synchronize()
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=f"cuda:{local}")
    clocks = Clocks(local)
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    clocks.start()
    step_ms, world_ms = [], []
    for _ in range(steps):
        flush.zero_()
        torch.cuda.synchronize()
        b.step(dt)
        b.synchronize()
        tot, per = b.times()
        step_ms.append(tot)
        world_ms.append(per[per > 0])
    clk = clocks.stop()
    batch_s = max_over_ranks(pg, sum(step_ms) / 1e3, f"cuda:{local}")
    value = n_dyn * 4 * steps / batch_s
    # e2e: the same steps with every world's body table read back each step
    bufs = [np.zeros(len(sc.bodies), dtype=vxp.abi.BODY_DTYPE) for sc in scenes]
    d2h = 0
    t0 = time.perf_counter()
    for _ in range(steps):
        b.step(dt)
        b.synchronize()
        for i in range(len(scenes)):
            b._check(b.lib.vxp_batch_world_get(b.b, i, vxp.abi.ptr(bufs[i]), len(bufs[i])))
            d2h += bufs[i].nbytes
    e2e_s = max_over_ranks(pg, time.perf_counter() - t0, f"cuda:{local}")
    states = []
    for i, sc in enumerate(scenes):
        st = b.get_world(i)
        st["collider_id"] -= offs[i]
        states.append(st)
    b.close()
    # plain path: each world stepped alone by its own launches, one world
    # after another, from the state the batch reached
    plain_ms = 0.0
    for sc, st in zip(scenes, states):
        # pair buffers sized up front: a fresh context's first device pair
        # list would otherwise overflow its default capacity on a settled world
        s = vxp.VoxelPhysicsSystem(substeps=4, device=local, max_pairs=max(1024, 16 * sc.dynamic_count))
        s.load_scene(sc)
        s.set_bodies(st)
        for _ in range(2):
            s.step(dt)
        s.synchronize()
        tt = []
        for _ in range(3):
            s.step(dt)
            out = np.zeros(3, dtype=np.float32)
            s._check(s.lib.vxp_last_step_ms(s.ctx, vxp.abi.ptr(out)))
            tt.append(float(out[2]))
        plain_ms += statistics.mean(tt)
        s.close()
    if pg:
        import torch.distributed as dist

        t = torch.tensor([plain_ms], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        plain_ms = float(t.item())
        gathered = [None] * ws
        dist.all_gather_object(gathered, [float(x) for x in np.concatenate(world_ms)] if world_ms else [])
        wm = np.array([x for g in gathered for x in g]) if any(gathered) else np.zeros(1)
    else:
        wm = np.concatenate(world_ms) if world_ms else np.zeros(1)
    plain_value = n_dyn * 4 / (plain_ms / 1e3)
    line = {
        "metric": "body_substeps_per_s", "value": value, "unit": "body-substeps/s", "n_gpus": ws,
        "steps": steps, "warmup": warmup, "ms_per_step": 1e3 * batch_s / steps,
        "higher_is_better": True, "scaling": "strong" if ws > 1 else "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": f"config3_batched_{len(all_scenes)}", "worlds": len(all_scenes), "bodies": n_dyn,
                   "settle_steps": args.batch_settle,
                   "parallelism": f"worlds sharded over {ws} GPUs by estimated cost" if ws > 1 else "one GPU",
                   "substeps": 4, "dt": "1/60", "l2": "flushed (256 MiB write) between timed steps",
                   "schedule": {"choice": vxp.VoxelWorldBatch.schedule_name(choice),
                                "autotune_ms": [float(x) for x in tune_ms]}},
        "plain_single_world": {"value": plain_value, "ms_per_batch_step": plain_ms,
                               "method": "each world alone from the batch's state, its own launches, "
                                         "3 timed steps after 2, summed"},
        "batched_over_plain": value / plain_value,
        "world_step_latency_ms": {"p50": float(np.percentile(wm, 50)), "p99": float(np.percentile(wm, 99)),
                                  "max": float(wm.max())},
        "e2e": {"value": n_dyn * 4 * steps / e2e_s, "unit": "body-substeps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": d2h // steps},
        "clocks": clk,
        "gpu_launches": steps,
    }
    if emit and rank == 0:
        print(json.dumps(line), flush=True)
    return line


def serving(args, jobs=None, emit=True, dist_ctx=(1, 0, 0, None)):
    """Jobs arrive as a Poisson process (mean 200 jobs/s), each a world of
    log-uniform 16..4096 config-2 boxes over its own slab running a uniform
    60..600 steps of dt 1/60 with 4 substeps; admitted against a 120 GB
    device-memory budget into a continuously batched set of world slots.
    With N ranks each job goes to one rank by estimated outstanding work
    (sharding.assign_jobs, the same on every rank, no exchange) and every rank
    serves its jobs on its own GPU; throughput is all jobs' work over the
    slowest rank's wall time, latency percentiles are over all jobs and steps.
    Returns the line (printed on rank 0 when emit)."""
    ws, rank, local, pg = dist_ctx
    n_jobs = args.jobs if jobs is None else jobs
    vxp = importlib.import_module("zig-voxel-physics_b200")
    sc = vxp.scenes
    lib = sc.shape_library()
    specs = sc.serving_jobs(n_jobs, seed=5)
    owner = vxp.sharding.assign_jobs(specs, ws)
    jobs = [vxp.server.Job(i, j["arrival"], sc.job_bodies(j), j["steps"]) for i, j in enumerate(specs)
            if owner[i] == rank]
    batch = vxp.VoxelWorldBatch(args.slots, substeps=4, device=local)
    for c in lib:
        batch.add_collider(c.id, c.voxel_size, c.bricks)
    batch.set_schedule(512, 1)
    server = vxp.server.SimulationServer(batch, 1.0 / 60.0, max_slots=args.slots, budget_bytes=120 * 10**9)
    clocks = Clocks(local)
    if pg:
        pg.barrier()
    clocks.start()
    out = server.run(jobs)
    clk = clocks.stop()
    batch.close()
    if pg:
        import torch.distributed as dist

        mine = (out["body_substeps"], out["wall_s"], list(server.step_ms),
                [j.finished_at - j.arrival for j in server.finished], out["jobs_finished"])
        got = [None] * ws
        dist.all_gather_object(got, mine)
        wall = max(g[1] for g in got)
        steps_ms = [x for g in got for x in g[2]]
        lat = [x for g in got for x in g[3]]
        out = dict(out, body_substeps=sum(g[0] for g in got), wall_s=wall,
                   body_substeps_per_s=sum(g[0] for g in got) / wall if wall > 0 else 0.0,
                   steps=len(steps_ms), jobs_finished=sum(g[4] for g in got), jobs_total=n_jobs,
                   step_ms_p50=float(np.percentile(steps_ms, 50)), step_ms_p99=float(np.percentile(steps_ms, 99)),
                   job_latency_s_p50=float(np.percentile(lat, 50)), job_latency_s_p99=float(np.percentile(lat, 99)))
    line = {
        "metric": "body_substeps_per_s", "value": out["body_substeps_per_s"], "unit": "body-substeps/s",
        "n_gpus": ws, "steps": out["steps"], "warmup": 0, "ms_per_step": out["step_ms_p50"],
        "higher_is_better": True, "scaling": "strong" if ws > 1 else "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": "config5_serving", "jobs": n_jobs, "arrival_rate_per_s": 200,
                   "parallelism": f"jobs sharded over {ws} GPUs by estimated work" if ws > 1 else "one GPU",
                   "bodies": "log-uniform 16..4096", "steps": "uniform 60..600", "dt": "1/60", "substeps": 4,
                   "slots": args.slots, "budget_bytes": 120 * 10**9},
        "serving": out,
        "clocks": clk,
    }
    if emit and rank == 0:
        print(json.dumps(line), flush=True)
    return line


def main():
    args = parse()
    if args.impl == "reference":
        return reference_arm(args)
    if args.workload in ("batched", "serving"):
        ws, rank, local, pg = dist_setup(args)
        import torch

        torch.cuda.set_device(local)
        (batched if args.workload == "batched" else serving)(args, dist_ctx=(ws, rank, local, pg))
        if pg:
            pg.barrier()
            pg.destroy_process_group()
        return 0
    return ours(args)


if __name__ == "__main__":
    sys.exit(main())
