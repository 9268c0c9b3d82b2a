"""Continuous-batching simulation server.

Jobs (a world of bodies plus a step count) arrive over time.  The server
keeps every running job's state resident on the device in one slot of a
VoxelWorldBatch and advances all of them with one launch per step; a job
that arrives while others run is admitted at the next step boundary as soon
as a slot is free and its device memory fits the budget, and its steps then
overlap with everyone else's on the GPU.  A finished job's final bodies are
read back and its slot freed; the slot keeps its device buffers for the next
job admitted there (no allocation or free while serving), and those buffers
stay counted against the budget.

Every world's arithmetic is independent of the batch it runs in, so a job's
result is bit-identical alone and in any mix.

Timing: per-step latency is the device time of each batch step; per-job
latency is host wall time from arrival to completion; throughput is
body-substeps per second of wall time over the run.
"""
from __future__ import annotations

import collections
import dataclasses
import time

import numpy as np


@dataclasses.dataclass
class Job:
    job_id: int
    arrival: float          # seconds after the server started
    bodies: np.ndarray      # body table (collider ids refer to the shape library)
    steps: int
    slot: int = -1
    done_steps: int = 0
    admitted_at: float = -1.0
    finished_at: float = -1.0
    result: np.ndarray | None = None
    device_bytes: int = 0

    @property
    def dynamic(self) -> int:
        return int((self.bodies["body_type"] == 2).sum())


def estimate_bytes(n_bodies: int, cache_entries: int = 1024) -> int:
    """Device memory a world of n bodies takes (WorldBuffers with the default
    pair capacity of 16 x n, at least 1024): ~1.4 KB per pair slot, ~480 B
    per body, the broad phase's hit masks (body capacity^2 / 8 bytes up to
    8192 bodies), ~0.4 MB of brick-pair cache and fixed scratch."""
    pairs = max(1024, 16 * n_bodies)
    cap = 1024
    while cap < pairs:
        cap *= 2
    bcap = 64
    while bcap < n_bodies:
        bcap *= 2
    # + two island key buffers per pair slot
    per_pair = 8 + 76 + 2 * 376 + 4 * 6 + 24 + 4 * 31 * 4 + 16 + 8 + 2 * 16 * 2 + 2 * 8
    # + the island arrays, the public collider id and the packed readback record
    per_body = 112 + 64 + 4 * 16 + 8 + 4 * 4 + 4 * 10 + 16 + 4 + 128
    masks = bcap * ((bcap + 31) // 32) * 4 if bcap <= 8192 else 0
    return (cap * per_pair + max(64, n_bodies) * per_body + masks + cache_entries * (24 + 368 + 4) +
            (64 << 10))


class SimulationServer:
    """Admission by free slot and device-memory budget, continuous batching."""

    def __init__(self, batch, dt: float, max_slots: int, budget_bytes: int = 120 * 10**9, clock=time.perf_counter):
        self.batch = batch
        self.dt = np.float32(dt)
        self.max_slots = int(max_slots)
        self.budget = int(budget_bytes)
        self.clock = clock
        self.free_slots = list(range(self.max_slots))
        self.held = [0] * self.max_slots  # device bytes each slot holds, running or not
        self.running: dict[int, Job] = {}
        self.waiting: collections.deque[Job] = collections.deque()
        self.finished: list[Job] = []
        self.used_bytes = 0
        self.step_ms: list[float] = []
        self.active_per_step: list[int] = []
        self.t0 = None

    # ----------------------------------------------------------- admission
    def submit(self, job: Job) -> None:
        self.waiting.append(job)

    def _admit(self, now: float) -> None:
        kept = collections.deque()
        while self.waiting:
            job = self.waiting.popleft()
            if job.arrival > now:
                kept.append(job)
                continue
            need = estimate_bytes(len(job.bodies))
            if not self.free_slots:
                kept.append(job)
                continue
            # the free slot whose buffers already fit with the least to spare,
            # else the one holding the most
            fits = [s for s in self.free_slots if self.held[s] >= need]
            slot = min(fits, key=lambda s: self.held[s]) if fits else max(self.free_slots, key=lambda s: self.held[s])
            if self.used_bytes + max(0, need - self.held[slot]) > self.budget:
                kept.append(job)
                continue
            self.free_slots.remove(slot)
            self.batch.set_world(slot, job.bodies)
            job.slot = slot
            job.admitted_at = now
            job.device_bytes = max(need, self.held[slot], self.batch.world_bytes(slot))
            self.used_bytes += job.device_bytes - self.held[slot]
            self.held[slot] = job.device_bytes
            self.running[slot] = job
        self.waiting = kept

    def _retire(self, now: float) -> None:
        for slot in [s for s, j in self.running.items() if j.done_steps >= j.steps]:
            job = self.running.pop(slot)
            job.result = self.batch.get_world(slot)
            job.finished_at = now
            self.batch.clear_world(slot)
            self.free_slots.append(slot)
            self.finished.append(job)

    # ---------------------------------------------------------------- loop
    def run(self, jobs: list, max_wall_s: float | None = None) -> dict:
        """Serves the jobs (arrival times relative to the start) to completion."""
        for j in sorted(jobs, key=lambda j: j.arrival):
            self.submit(j)
        self.t0 = self.clock()
        total_body_substeps = 0
        substeps = int(getattr(self.batch.config, "substeps", 4))
        while self.waiting or self.running:
            now = self.clock() - self.t0
            if max_wall_s is not None and now > max_wall_s:
                break
            self._admit(now)
            if not self.running:
                # idle until the next arrival
                nxt = min(j.arrival for j in self.waiting)
                while self.clock() - self.t0 < nxt:
                    pass
                continue
            self.batch.step(self.dt, 1)
            self.batch.synchronize()
            total_ms, _ = self.batch.times()
            self.step_ms.append(total_ms)
            self.active_per_step.append(len(self.running))
            for job in self.running.values():
                job.done_steps += 1
                total_body_substeps += job.dynamic * substeps
            self._retire(self.clock() - self.t0)
        wall = self.clock() - self.t0
        lat = [j.finished_at - j.arrival for j in self.finished]
        return {
            "jobs_finished": len(self.finished),
            "jobs_total": len(jobs),
            "wall_s": wall,
            "body_substeps": total_body_substeps,
            "body_substeps_per_s": total_body_substeps / wall if wall > 0 else 0.0,
            "steps": len(self.step_ms),
            "step_ms_p50": float(np.percentile(self.step_ms, 50)) if self.step_ms else None,
            "step_ms_p99": float(np.percentile(self.step_ms, 99)) if self.step_ms else None,
            "job_latency_s_p50": float(np.percentile(lat, 50)) if lat else None,
            "job_latency_s_p99": float(np.percentile(lat, 99)) if lat else None,
            "mean_active_jobs": float(np.mean(self.active_per_step)) if self.active_per_step else 0.0,
        }
