"""Admission and retirement logic of the simulation server, on a fake batch
(no GPU): FIFO admission at step boundaries, slot and memory-budget limits,
every job runs exactly its step count."""
import numpy as np

from conftest import load_package

srv = load_package().server


class FakeBatch:
    def __init__(self, n_slots):
        self.config = type("C", (), {"substeps": 4})()
        self.worlds = {}
        self.steps = {}

    def set_world(self, slot, bodies):
        assert slot not in self.worlds
        self.worlds[slot] = bodies.copy()
        self.steps[slot] = 0

    def world_bytes(self, slot):
        return 0

    def step(self, dt, n):
        for s in self.worlds:
            self.steps[s] += n

    def synchronize(self):
        pass

    def times(self):
        return 1.0, None

    def get_world(self, slot):
        return self.worlds[slot]

    def clear_world(self, slot):
        del self.worlds[slot]
        del self.steps[slot]


class FakeClock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        self.t += 0.001
        return self.t


def make_jobs(n, rng):
    jobs = []
    for i in range(n):
        b = np.zeros(int(rng.integers(16, 200)), dtype=load_package().abi.BODY_DTYPE)
        b["body_type"] = 2
        jobs.append(srv.Job(i, float(i) * 0.002, b, int(rng.integers(3, 12))))
    return jobs


def test_every_job_runs_exactly_its_steps():
    rng = np.random.default_rng(0)
    jobs = make_jobs(40, rng)
    fb = FakeBatch(8)
    s = srv.SimulationServer(fb, 1 / 60, max_slots=8, clock=FakeClock())
    steps_seen = {}
    orig_clear = fb.clear_world

    def clear(slot):
        steps_seen[slot] = fb.steps[slot]
        orig_clear(slot)

    fb.clear_world = clear
    out = s.run(jobs)
    assert out["jobs_finished"] == 40
    for j in s.finished:
        assert j.done_steps == j.steps
        assert j.admitted_at >= j.arrival
        assert j.finished_at > j.admitted_at
    assert max(s.active_per_step) <= 8


def test_memory_budget_limits_admission():
    rng = np.random.default_rng(1)
    jobs = make_jobs(12, rng)
    budget = 3 * srv.estimate_bytes(200)
    s = srv.SimulationServer(FakeBatch(64), 1 / 60, max_slots=64, budget_bytes=budget, clock=FakeClock())
    peak = [0]
    orig = s._admit

    def admit(now):
        orig(now)
        peak[0] = max(peak[0], s.used_bytes)
        assert s.used_bytes <= budget

    s._admit = admit
    out = s.run(jobs)
    assert out["jobs_finished"] == 12
    assert peak[0] <= budget


def test_fifo_when_slots_are_scarce():
    rng = np.random.default_rng(2)
    jobs = make_jobs(10, rng)
    s = srv.SimulationServer(FakeBatch(2), 1 / 60, max_slots=2, clock=FakeClock())
    s.run(jobs)
    admitted = sorted(s.finished, key=lambda j: j.admitted_at)
    assert [j.job_id for j in admitted] == sorted(j.job_id for j in admitted)
