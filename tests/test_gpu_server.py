"""The served path: jobs arriving over time into a continuously batched
world set; each job's result must equal the same job stepped alone."""
import numpy as np
import pytest

import oracle_api as O

pytestmark = pytest.mark.gpu


class StepClock:
    """Deterministic clock: 1 ms per call."""

    def __init__(self):
        self.t = 0.0

    def __call__(self):
        self.t += 0.001
        return self.t


def test_jobs_alone_equal_jobs_in_the_mix(vxp):
    sc = vxp.scenes
    lib = sc.shape_library(O.mass_fn)
    specs = sc.serving_jobs(10, seed=31, lo=16, hi=300, steps_lo=20, steps_hi=70)
    dt = np.float32(1.0 / 60.0)
    batch = vxp.VoxelWorldBatch(4, substeps=4)
    for c in lib:
        batch.add_collider(c.id, c.voxel_size, c.bricks)
    jobs = [vxp.server.Job(i, j["arrival"] * 0.2, sc.job_bodies(j, O.mass_fn), j["steps"]) for i, j in enumerate(specs)]
    server = vxp.server.SimulationServer(batch, dt, max_slots=4, clock=StepClock())
    out = server.run(jobs)
    assert out["jobs_finished"] == len(jobs)
    assert max(server.active_per_step) <= 4
    overlapped = sum(1 for a in server.active_per_step if a > 1)
    assert overlapped > 0  # jobs did share steps
    for job in server.finished:
        # alone: a fresh context (empty contact manager and cache) per job
        s = vxp.VoxelPhysicsSystem(substeps=4)
        used = np.unique(job.bodies["collider_id"])
        for c in lib:
            if c.id in used:
                s.add_collider(c.id, c.voxel_size, c.bricks)
        s.set_bodies(job.bodies)
        for _ in range(job.steps):
            s.step(dt)
        assert s.get_bodies().tobytes() == job.result.tobytes(), f"job {job.job_id} differs alone vs in the mix"
        s.close()
    batch.close()
