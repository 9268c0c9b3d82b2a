"""The device path (C ABI, device pair source) against the committed golden
fixtures of config 1: body tables after steps 1, 10, 50, 150, 300 and the
manifolds after step 20, bit for bit, in both launch modes and with the
cluster sweeps."""
import os

import numpy as np
import pytest

import oracle_api as O

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("mode,solver", [(0, None), (1, 1), (1, 2)])
def test_device_path_matches_golden(vxp, mode, solver):
    gold = np.load(os.path.join(GOLD, "config1_bodies.npz"))
    gman = np.load(os.path.join(GOLD, "config1_manifolds.npy"))
    sc = vxp.scenes.config1(O.mass_fn)
    g = vxp.VoxelPhysicsSystem(substeps=4)
    g.load_scene(sc)
    g.set_launch_mode(mode)
    if solver is not None:
        g.set_solver_mode(solver)
    dt = np.float32(sc.dt)
    for s in range(1, 301):
        g.step(dt)
        if f"step{s}" in gold.files:
            assert g.get_bodies().tobytes() == gold[f"step{s}"].tobytes(), f"step {s}"
        if s == 20:
            assert g.manifolds().tobytes() == gman.tobytes(), "manifolds after step 20"
    g.close()
