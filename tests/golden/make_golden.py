"""Writes the golden fixtures of this directory from the CPU oracle.

    python tests/golden/make_golden.py

config1_bodies.npz     body table (vxp_body records) of config 1 (64 cubes on
                       the 64x1x64 slab, dt 1/60, 4 substeps, seed 1) after
                       steps 1, 10, 50, 150 and 300, each world building its
                       own pair list (AABB margin 0.1 m)
config1_manifolds.npy  the contact manager's manifolds after step 20
                       (vxp_manifold records, manifold order)

The Zig reference cannot be built here, so the fixtures are the oracle's
outputs; tests/test_golden.py keeps the oracle on them and
tests/test_gpu_golden.py holds the device path to them, bit for bit.
"""
import importlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle_api as O  # noqa: E402

STEPS = (1, 10, 50, 150, 300)
MANIFOLD_STEP = 20


def config1_run(vxp):
    sc = vxp.scenes.config1(O.mass_fn)
    w = O.OracleWorld(substeps=4)
    w.load_scene(sc)
    dt = np.float32(sc.dt)
    snaps, man = {}, None
    for s in range(1, max(STEPS) + 1):
        w.step(dt)
        if s in STEPS:
            snaps[f"step{s}"] = w.get_bodies()
        if s == MANIFOLD_STEP:
            man = w.manifolds()
    w.close()
    return snaps, man


def main():
    vxp = importlib.import_module("zig-voxel-physics_b200")
    snaps, man = config1_run(vxp)
    np.savez_compressed(os.path.join(HERE, "config1_bodies.npz"), **snaps)
    np.save(os.path.join(HERE, "config1_manifolds.npy"), man)
    print("wrote", sorted(snaps), "and", len(man), "manifolds")


if __name__ == "__main__":
    main()
