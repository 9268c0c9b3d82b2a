"""Trajectory drift of the FP32 path against an FP64 replay of the same solver.

The device path is bit-identical to the FP32 oracle on every trajectory the
parity tests run (tests/test_gpu_parity.py), so its drift against FP64 is the
FP32 oracle's drift against the FP64 oracle, measured here on the CPU: both
worlds start from the same bodies and each builds its own pair list from its
own state, step after step.

    python tests/drift_report.py [--steps 300] [--out report.md]

prints a markdown table of the drift per step bracket.
"""
from __future__ import annotations

import argparse
import importlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(HERE))

import oracle_api as O  # noqa: E402


def _angle(q1: np.ndarray, q2: np.ndarray) -> np.ndarray:
    """Rotation angle of conj(q1) * q2 (x, y, z, w), in double."""
    a = q1.astype(np.float64)
    b = q2.astype(np.float64)
    w = a[:, 3] * b[:, 3] + np.sum(a[:, :3] * b[:, :3], axis=1)
    v = a[:, 3:4] * b[:, :3] - b[:, 3:4] * a[:, :3] - np.cross(a[:, :3], b[:, :3])
    return 2.0 * np.arctan2(np.linalg.norm(v, axis=1), np.abs(w))


def nudged(scene):
    """The scene with the first dynamic body's x moved by one float ulp."""
    import copy
    sc = copy.copy(scene)
    sc.bodies = scene.bodies.copy()
    k = int(np.flatnonzero(sc.bodies["body_type"] == 2)[0])
    x = np.float32(sc.bodies["position"][k, 0])
    sc.bodies["position"][k, 0] = np.nextafter(x, np.float32(np.inf), dtype=np.float32)
    return sc


def drift(scene, steps: int, dt: np.float32, precision_b: int = 64, scene_b=None, **cfg) -> list[dict]:
    """Per step: max position difference (m), max relative position
    difference (|dx| / max(|x|, 1 m)), max linear velocity difference (m/s),
    max rotation difference (rad) over the dynamic bodies, between the FP32
    world on `scene` and a second world (FP64 by default) on `scene_b`."""
    w32 = O.OracleWorld(precision=32, **cfg)
    w64 = O.OracleWorld(precision=precision_b, **cfg)
    w32.load_scene(scene)
    w64.load_scene(scene if scene_b is None else scene_b)
    dyn = scene.bodies["body_type"] == 2
    rows = []
    for s in range(steps):
        w32.step(dt)
        w64.step(dt)
        a, b = w32.get_bodies()[dyn], w64.get_bodies()[dyn]
        dx = np.linalg.norm(a["position"].astype(np.float64) - b["position"].astype(np.float64), axis=1)
        scale = np.maximum(np.linalg.norm(b["position"].astype(np.float64), axis=1), 1.0)
        dv = np.linalg.norm(a["linear_velocity"].astype(np.float64) - b["linear_velocity"].astype(np.float64), axis=1)
        rows.append({"step": s + 1, "max_dx": float(dx.max()), "max_rel_dx": float((dx / scale).max()),
                     "mean_dx": float(dx.mean()), "max_dv": float(dv.max()),
                     "max_dq": float(_angle(a["rotation"], b["rotation"]).max()),
                     "mean_y32": float(a["position"][:, 1].astype(np.float64).mean()),
                     "mean_y64": float(b["position"][:, 1].astype(np.float64).mean()),
                     "sleeping32": int(a["is_sleeping"].sum()), "sleeping64": int(b["is_sleeping"].sum())})
    w32.close()
    w64.close()
    return rows


def table(rows: list[dict], brackets=(1, 10, 30, 60, 100, 150, 200, 300, 600)) -> str:
    out = ["| step | max dx (m) | max rel dx | mean dx (m) | max dv (m/s) | max dq (rad) | mean height (m) | sleeping |",
           "|---|---|---|---|---|---|---|---|"]
    for r in rows:
        if r["step"] in brackets or r["step"] == rows[-1]["step"]:
            out.append(f"| {r['step']} | {r['max_dx']:.3e} | {r['max_rel_dx']:.3e} | {r['mean_dx']:.3e} | "
                       f"{r['max_dv']:.3e} | {r['max_dq']:.3e} | {r['mean_y32']:.3f} / {r['mean_y64']:.3f} | "
                       f"{r['sleeping32']}/{r['sleeping64']} |")
    return "\n".join(out)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--out", default=None)
    args = ap.parse_args()
    vxp = importlib.import_module("zig-voxel-physics_b200")
    sc = vxp.scenes.config1(O.mass_fn)
    rows = drift(sc, args.steps, np.float32(sc.dt), substeps=4)
    base = drift(sc, args.steps, np.float32(sc.dt), precision_b=32, scene_b=nudged(sc), substeps=4)
    text = (f"config 1 (64 cubes on the 64x1x64 slab, dt 1/60, 4 substeps), {args.steps} steps\n\n"
            "FP32 vs FP64 replay of the same solver:\n\n" + table(rows) +
            "\n\nChaos baseline, FP32 vs FP32 with one body's starting x moved by one ulp:\n\n" + table(base))
    print(text)
    if args.out:
        with open(args.out, "w") as f:
            f.write(text + "\n")


if __name__ == "__main__":
    main()
