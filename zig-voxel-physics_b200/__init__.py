"""B200-native voxel contact generation and TGS-soft solving.

A drop-in for the per-step hot path of nitanmarcel/zig-voxel-physics
(NarrowPhase + ContactSolver behind VoxelPhysicsSystem.step).  The kernels
live in libvxp.so (csrc/, C ABI in include/vxp.h); this package holds the
host-side mirror of the reference interface (system.py), the ctypes layer
(abi.py), the seeded benchmark scenes (scenes.py), the continuous-batching
server (server.py), the sharding of worlds and jobs over GPUs (sharding.py)
and the build (build.py).

The directory name is not a Python identifier: import it with
importlib.import_module("zig-voxel-physics_b200").
"""
from . import abi, scenes, server, sharding  # noqa: F401
from .system import VoxelPhysicsSystem, VoxelWorldBatch, VxpError  # noqa: F401

__all__ = ["abi", "scenes", "server", "sharding", "VoxelPhysicsSystem", "VoxelWorldBatch", "VxpError"]
