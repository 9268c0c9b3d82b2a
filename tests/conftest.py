"""Shared fixtures: the package (its directory name is not an identifier), the
CPU oracle and the GPU marker."""
import importlib
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
TESTS = os.path.dirname(os.path.abspath(__file__))
if TESTS not in sys.path:
    sys.path.insert(0, TESTS)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libvxp.so")
    config.addinivalue_line("markers", "slow: long-running check")


def load_package():
    return importlib.import_module("zig-voxel-physics_b200")


@pytest.fixture(scope="session")
def vxp():
    return load_package()


@pytest.fixture(scope="session")
def oracle():
    import oracle_api

    return oracle_api


@pytest.fixture(scope="session")
def oracle_mass(oracle):
    return oracle.mass_fn
