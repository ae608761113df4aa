"""Test configuration: the `gpu` marker, import paths, shared meshes.

CPU tests (``-m "not gpu"``) cover the oracle against the reference's own invariant tests and the golden vectors,
the host logic and the C-ABI exports. GPU tests (``-m gpu``) compare the CUDA path, called through the C ABI, with
the oracle on the same seeded inputs.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "three-virtual-geometry_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the sm_100a kernels")


def _has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device on this host")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session")
def terrain():
    """The reference cut test's terrain: PlaneGeometry(400, 400, 96, 96), y = 30 sin(0.05 x) cos(0.04 z)
    (tests/cut.test.ts:14-19), built into a cluster DAG by this repository's builder."""
    from vgcut import build as B
    pos, idx = B.gen_terrain(400.0, 96, 30.0, 0.05, 0.04)
    return B.build_virtual_mesh(pos, idx)


class ParkMiller:
    """The reference tests' seeded RNG: seed = seed * 16807 % (2^31 - 1) (tests/cut.test.ts:11-12)."""

    def __init__(self, seed: int):
        self.seed = seed

    def __call__(self) -> float:
        self.seed = (self.seed * 16807) % 2147483647
        return self.seed / 2147483647


@pytest.fixture
def park_miller():
    return ParkMiller
