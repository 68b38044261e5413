"""Shared fixtures and import paths for the evaluator's tests.

Markers: ``gpu`` -- needs a CUDA device (the parity tests proper, through the
C-ABI).  Everything else runs on the CPU.
"""
import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "solver-informed-dispatching-rules_b200")
for p in (PKG, os.path.join(REPO, "oracle"), REPO):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(REPO, "tests", "golden")
REFERENCE_TREE = "/root/reference"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def oracle():
    from oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def reference():
    from oracle import Reference, reference_available
    if not reference_available():
        pytest.skip("oracle/_ref (the reference compiled from its own headers) not built")
    return Reference()


@pytest.fixture(scope="session")
def reference_tree():
    if not os.path.isdir(os.path.join(REFERENCE_TREE, "instances")):
        pytest.skip("reference tree not present")
    return REFERENCE_TREE
