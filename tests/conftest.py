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


def _reference_tree():
    """The reference source tree: SIDR_REF, else the tree oracle/Makefile built
    oracle/_ref from (it records the path in oracle/_ref/reference_tree.txt);
    None when neither is known (on a machine without the tree the tests that
    read it are skipped)."""
    if os.environ.get("SIDR_REF"):
        return os.environ["SIDR_REF"]
    rec = os.path.join(REPO, "oracle", "_ref", "reference_tree.txt")
    if os.path.exists(rec):
        with open(rec) as f:
            return f.read().strip() or None
    return None


REFERENCE_TREE = _reference_tree()


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
    if not REFERENCE_TREE or not os.path.isdir(os.path.join(REFERENCE_TREE, "instances")):
        pytest.skip("reference tree not present")
    return REFERENCE_TREE
