"""The C++ drop-in, proven on the reference's own drivers.

oracle/Makefile (target dropin) compiles the reference's verify/verify_cuda.cu
and engine/gp_engine.cu where they lie, unchanged, as plain C++ against
tests/cpp/dropin/engine/factory.cuh -- the reference's engine/factory.cuh
after the maintainer's edit INTEGRATION.md describes (its PackedTrees format
kept, FactoryContext aliased to sidr::FactoryContextT from
include/sidr_factory.hpp) -- and links them against libsidr_b200.so.

* CPU: both drivers build and link against the library; without a device,
  verify_cuda stops the way the reference's CUDA_CHECK does (message, exit 2).
* GPU: verify_cuda runs its own gate through this library -- part (a) the
  golden simulator cases (verify/verify_cuda.cu:44-105), part (b) the CPU
  simulator against the evaluator on the all-61 sum tree (:107-142) -- and
  must report bit-exact agreement.
"""
import os
import subprocess

import pytest

from conftest import REPO, cuda_available

DROPIN = os.path.join(REPO, "oracle", "_ref", "dropin")
DATA = os.path.join(DROPIN, "data")


def _built():
    return os.path.exists(os.path.join(DROPIN, "verify_cuda"))


def test_reference_drivers_build_against_dropin(reference_tree):
    r = subprocess.run(["make", "-C", os.path.join(REPO, "oracle"), "dropin"], capture_output=True,
                       text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    for exe in ("verify_cuda", "gp_engine"):
        path = os.path.join(DROPIN, exe)
        assert os.access(path, os.X_OK), path
        libs = subprocess.run(["ldd", path], capture_output=True, text=True).stdout
        assert "libsidr_b200.so" in libs and "not found" not in libs, libs
    if not cuda_available():
        v = subprocess.run([os.path.join(DROPIN, "verify_cuda"), os.path.join(DATA, "sim.txt")],
                           capture_output=True, text=True, env=dict(os.environ, GITC_DATA=DATA))
        assert v.returncode == 2 and "sidr error" in v.stderr, (v.returncode, v.stderr)


@pytest.mark.gpu
@pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")
@pytest.mark.skipif(not _built(), reason="drop-in binaries not built (no reference tree at build time)")
def test_reference_verify_cuda_passes_through_dropin():
    v = subprocess.run([os.path.join(DROPIN, "verify_cuda"), os.path.join(DATA, "sim.txt")],
                       capture_output=True, text=True, env=dict(os.environ, GITC_DATA=DATA),
                       timeout=600)
    out = v.stdout
    assert v.returncode == 0, out + v.stderr
    assert "part (a) GPU vs recorded fixtures: 240 compared" in out, out
    assert "0 nonzero" in out and "OK bit-exact" in out, out
