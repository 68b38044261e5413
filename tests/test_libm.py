"""The evaluator's erf, erfc and exp (csrc/sidr_libm.cuh) against the host C
library, bit for bit: the host build of the same header over random
arguments in every interval of the algorithms (CPU), and the device build
over the same kind of arguments (GPU)."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from conftest import PKG, REPO, cuda_available

import sidr

CSRC = os.path.join(PKG, "csrc")


def test_host_build_matches_libc(tmp_path):
    exe = tmp_path / "libm_check"
    subprocess.run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-I", CSRC,
                    os.path.join(REPO, "tests", "cpp", "libm_check.cpp"), "-o", str(exe)],
                   check=True)
    r = subprocess.run([str(exe), "200000", "3"], capture_output=True, text=True)
    rows = [ln.split() for ln in r.stdout.splitlines() if not ln.startswith("#")]
    assert len(rows) == 27
    bad = [row for row in rows if row[3] != "0"]
    assert not bad and r.returncode == 0, r.stdout


LIBC = ctypes.CDLL("libm.so.6")
for _f in ("erf", "erfc", "exp"):
    getattr(LIBC, _f).restype = ctypes.c_double
    getattr(LIBC, _f).argtypes = [ctypes.c_double]

INTERVALS = {
    "erf": [(-0.84375, 0.84375), (0.84375, 1.25), (-1.25, -0.84375), (1.25, 2.857142857142857),
            (2.857142857142857, 6.0), (-6.0, -1.25), (-1e-8, 1e-8)],
    "erfc": [(-0.25, 0.25), (0.25, 0.84375), (0.84375, 1.25), (-1.25, -0.84375), (1.25, 6.0),
             (6.0, 28.0), (-6.5, -1.25)],
    "exp": [(-40.0, 1.0), (-745.5, -512.0), (512.0, 709.7), (-1e-6, 1e-6)],
}


@pytest.mark.gpu
@pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")
@pytest.mark.parametrize("fn", ["erf", "erfc", "exp"])
def test_device_matches_libc(fn):
    rng = np.random.default_rng(11)
    xs = np.concatenate([rng.uniform(a, b, 100000) for a, b in INTERVALS[fn]] +
                        [np.array([0.0, -0.0, 1.0, -1.0, 6.0, -6.0, 28.0, np.inf, -np.inf])])
    got = sidr.libm_eval(fn, xs)
    f = getattr(LIBC, fn)
    exp = np.array([f(float(x)) for x in xs])
    bad = np.nonzero(got.view(np.uint64) != exp.view(np.uint64))[0]
    assert bad.size == 0, [(float(xs[i]).hex(), float(got[i]).hex(), float(exp[i]).hex())
                           for i in bad[:5]]
