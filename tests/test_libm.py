"""The evaluator's erf, erfc, exp and pow (csrc/sidr_libm.cuh) against the host
C library, bit for bit: the host build of the same header over random
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
    assert len(rows) == 27 + 8 + 1  # erf/erfc/exp intervals, 7 pow families, pow specials, rmod
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


@pytest.mark.gpu
@pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")
def test_device_pow_matches_libc():
    """rmod's pow on the device: x >= 0, y in [1, 2] over many magnitudes,
    rule-like ratios, the whole double range, other exponents, subnormal and
    negative bases, and the special operands."""
    rng = np.random.default_rng(12)
    n = 200000
    xs = [np.exp2(rng.uniform(-30, 30, n)), rng.uniform(0.5, 2.0, n),
          np.exp2(rng.uniform(-1074, 1023.9, n)),
          rng.integers(1, 1000001, n) / rng.integers(1, 1001, n),
          np.exp2(rng.uniform(-1022, 1023.9, n)),
          (rng.integers(0, 1 << 52, n, dtype=np.uint64)).view(np.float64),
          -np.exp2(rng.uniform(-10, 10, n))]
    ys = [rng.uniform(1, 2, n), rng.uniform(1, 2, n), rng.uniform(1, 2, n),
          1.0 + rng.integers(0, 1001, n) / 1000.0, rng.uniform(-8, 8, n), rng.uniform(0.5, 2, n),
          np.trunc(rng.uniform(-10, 10, n)) + 0.5 * rng.integers(0, 2, n)]
    sx = np.array([0.0, -0.0, 1.0, -1.0, 2.0, 0.5, 5e-324, 1e308, np.inf, -np.inf, np.nan, -2.0])
    sy = np.array([0.0, 1.0, 2.0, 1.5, -1.0, 0.5, 3.0, np.inf, -np.inf, np.nan, 1075.0])
    gx, gy = np.meshgrid(sx, sy)
    x = np.concatenate(xs + [gx.ravel()])
    y = np.concatenate(ys + [gy.ravel()])
    got = sidr.libm_pow(x, y)
    LIBC.pow.restype = ctypes.c_double
    LIBC.pow.argtypes = [ctypes.c_double, ctypes.c_double]
    exp = np.array([LIBC.pow(float(a), float(b)) for a, b in zip(x, y)])
    same = (got.view(np.uint64) == exp.view(np.uint64)) | (np.isnan(got) & np.isnan(exp))
    bad = np.nonzero(~same)[0]
    assert bad.size == 0, [(float(x[i]).hex(), float(y[i]).hex(), float(got[i]).hex(),
                            float(exp[i]).hex()) for i in bad[:5]]
