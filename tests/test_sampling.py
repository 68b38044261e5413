"""The Box-Muller step of the on-device sampler (csrc/sidr_sample.cuh), built
for the host, against the host C library the reference samples with
(engine/rng.hpp:135-147): every log, sin and cos value the double-double
evaluation names is the library's (or one of the two it names), every pair it
settles equals the library's, and the pairs it leaves to the library stay a
small share.  Argument checks of sidr_gen_durations_device need no device."""
import math
import os
import subprocess

import numpy as np
import pytest

from conftest import PKG, REPO

import sidr
from sidr import gp as GP


def test_host_build_matches_libc(tmp_path):
    exe = tmp_path / "sample_check"
    subprocess.run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-I", os.path.join(PKG, "csrc"),
                    os.path.join(REPO, "tests", "cpp", "sample_check.cpp"), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe), "300000", "3"], capture_output=True, text=True)
    rows = {ln.split()[0]: [int(x) for x in ln.split()[1:]] for ln in r.stdout.splitlines()
            if not ln.startswith("#")}
    assert r.returncode == 0, r.stdout
    for name in ("log", "sin", "cos"):
        checked, single, bad = rows[name]
        assert bad == 0 and single > 0.8 * checked, (name, rows[name])
    assert rows["generator"][2] == 0, rows["generator"]
    pairs, settled, bad = rows["pairs"]
    assert bad == 0 and settled > 0.9 * pairs, rows["pairs"]


def test_device_sampler_refuses_bad_arguments():
    with pytest.raises(sidr.SidrError):
        GP.gen_durations_device([10.0, math.nan], 0.2, 4, 1)
    with pytest.raises(sidr.SidrError):
        GP.gen_durations_device([10.0, 5.0], math.inf, 4, 1)
