"""Builds libsidr_b200.so in-tree (this directory) for sm_100a.

    python solver-informed-dispatching-rules_b200/build.py [--force]

CUDA sources are compiled by nvcc with -gencode arch=compute_100a,code=sm_100a,
-fmad=false (no multiply-add contraction: the evaluator must reproduce the
reference CPU simulator's IEEE operations one by one) and -lineinfo; host C++
with -ffp-contract=off for the same reason.  The CUDA runtime is linked
statically.  No JIT cache is involved: the built .so is a plain file next to
this script.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libsidr_b200.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-std=c++17", "-O3", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC,-ffp-contract=off",
           "-Xptxas", "-v"]
CXXFLAGS = ["-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-Wall"]

CU_SOURCES = ["sidr_capi.cu", "sidr_surrogate.cu", "sidr_sample.cu"]
CPP_SOURCES = ["sidr_host.cpp", "sidr_gp.cpp", "sidr_campaign.cpp", "sidr_sgp.cpp"]
HEADERS = ["sidr_internal.hpp", "sidr_kernel.cuh", "sidr_host.hpp", "sidr_libm.cuh", "sidr_exp_table.h",
           "sidr_gp_core.hpp", "sidr_mlp.cuh", "sidr_sgp_select.hpp", "sidr_device.hpp",
           "sidr_sample.cuh", "sidr_sample_consts.h"]
PUBLIC_HEADERS = ["sidr.h", "sidr_gp.h", "sidr_campaign.h", "sidr_surrogate.h"]


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, log=None):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if log is not None:
        with open(log, "w") as f:
            f.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
    if r.returncode != 0:
        raise RuntimeError("build step failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    deps_common = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, h) for h in PUBLIC_HEADERS]
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _newer(o, [s] + deps_common):
            _run([NVCC] + ARCH + NVFLAGS + ["-I", INCLUDE, "-c", s, "-o", o],
                 log=os.path.join(BUILD, src + ".log"))
    for src in CPP_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _newer(o, [s] + deps_common):
            _run(["g++"] + CXXFLAGS + ["-I", INCLUDE, "-c", s, "-o", o])
    if force or _newer(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lpthread"])
    if verbose:
        print("built", LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    try:
        build(force=a.force, verbose=True)
    except RuntimeError as e:
        print(e, file=sys.stderr)
        sys.exit(1)
