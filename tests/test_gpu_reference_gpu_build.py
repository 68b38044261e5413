"""This evaluator against the reference's own GPU evaluator on the same device.

The reference's GPU path (engine/factory.cuh: one thread per (rule, scenario)
pair, FactoryContext::evaluate with host buffers) is compiled in place by
oracle/Makefile with its Makefile's flags into oracle/_ref/libsidr_ref_gpu.so.
On the benchmark generation (the GP's initial 1024 rules over the 29-terminal
menu on the clustered 100-customer instance, 500 scenarios), both called with
host buffers:

* this evaluator is faster;
* wherever the two disagree, this evaluator gives the CPU simulator's score
  (the reference's GPU build contracts multiply-adds, so it can leave the CPU
  simulator's result; the C oracle stands in for the simulator).

The timings are printed (pytest -s) as one JSON line."""
import json
import os
import time

import numpy as np
import pytest

from conftest import cuda_available

import sidr
from sidr import workload

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]


def test_faster_than_reference_gpu_build_and_equal_where_it_is_exact(oracle):
    from oracle import REF_GPU_SO, ReferenceGPU
    if not os.path.exists(REF_GPU_SO):
        pytest.skip("the reference's GPU build is not in oracle/_ref")
    w = workload.gp_generation(P=1024, S=500)
    zp = sidr.zstats(w.sd)
    ref = ReferenceGPU()
    ctx = sidr.Context(w.sd, zp)
    one = w.rules.subset([0])
    ref.evaluate(w.sd, zp, one, w.sampled[:1], 1, w.mask)  # context and module load
    ctx.evaluate(one, w.sampled[:1], 1, w.mask)

    t0 = time.perf_counter()
    theirs = ref.evaluate(w.sd, zp, w.rules, w.sampled, w.S, w.mask)
    t_ref = time.perf_counter() - t0
    t0 = time.perf_counter()
    ours = ctx.evaluate(w.rules, w.sampled, w.S, w.mask)
    t_ours = time.perf_counter() - t0
    ctx.close()

    pairs = w.rules.P * w.S
    diff = np.nonzero((ours.view(np.uint64) != theirs.view(np.uint64)).any(axis=1))[0]
    print(json.dumps({"pairs": pairs, "reference_gpu_evals_per_s": pairs / t_ref,
                      "this_evaluator_evals_per_s": pairs / t_ours, "speedup": t_ref / t_ours,
                      "rules_where_the_builds_differ": int(diff.size)}))
    assert t_ours < t_ref
    assert diff.size <= 64, "the two GPU builds differ on too many rules to check here"
    if diff.size:
        sub = w.rules.subset([int(p) for p in diff])
        want = oracle.eval_pairs(w.sd, zp, sub, w.sampled, w.S, w.mask)
        assert np.array_equal(ours[diff].view(np.uint64), want.view(np.uint64))
