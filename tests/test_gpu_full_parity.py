"""Parity at the benchmark's own sizes: every evaluated (rule, scenario) pair
against the C oracle (the CPU simulator, sim_batch of engine/sim_host.hpp:
67-83, on all host threads), bit for bit.

* the plain CPU-runnable evaluation in full: 256 rules x 500 scenarios of the
  uniform 100-customer instance (H = 230, m = 4) through sidr_evaluate --
  128,000 route simulations, the sweep verify/verify_cuda.cu:107-149 makes on
  its own golden cases;
* the uneven 40-instance layout (25/50/100/288 customers, three layouts,
  m 2-4, H 230/1000, rules of log-uniform length 3-255) in one multi-instance
  launch, with every instance compared, not a sample of them;
* an evolved population of the benchmark GP run (generation 49), whose rules
  lean on ATRISK and keep routes alive for 80 decisions.
"""
import numpy as np
import pytest

from conftest import cuda_available

import sidr
from sidr import workload

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.uint64)


def mismatches(got, want):
    return int(np.count_nonzero(bits(got).reshape(-1) != bits(want).reshape(-1)))


def test_plain_eval_full_size(oracle):
    w = workload.plain_eval()
    assert (w.rules.P, w.S) == (256, 500)
    zp = sidr.zstats(w.sd)
    ctx = sidr.Context(w.sd, zp)
    got = ctx.evaluate(w.rules, w.sampled, w.S, w.mask)
    ctx.close()
    want = oracle.eval_pairs(w.sd, zp, w.rules, w.sampled, w.S, w.mask)
    assert got.shape == (256, 500)
    bad = mismatches(got, want)
    assert bad == 0, f"{bad} of {want.size} pairs differ"
    # per-rule fitness (engine/gp_engine.cu:76-81): sums of integer scores
    assert np.array_equal(bits(got.sum(axis=1) / 500), bits(want.sum(axis=1) / 500))


def test_uneven_batch_every_instance(oracle):
    mw = workload.batched_uneven(K=40, rules_per_instance=16, S=6)
    zps = [sidr.zstats(sd) for sd in mw.sds]
    m = sidr.Multi(mw.sds, zps, mw.rules, mw.sampled, mw.S, mw.masks)
    m.run()
    got = m.read()
    m.close()
    sizes = set()
    for k in range(len(mw.sds)):
        want = oracle.eval_pairs(mw.sds[k], zps[k], mw.rules[k], mw.sampled[k], mw.S, mw.masks[k])
        assert mismatches(got[k], want) == 0, f"instance {k} (n = {mw.sds[k].n})"
        sizes.add(mw.sds[k].n)
    assert sizes == {25, 50, 100, 288}


def test_evolved_population_matches_oracle(oracle):
    w = workload.evolved(49, P=1024, S=500)
    idx = list(range(0, 1024, 32))  # 32 rules x 40 scenarios: the oracle's share stays small
    sub = w.rules.subset(idx)
    zp = sidr.zstats(w.sd)
    ctx = sidr.Context(w.sd, zp)
    got = ctx.evaluate(sub, w.sampled[:40], 40, w.mask)
    ctx.close()
    want = oracle.eval_pairs(w.sd, zp, sub, w.sampled[:40], 40, w.mask)
    assert mismatches(got, want) == 0
