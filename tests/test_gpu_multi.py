"""Multi-instance batches (sidr_multi_*): instances of uneven size in one
persistent launch give, rule for rule, the scores of per-instance evaluation,
under every compiled block shape, after autotuning, and replayed as a CUDA
graph."""
import numpy as np
import pytest

from conftest import cuda_available

import sidr
from sidr import workload

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.uint64)


def test_multi_matches_per_instance(oracle):
    mw = workload.batched_uneven(K=8, rules_per_instance=24, S=3)
    zps = [sidr.zstats(sd) for sd in mw.sds]
    want = []
    for sd, zp, r, smp, mk in zip(mw.sds, zps, mw.rules, mw.sampled, mw.masks):
        ctx = sidr.Context(sd, zp)
        want.append(ctx.evaluate(r, smp, mw.S, mk))
        ctx.close()
    # spot check against the oracle on the 288-customer instance
    k = 3
    assert mw.sds[k].n == 288
    assert np.array_equal(bits(want[k]), bits(oracle.eval_pairs(
        mw.sds[k], zps[k], mw.rules[k], mw.sampled[k], mw.S, mw.masks[k])))
    m = sidr.Multi(mw.sds, zps, mw.rules, mw.sampled, mw.S, mw.masks)
    for shape in range(len(sidr.Multi.SHAPES)):
        m.set_shape(shape)
        m.run()
        for k, got in enumerate(m.read()):
            assert np.array_equal(bits(got), bits(want[k])), (shape, k)
    chosen, ms = m.autotune(reps=1)
    assert 0 <= chosen < len(ms) and all(t > 0 for t in ms)
    chosen, ms = m.autotune_sampled(stride=4, reps=1)  # timed on every 4th rule of the work order
    assert 0 <= chosen < len(ms) and all(t > 0 for t in ms)
    m.run()
    for k, got in enumerate(m.read()):
        assert np.array_equal(bits(got), bits(want[k])), ("after sampled tuning", k)
    m.capture()
    for _ in range(2):
        m.run()
        for k, got in enumerate(m.read()):
            assert np.array_equal(bits(got), bits(want[k])), ("graph", k)
    m.close()


def test_large_combined_shape_matches_oracle(oracle):
    """The large combined run's batch at reduced counts: 288-customer
    instances (12-cluster and uniform layouts), m = 4, H = 1000, the initial
    populations of three GP seeds per instance, all in one launch, bit for
    bit against the C oracle."""
    mw = workload.large_combined(K=2, seeds=3, rules_per_seed=6, S=3)
    zps = [sidr.zstats(sd) for sd in mw.sds]
    m = sidr.Multi(mw.sds, zps, mw.rules, mw.sampled, mw.S, mw.masks)
    m.run()
    got = m.read()
    m.close()
    for k in range(2):
        want = oracle.eval_pairs(mw.sds[k], zps[k], mw.rules[k], mw.sampled[k], mw.S, mw.masks[k])
        assert np.array_equal(bits(got[k]), bits(want)), k


def test_multi_rejects_bad_layouts():
    mw = workload.batched_uneven(K=2, rules_per_instance=2, S=2)
    zps = [sidr.zstats(sd) for sd in mw.sds]
    short = [mw.sampled[0], mw.sampled[1][:1]]  # instance 1 lacks a scenario
    with pytest.raises(sidr.SidrError):
        sidr.Multi(mw.sds, zps, mw.rules, short, mw.S, mw.masks)
