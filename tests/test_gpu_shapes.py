"""Block shapes of the single-instance evaluator (sidr_batch_set_shape,
sidr_batch_autotune_sampled, sidr_ctx_set_shape): every shape gives the
scores of the CPU oracle bit for bit, and tuning picks a valid shape and
leaves the batch's results unchanged."""
import numpy as np
import pytest

from conftest import cuda_available

import sidr
from sidr import workload

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.uint64)


def test_every_shape_matches_oracle(oracle):
    w = workload.evolved(49, P=48, S=1)
    base = workload.gp_generation(P=1, S=12)
    zp = sidr.zstats(base.sd)
    want = oracle.eval_pairs(base.sd, zp, w.rules, base.sampled, 12, base.mask)
    ctx = sidr.Context(base.sd, zp)
    try:
        for shape in range(len(sidr.Batch.SHAPES)):
            ctx.set_shape(shape)
            got = ctx.evaluate(w.rules, base.sampled, 12, base.mask)
            assert np.array_equal(bits(got), bits(want)), f"shape {shape}"
            b = ctx.batch(w.rules, base.sampled, 12, base.mask)
            b.set_shape(shape)
            b.run()
            assert np.array_equal(bits(b.read()), bits(want)), f"batch shape {shape}"
            b.close()
    finally:
        ctx.close()


def test_autotune_picks_a_shape_and_keeps_results():
    w = workload.gp_generation(P=128, S=40)
    ctx = sidr.Context(w.sd, sidr.zstats(w.sd))
    try:
        b = ctx.batch(w.rules, w.sampled, w.S, w.mask)
        b.run()
        before = b.read()
        shape, ms = b.autotune_sampled(stride=8, reps=1)
        assert shape in range(len(sidr.Batch.SHAPES))
        assert len(ms) == len(sidr.Batch.SHAPES) and all(t > 0 for t in ms)
        assert ms[shape] == min(ms)
        b.run()
        assert np.array_equal(bits(b.read()), bits(before))
        b.close()
        with pytest.raises(sidr.SidrError):
            ctx.set_shape(len(sidr.Batch.SHAPES))
    finally:
        ctx.close()
