"""Pair groups of 16 and 8 lanes: the evaluator's block shapes that run two or
four (rule, scenario) pairs per warp give the CPU oracle's scores bit for bit.

* Single-instance shapes (sidr.Batch.SHAPES, 16 lanes per pair in shapes 2 and
  3) on instances of 1, 2, 5 (no vehicles), 25, 33 (a partial second word of
  customers), 50, 288 and 512 customers, with rules over all 61 terminals,
  ERC constants and rmod under the all-61 mask, and with ATRISK-heavy rules
  under the 29-terminal menu.
* Multi-instance batches: each size class of instances runs in its own launch
  with its own shape (8, 16 or 32 lanes per pair, in any assignment), every
  instance compared with the oracle; per-class tuning picks a timed shape for
  each class that has rules, and the graph replay keeps the scores.
"""
import numpy as np
import pytest

from conftest import cuda_available

import sidr
from sidr import rules as R
from sidr import workload
from sidr.instance import SimData, generate_instance, parse_solomon_text

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.uint64)


def _instance(n, layout, H, seed, m):
    return SimData.from_instance(parse_solomon_text(generate_instance(n, layout, H, seed)), m=m)


ATRISK_RULES = ["ATRISK", "(+ ATRISK (* C1 SCORE))", "(- (/ SCORE ATRISK) MAXN)",
                "(min ZATRISK (- TC TA))", "(- NSTW REGRET)", "(* NSROB MAXN)"]


@pytest.mark.parametrize("n,m,layout,H", [(1, 2, "uniform", 230.0), (2, 1, "uniform", 230.0),
                                          (5, 0, "uniform", 230.0), (25, 2, "uniform", 230.0),
                                          (33, 4, "clustered", 1000.0), (50, 3, "mixed", 1000.0),
                                          (288, 4, "uniform", 1000.0), (512, 4, "mixed", 1000.0)])
def test_every_single_instance_shape(oracle, n, m, layout, H):
    sd = _instance(n, layout, H, 40 + n, m)
    zp = sidr.zstats(sd)
    S = 2 if n >= 288 else 4
    cases = [
        (R.pack(R.ramped_half_and_half(R.TERM_NAMES + ["ERC"], R.FUNCS_RMOD, 1, 4, n, 12)),
         np.ones(61, dtype=np.int64)),
        (R.pack(ATRISK_RULES), R.term_mask_from(workload.MENU29 + ["DOWNSLACK", "ZATRISK", "C1"])),
    ]
    sampled = R.gen_durations(sd.durations, sd.sigma, S, 3 + n)
    ctx = sidr.Context(sd, zp)
    try:
        for rules, mask in cases:
            want = oracle.eval_pairs(sd, zp, rules, sampled, S, mask)
            for shape in range(len(sidr.Batch.SHAPES)):
                ctx.set_shape(shape)
                got = ctx.evaluate(rules, sampled, S, mask)
                assert np.array_equal(bits(got), bits(want)), f"n={n} shape {sidr.Batch.SHAPES[shape]}"
    finally:
        ctx.close()


def test_class_shapes_and_class_tuning(oracle):
    mw = workload.batched_uneven(K=8, rules_per_instance=10, S=2)
    zps = [sidr.zstats(sd) for sd in mw.sds]
    want = [oracle.eval_pairs(sd, zp, r, smp, mw.S, mk)
            for sd, zp, r, smp, mk in zip(mw.sds, zps, mw.rules, mw.sampled, mw.masks)]
    m = sidr.Multi(mw.sds, zps, mw.rules, mw.sampled, mw.S, mw.masks)
    try:
        _, counts = m.shapes()
        # 25, 50, 100 and 288 customers: every class has two instances' rules
        assert counts == [20, 20, 20, 20]
        for assign in ([4, 3, 0, 1], [3, 4, 2, 0], [4, 4, 4, 4], [3, 3, 3, 3]):
            for c, sh in enumerate(assign):
                m.set_class_shape(c, sh)
            assert m.shapes()[0] == assign
            m.run()
            for k, got in enumerate(m.read()):
                assert np.array_equal(bits(got), bits(want[k])), (assign, k, mw.sds[k].n)
        chosen, ms = m.autotune_classes(stride=2, reps=1)
        assert m.shapes()[0] == chosen
        for c in range(len(sidr.Multi.CLASSES)):
            assert 0 <= chosen[c] < len(sidr.Multi.SHAPES)
            assert all(t > 0 for t in ms[c]) and ms[c][chosen[c]] == min(ms[c])
        m.capture()
        for _ in range(2):
            m.run()
            for k, got in enumerate(m.read()):
                assert np.array_equal(bits(got), bits(want[k])), ("graph", k)
    finally:
        m.close()


def test_class_tuning_reports_empty_classes():
    # 288-customer instances only: the three smaller classes have no rules
    mw = workload.large_combined(K=1, seeds=1, rules_per_seed=4, S=2)
    zps = [sidr.zstats(sd) for sd in mw.sds]
    m = sidr.Multi(mw.sds, zps, mw.rules, mw.sampled, mw.S, mw.masks)
    try:
        assert m.shapes()[1] == [0, 0, 0, 4]
        chosen, ms = m.autotune_classes(stride=1, reps=1)
        assert chosen[:3] == [-1, -1, -1] and 0 <= chosen[3] < len(sidr.Multi.SHAPES)
        assert all(t == -1 for c in range(3) for t in ms[c])
        with pytest.raises(sidr.SidrError):
            m.set_class_shape(len(sidr.Multi.CLASSES), 0)
        with pytest.raises(sidr.SidrError):
            m.set_class_shape(0, len(sidr.Multi.SHAPES))
    finally:
        m.close()
