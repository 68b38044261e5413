"""Parity on short candidate lists, fractional scores and long customer lists.

* Small instances (25, 50 customers) keep most scoring rounds far below 32
  candidates, with lanes idle; rules that read only order-free neighbour
  accumulators (maxima, arg-maxima, the slack minimum, FRAGCNT and the score
  sums REGRET / FRAGSCORE) are mixed with rules that read the ordered ratio
  sums NS, NSTW and NSROB.
* Fractional scores: the score sums are then order-dependent like the ratio
  sums, so any regrouping of REGRET / FRAGSCORE would show.
* A 288-customer instance (H = 1000): decisions with more than 64 candidates,
  ATRISK over long customer lists whose erf arguments overflow one queue.

Each case is compared with the CPU oracle bit for bit.
"""
import dataclasses

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


def mismatches(got, want):
    return int(np.count_nonzero(bits(got).reshape(-1) != bits(want).reshape(-1)))


# Rules that read only order-free scan accumulators (plus ATRISK).
ORDER_FREE = [
    "(+ ATRISK MAXN)",
    "(- SCORE (* REGRET FRAGCNT))",
    "(/ (min TC SCORE) (+ REGRET (- ATRISK FRAGCNT)))",
    "(+ (* FRAGSCORE DOWNSLACK) PBUST)",
    "(- (+ REACH1 REACH3) (* REACH5 REACH2))",
    "(max (- REACH2ROB REGRET) ATRISK)",
    "(* (+ MAXN FRAGCNT) (- DOWNSLACK REGRET))",
]
# Rules that read an ordered ratio sum (NS, NSTW, NSROB).
ORDERED = [
    "(+ NS ATRISK)",
    "(- NSTW REGRET)",
    "(* NSROB MAXN)",
]


def _instance(n, layout, H, seed, m, frac=False):
    sd = SimData.from_instance(parse_solomon_text(generate_instance(n, layout, H, seed)), m=m)
    if frac:
        sd = dataclasses.replace(sd, scores=np.ascontiguousarray(sd.scores + 0.375))
    return sd


def _check(oracle, sd, trees, S=24, seed=7):
    rules = R.pack(trees)
    sampled = R.gen_durations(sd.durations, sd.sigma, S, seed)
    mask = R.term_mask_from(MENU)
    zp = sidr.zstats(sd)
    ctx = sidr.Context(sd, zp)
    try:
        got = ctx.evaluate(rules, sampled, S, mask)
    finally:
        ctx.close()
    want = oracle.eval_pairs(sd, zp, rules, sampled, S, mask)
    return mismatches(got, want), want.size


MENU = workload.MENU29 + ["DOWNSLACK", "ZATRISK", "C1"]


def _menu_ok(trees):
    for t in trees:
        for tok in t.replace("(", " ( ").replace(")", " ").split():
            assert tok == "(" or tok in MENU or tok in R.FUNCTIONS, tok


@pytest.mark.parametrize("n,layout,H,m", [(25, "uniform", 230.0, 2), (50, "clustered", 1000.0, 3),
                                          (100, "mixed", 1000.0, 4)])
def test_short_candidate_lists(oracle, n, layout, H, m):
    trees = ORDER_FREE + ORDERED
    _menu_ok(trees)
    bad, total = _check(oracle, _instance(n, layout, H, 11 + n, m), trees)
    assert bad == 0, f"{bad} of {total} pairs differ"


@pytest.mark.parametrize("n", [25, 100])
def test_fractional_scores(oracle, n):
    trees = ORDER_FREE + ORDERED
    bad, total = _check(oracle, _instance(n, "clustered", 1000.0, 5 + n, 3, frac=True), trees)
    assert bad == 0, f"{bad} of {total} pairs differ"


def test_atrisk_on_288_customers(oracle):
    # 288 customers and H = 1000: decisions with more than 64 candidates
    # (three or more scoring rounds), nine words of customers, and words whose
    # erf arguments overflow the queue in the value rows.
    sd = _instance(288, "uniform", 1000.0, 3, 4)
    trees = ["ATRISK", "(+ ATRISK (* C1 SCORE))", "(- (/ SCORE ATRISK) MAXN)",
             "(min ZATRISK (- TC TA))"]
    _menu_ok(trees)
    bad, total = _check(oracle, sd, trees, S=6)
    assert bad == 0, f"{bad} of {total} pairs differ"


def test_evolved_population_small_instance(oracle):
    # The generation-49 rules (ATRISK, MAXN, FRAGCNT, REGRET, PBUST) on a
    # 50-customer instance: most rounds have few candidates.
    w = workload.evolved(49, P=64, S=1)
    sd = _instance(50, "clustered", 1000.0, 21, 3)
    bad, total = _check(oracle, sd, w.trees[:64], S=16)
    assert bad == 0, f"{bad} of {total} pairs differ"
