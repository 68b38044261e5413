"""Parity of the CUDA evaluator (through the C-ABI) with the reference: the
golden fixtures, and the CPU oracle on seeded synthetic workloads and edge
cases.  The bar is bit-exact: every per-scenario route score is compared by
its IEEE bit pattern."""
import random

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


def assert_bitexact(got, want, what=""):
    got = np.asarray(got)
    want = np.asarray(want)
    assert got.shape == want.shape, what
    bad = np.nonzero(bits(got).reshape(-1) != bits(want).reshape(-1))[0]
    assert bad.size == 0, f"{what}: {bad.size} of {want.size} differ, first at {bad[:5]}: " \
                          f"{got.reshape(-1)[bad[:5]]} vs {want.reshape(-1)[bad[:5]]}"


@pytest.fixture(scope="module")
def ctx_cache():
    cache = {}
    yield cache
    for c in cache.values():
        c.close()


def ctx_for(cache, key, sd, zp):
    if key not in cache:
        cache[key] = sidr.Context(sd, zp)
    return cache[key]


# ------------------------------------------------------------- golden pins

def test_golden_sim_cases(ctx_cache):
    from test_oracle import SIM_CASES
    for name, sd, rules, mask, zp, sampled, expected in SIM_CASES:
        ctx = ctx_for(ctx_cache, name.split("_")[0], sd, zp)
        out = ctx.evaluate(rules, sampled, sampled.shape[0], mask)
        assert_bitexact(out[0], expected, name)


def test_golden_gp_generations(ctx_cache):
    """6144 fitnesses of verify/golden/gp.txt (ns11 and ext29+rmod)."""
    from test_oracle import load_gp_blocks
    for b, sd, rules, mask, sampled, expected in load_gp_blocks():
        ctx = ctx_for(ctx_cache, "c101gp", sd, sidr.zstats(sd))
        out = ctx.evaluate(rules, sampled, 1, mask)
        assert_bitexact(out[:, 0], expected, b)


# -------------------------------------------------- synthetic vs the oracle

@pytest.mark.parametrize("builder,P,S", [(workload.plain_eval, 96, 12),
                                         (workload.gp_generation, 48, 6)])
def test_workloads_match_oracle(oracle, builder, P, S):
    w = builder(P=P, S=S)
    zp = sidr.zstats(w.sd)
    ctx = sidr.Context(w.sd, zp)
    out = ctx.evaluate(w.rules, w.sampled, w.S, w.mask)
    want = oracle.eval_pairs(w.sd, zp, w.rules, w.sampled, w.S, w.mask)
    assert_bitexact(out, want, w.name)
    ctx.close()


def test_batch_api_and_fitness(oracle):
    w = workload.plain_eval(P=40, S=10)
    zp = sidr.zstats(w.sd)
    ctx = sidr.Context(w.sd, zp)
    b = ctx.batch(w.rules, w.sampled, w.S, w.mask)
    b.run()
    out = b.read()
    want = oracle.eval_pairs(w.sd, zp, w.rules, w.sampled, w.S, w.mask)
    assert_bitexact(out, want, "batch")
    fit = b.fitness()
    ref_fit = np.array([sum(float(v) for v in row) / w.S for row in want])
    assert_bitexact(fit, ref_fit, "fitness")
    b.set_counting(True)
    b.run()
    assert_bitexact(b.read(), want, "counting run")
    c = b.counts()
    assert c["decisions"] > 0 and c["candidates"] > 0 and c["scan_iters"] > 0
    b.run()
    b.run()
    assert_bitexact(b.read(), want, "repeat runs")
    b.close()
    ctx.close()


def test_grouped_and_grouped_masks(oracle):
    w = workload.plain_eval(P=36, S=5)
    zp = sidr.zstats(w.sd)
    ctx = sidr.Context(w.sd, zp)
    G = 3
    grouped = np.concatenate([R.gen_durations(w.sd.durations, 0.2, w.S, 100 * g) for g in range(G)])
    out = ctx.evaluate_grouped(w.rules, grouped, G, w.S, 12, w.mask)
    want = oracle.eval_pairs(w.sd, zp, w.rules, grouped, w.S, w.mask, group_size=12)
    assert_bitexact(out, want, "grouped")
    masks = np.stack([R.term_mask_from(R.NS_TERMINALS), w.mask,
                      R.term_mask_from(R.NS_TERMINALS + ["ATRISK", "REACH5", "PBUST"])])
    out = ctx.evaluate_grouped_masks(w.rules, grouped, G, w.S, 12, 12, masks)
    want = oracle.eval_pairs(w.sd, zp, w.rules, grouped, w.S, masks, group_size=12, mask_group=12)
    assert_bitexact(out, want, "grouped_masks")
    ctx.close()


# ------------------------------------------------------------- all 61 slots

def _all_slot_rules(seed, P, depth):
    names = R.TERM_NAMES + ["ERC"]
    trees = R.ramped_half_and_half(names, R.FUNCS_RMOD, 1, depth, seed, P)
    return R.pack(trees)


def _sum_tree(names):
    if len(names) == 1:
        return names[0]
    mid = len(names) // 2
    return f"(+ {_sum_tree(names[:mid])} {_sum_tree(names[mid:])})"


def test_every_slot_with_random_masks(oracle):
    """Rules over all 61 terminals, ERC constants and rmod, under random masks
    (one per 8 rules) and the all-61 mask, on a Cordeau-sized instance."""
    text = generate_instance(60, "mixed", 1000.0, seed=11)
    sd = SimData.from_instance(parse_solomon_text(text), m=3)
    zp = sidr.zstats(sd)
    rules = _all_slot_rules(3, 64, 5)
    rng = np.random.default_rng(5)
    masks = (rng.random((8, 61)) < 0.5).astype(np.int64)
    masks[0, :] = 1
    sampled = R.gen_durations(sd.durations, 0.2, 4, 77)
    ctx = sidr.Context(sd, zp)
    out = ctx.evaluate_grouped_masks(rules, sampled, 1, 4, 64, 8, masks)
    want = oracle.eval_pairs(sd, zp, rules, sampled, 4, masks, group_size=64, mask_group=8)
    assert_bitexact(out, want, "random masks")
    s61 = R.pack([_sum_tree(R.TERM_NAMES)])
    out = ctx.evaluate(s61, sampled, 4, np.ones(61, dtype=np.int64))
    want = oracle.eval_pairs(sd, zp, s61, sampled, 4, np.ones(61, dtype=np.int64))
    assert_bitexact(out, want, "sum61")
    ctx.close()


# --------------------------------------------------------------- edge cases

def test_edge_priorities_and_degenerate_rules(oracle):
    w = workload.plain_eval(P=1, S=6)
    zp = sidr.zstats(w.sd)
    inf = "2000.0"
    for _ in range(7):  # 2000^128 overflows to +inf
        inf = f"(* {inf} {inf})"
    trees = [
        "SCORE", "0.5", "-1.0", "TA",                       # single leaves and constants
        f"(- {inf} {inf})",                                 # NaN everywhere: nobody is picked
        f"(* {inf} (- TA 30.0))",                           # +inf / -inf / NaN mixed
        f"(/ {inf} SCORE)",                                 # +inf ties: lowest index wins
        f"(- 0.0 {inf})",                                   # -inf everywhere
        "(- SCORE SCORE)",                                  # exact ties at zero
        "(/ SCORE (- TA TA))",                              # protected division
        "(max (min TC TO) (- 0.0 0.0))",                    # signed zeros
        "(rmod (/ SCORE 10.0) (- TC 0.5))",                 # rmod
    ]
    rules = R.pack(trees)
    ctx = sidr.Context(w.sd, zp)
    for mask in (w.mask, np.ones(61, dtype=np.int64), np.zeros(61, dtype=np.int64)):
        out = ctx.evaluate(rules, w.sampled, w.S, mask)
        want = oracle.eval_pairs(w.sd, zp, rules, w.sampled, w.S, mask)
        assert_bitexact(out, want, "edge rules")
    assert np.all(out[4] == 0.0)
    # empty batches
    empty = R.pack_compiled([])
    assert ctx.evaluate(empty, w.sampled, w.S, w.mask).shape == (0, w.S)
    assert ctx.evaluate(rules, w.sampled[:0], 0, w.mask).shape == (rules.P, 0)
    ctx.close()


def test_zero_vehicles_and_tiny_instances(oracle):
    for n, m in ((1, 2), (2, 1), (5, 0), (33, 4)):
        text = generate_instance(n, "uniform", 230.0, seed=n)
        sd = SimData.from_instance(parse_solomon_text(text), m=m)
        zp = sidr.zstats(sd)
        w_rules = _all_slot_rules(n, 16, 4)
        sampled = R.gen_durations(sd.durations, 0.2, 3, 5)
        mask = np.ones(61, dtype=np.int64)
        ctx = sidr.Context(sd, zp)
        out = ctx.evaluate(w_rules, sampled, 3, mask)
        want = oracle.eval_pairs(sd, zp, w_rules, sampled, 3, mask)
        assert_bitexact(out, want, f"n={n} m={m}")
        if m == 0:
            assert np.all(out == 0.0)
        ctx.close()


def test_coincident_customers(oracle):
    """Customers sharing coordinates (zero distances): the coincident-location
    skips of the NS family and the structural search."""
    inst = parse_solomon_text(generate_instance(40, "clustered", 1000.0, seed=3, n_clusters=3))
    rng = random.Random(4)
    for k in range(1, 12):
        src = inst.pois[rng.randrange(1, 41)]
        dst = inst.pois[rng.randrange(1, 41)]
        dst.x, dst.y = src.x, src.y
    inst.pois[7].x, inst.pois[7].y = 50.0, 50.0  # on the depot
    sd = SimData.from_instance(inst, m=3)
    zp = sidr.zstats(sd)
    rules = _all_slot_rules(9, 48, 4)
    sampled = R.gen_durations(sd.durations, 0.2, 4, 9)
    mask = np.ones(61, dtype=np.int64)
    ctx = sidr.Context(sd, zp)
    out = ctx.evaluate(rules, sampled, 4, mask)
    want = oracle.eval_pairs(sd, zp, rules, sampled, 4, mask)
    assert_bitexact(out, want, "coincident")
    ctx.close()


@pytest.mark.parametrize("n", [288, 512])
def test_large_instances(oracle, n):
    """Multi-word visited bitmasks up to the MAX_N limit."""
    sd = SimData.from_instance(parse_solomon_text(generate_instance(n, "mixed", 1000.0, seed=n)),
                               m=4)
    zp = sidr.zstats(sd)
    trees = R.ramped_half_and_half(workload.MENU29, R.FUNCTIONS, 2, 4, n, 6)
    rules = R.pack(trees)
    sampled = R.gen_durations(sd.durations, 0.2, 2, 3)
    mask = R.term_mask_from(R.NS_TERMINALS + ["REGRET", "MAXN", "REACH2", "SAT", "NFEAS"])
    ctx = sidr.Context(sd, zp)
    out = ctx.evaluate(rules, sampled, 2, mask)
    want = oracle.eval_pairs(sd, zp, rules, sampled, 2, mask)
    assert_bitexact(out, want, f"n={n}")
    ctx.close()


def test_invalid_inputs_fail_without_launch():
    w = workload.plain_eval(P=4, S=2)
    ctx = sidr.Context(w.sd, sidr.zstats(w.sd))
    before = sidr.kernel_launches()
    bad = w.sampled.copy()
    bad[1, 3] = np.inf
    with pytest.raises(sidr.SidrError) as e:
        ctx.evaluate(w.rules, bad, w.S, w.mask)
    assert e.value.status == 7
    with pytest.raises(sidr.SidrError) as e:
        ctx.evaluate_grouped(w.rules, w.sampled, 1, 1, 2, w.mask)  # needs 2 groups
    assert e.value.status == 1
    r = R.pack_compiled([([-1, 7], [0, 0, 0, 0])])
    with pytest.raises(sidr.SidrError):
        ctx.evaluate(r, w.sampled, w.S, w.mask)
    assert sidr.kernel_launches() == before
    ctx.close()


def test_kernel_guard_raises_error_word(oracle):
    """The kernel's rule-record guard, tripped on purpose by launching a batch
    with slices too small for its rules (sidr_batch_guard_check): the launch
    refuses every rule, raises the error word, and the host reports
    SIDR_ERR_KERNEL; reading that launch's scores reports it too; the next
    ordinary launch clears the word and gives the oracle's scores."""
    w = workload.plain_eval(P=12, S=3)
    zp = sidr.zstats(w.sd)
    ctx = sidr.Context(w.sd, zp)
    b = ctx.batch(w.rules, w.sampled, w.S, w.mask)
    for _ in range(2):
        assert b.guard_check() == 6  # SIDR_ERR_KERNEL
        with pytest.raises(sidr.SidrError) as e:
            b.read()
        assert e.value.status == 6 and "shared-memory slice" in str(e.value)
    b.run()
    assert_bitexact(b.read(), oracle.eval_pairs(w.sd, zp, w.rules, w.sampled, w.S, w.mask), "after")
    b.close()
    ctx.close()


def test_rmod_heavy_rules_match_oracle(oracle):
    """rmod (opcode 6, pow(max(a, 0), 1 + clip(b, 0, 1)), engine/sim_core.hpp:
    30-35) runs on glibc's pow restated for the device, so rules built from it
    give the CPU simulator's scores by construction: 256 rules of depth 2-6
    over the 29-terminal menu with ERC constants and rmod among the
    functions, every one of which applies rmod, on 40 scenarios of the
    GP-generation instance."""
    w = workload.gp_generation(P=1, S=40)
    pool = R.ramped_half_and_half(workload.MENU29 + ["ERC"], R.FUNCS_RMOD, 2, 6, 77, 1200)
    trees = [t for t in pool if "rmod" in R.to_prefix(t)][:256]
    assert len(trees) == 256
    rules = R.pack(trees)
    mask = R.term_mask_from(workload.MENU29 + ["ERC"])
    zp = sidr.zstats(w.sd)
    ctx = sidr.Context(w.sd, zp)
    out = ctx.evaluate(rules, w.sampled, w.S, mask)
    ctx.close()
    assert_bitexact(out, oracle.eval_pairs(w.sd, zp, rules, w.sampled, w.S, mask), "rmod rules")


def test_rmod_last_bit_rules_match_oracle(oracle):
    """Rules in which the last bit of pow(x, 2.0) decides the route (rmod with
    the regime clipped to 1, minus x * x): the restated pow gives the CPU
    simulator's routes."""
    w = workload.gp_generation(P=1, S=300)
    mask = R.term_mask_from(workload.MENU29 + ["ERC"])
    rules = R.pack([f"(- (rmod {t} 1.5) (* {t} {t}))" for t in ("NSTW", "TFV", "BOLSAO", "HARVEST")])
    zp = sidr.zstats(w.sd)
    ctx = sidr.Context(w.sd, zp)
    out = ctx.evaluate(rules, w.sampled, w.S, mask)
    ctx.close()
    assert_bitexact(out, oracle.eval_pairs(w.sd, zp, rules, w.sampled, w.S, mask), "rmod last bit")
