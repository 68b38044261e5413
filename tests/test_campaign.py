"""Campaign drivers on the host (include/sidr_campaign.h): the prefix-rule
compiler against the rule compiler pinned to the reference's compile_rmod,
and the vocabulary GA's host logic (s4_selection/ga.cu:288-523) against the
oracle's restatement, driven by a synthetic fitness so that no GPU is
needed."""
import pytest

import sidr
from sidr import campaign
from sidr import rules as R

import vocab_ga

UNIVERSE = ["REGRET", "NSROB", "MAXN", "REACH2", "NSTW", "FRAGCNT", "PBUST", "REACH1", "ATRISK",
            "NFEAS"]


# ---------------------------------------------------------- prefix compiler

def test_compile_prefix_matches_rule_compiler():
    trees = R.ramped_half_and_half(R.NS_TERMINALS + R.EXTRA + ["ERC"], R.FUNCS_RMOD, 1, 6, 3, 400)
    for t in trees:
        text = R.to_prefix(t)
        ops, args = campaign.compile_prefix(text)
        eo, ea = R.compile_rule(text)
        assert list(ops) == list(eo), text
        assert list(args) == list(ea), text


def test_compile_prefix_errors_and_aliases():
    ops, args = campaign.compile_prefix("(+ D2D (* SLACK 0.5))")
    assert list(ops) == [-1, -1, -2, 2, 0]
    assert list(args) == [5, 0, 8, 0, 500, 0, 1, 2, 0, 3]
    for bad in ("(+ SCORE)", "(pow SCORE DUR)", "(+ SCORE DUR", "(+ SCORE DUR) TA", ")"):
        with pytest.raises(sidr.SidrError):
            campaign.compile_prefix(bad)


# ------------------------------------------------------------ vocabulary GA

def synthetic(weights, seed_slope=0.25, gen_slope=0.125):
    """A fitness with ties: weighted bit sums (multiples of 0.5) plus exact
    per-seed and per-generation offsets."""
    def fit(genomes, n, ng):
        out = []
        for g in genomes:
            base = sum(w for b, w in enumerate(weights) if g >> b & 1)
            out.append([base + seed_slope * s + gen_slope * ng for s in range(n)])
        return out
    return fit


def strip_timing(log):
    return [ln for ln in log.split("\n") if not ln.startswith("  batch ") and
            not ln.startswith("PERF ")][:-1]


CASES = [
    dict(weights=[3, -1, 2, 0.5, 1, -2, 0, 1.5, -0.5, 2.5], kw=dict()),
    dict(weights=[1, 1, 1, 1, 1, 1, 1, 1, 1, 1], kw=dict(seeds_neutral=1, gens=12, stag=3)),
    dict(weights=[0.5, -3, 2, 2, 0, 0, 1, -1, 4, 0.5],
         kw=dict(seeds_neutral=1, nofull=1, pm=1.5, top=3, bmax=4, ga_seed=7)),
    dict(weights=[2, 0, -1, 1, 0.5, 0, 0, 0, 3, -2], kw=dict(gens=30, stag=8, proxy=3, confirm=5)),
]


@pytest.mark.parametrize("case", range(len(CASES)))
def test_vocab_ga_matches_restatement(case):
    c = CASES[case]
    fit = synthetic(c["weights"])
    kw = dict(c["kw"])
    res = campaign.run_ga(UNIVERSE, "inst7", fitness=fit, gp={"generations": 9}, **kw)
    ref_kw = dict(pgens=kw.get("pgens", 51), proxy=kw.get("proxy", 16),
                  confirm=kw.get("confirm", 30), gens=kw.get("gens", 50), stag_k=kw.get("stag", 5),
                  bmax=kw.get("bmax", 10), top_n=kw.get("top", 4), pm_mult=kw.get("pm", 0.5),
                  seed_mode="neutral" if kw.get("seeds_neutral") else "random",
                  nofull=bool(kw.get("nofull")), cgens=9, ga_seed=kw.get("ga_seed", 20260714))
    champ, mean, evals, lines, _ = vocab_ga.run_ga(UNIVERSE, fit, instance="inst7", **ref_kw)
    assert strip_timing(res.log) == lines
    assert (res.champion, res.champion_mean, res.evals) == (champ, mean, evals)


def test_vocab_ga_small_universe_reinjects():
    uni = ["REGRET", "NSROB", "MAXN"]
    fit = synthetic([1, 0, -1])
    res = campaign.run_ga(uni, "tiny", fitness=fit, gens=10, stag=20)
    champ, mean, evals, lines, _ = vocab_ga.run_ga(uni, fit, instance="tiny", gens=10, stag_k=20)
    assert "  reinject 2" in lines
    assert strip_timing(res.log) == lines
    assert res.champion == champ


def test_vocab_ga_cache_file_roundtrip(tmp_path):
    fit = synthetic(CASES[0]["weights"])
    path = str(tmp_path / "ga.cache")
    calls = []

    def counted(gs, n, ng):
        calls.append(len(gs))
        return fit(gs, n, ng)

    r1 = campaign.run_ga(UNIVERSE, "inst7", fitness=counted, cache_path=path, gens=6)
    _, _, _, lines1, cache_text = vocab_ga.run_ga(UNIVERSE, fit, instance="inst7", gens=6,
                                                  cache=True)
    assert strip_timing(r1.log) == lines1
    assert open(path).read() == cache_text
    first = sum(calls)
    # a relaunch retraces the same genomes: every batch is a hit
    calls.clear()
    r2 = campaign.run_ga(UNIVERSE, "inst7", fitness=counted, cache_path=path, gens=6)
    assert sum(calls) == 0 < first
    _, _, _, lines2, cache2 = vocab_ga.run_ga(UNIVERSE, fit, instance="inst7", gens=6,
                                              preload=cache_text)
    assert strip_timing(r2.log) == [ln.replace("CACHE", path) for ln in lines2]
    assert r2.champion == r1.champion
    assert open(path).read() == cache2
    # another setting changes the header: the file is discarded
    calls.clear()
    campaign.run_ga(UNIVERSE, "inst7", fitness=counted, cache_path=path, gens=6, proxy=8)
    assert sum(calls) > 0
    assert open(path).read().split("\n")[0].endswith("proxy=8 pgens=51 confirm=30 cgens=51")


def test_vocab_ga_rejects_bad_settings():
    fit = synthetic([1] * 3)
    with pytest.raises(sidr.SidrError):
        campaign.run_ga(["REGRET", "BOGUS"], "x", fitness=fit)
    with pytest.raises(sidr.SidrError):
        campaign.run_ga(["REGRET"], "x", fitness=fit, stag=0)
    with pytest.raises(sidr.SidrError):
        campaign.run_ga(["REGRET"] * 31, "x", fitness=fit)
    with pytest.raises(sidr.SidrError):
        campaign.run_ga(["REGRET"], "x")  # no evaluator and no callback

    def broken(gs, n, ng):
        raise ValueError("fitness failed")

    with pytest.raises(ValueError):
        campaign.run_ga(["REGRET", "NSROB"], "x", fitness=broken)
