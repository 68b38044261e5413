"""Campaign drivers on the B200 evaluator (include/sidr_campaign.h).

Against CPU replicas at small sizes (the host GP sessions stepped with the
oracle's fitness), against the --gate equality of batched and sequential
scoring, and against the reference campaign's own artefacts: its generation
traces (s3_generation/gen_trace.cu output for c101, r101, rc101, pr01), the
held-out gains recorded in them (redeploy sealing), and the head of its
vocabulary-GA log on c101."""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, cuda_available

import sidr
from sidr import campaign, gp
from sidr import rules as R
from sidr import workload
from sidr.instance import SimData

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]

UNIVERSE = ["REGRET", "NSROB", "MAXN", "REACH2", "NSTW", "FRAGCNT", "PBUST", "REACH1", "ATRISK",
            "NFEAS"]


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.uint64)


def campaign_case(name):
    z = np.load(os.path.join(GOLDEN, "campaign.npz"))
    sd = SimData.from_arrays(*[z[f"{name}/inst_{k}"] for k in
                               ("x", "y", "score", "open", "close", "dur", "tmax")], m=3, name=name)
    return sd, float(z[f"{name}/km"][0]), str(z[f"{name}/trace"])


def round_half_even(x, k):
    """engine/jwrite.hpp's decimal rounding."""
    m = 10.0 ** k
    v = x * m
    f = np.floor(v)
    d = v - f
    r = f + 1 if d > 0.5 else (f if d < 0.5 else (f if np.fmod(f, 2.0) == 0.0 else f + 1))
    return r / m


@pytest.fixture(scope="module")
def plain():
    w = workload.plain_eval(P=2, S=1)
    ctx = sidr.Context(w.sd, sidr.zstats(w.sd))
    yield w, ctx
    ctx.close()


def test_gate_batched_equals_sequential(plain):
    w, ctx = plain
    cmp_, bad, mx = campaign.gate(ctx, UNIVERSE, n_seeds=3, n_gens=3, bmax=2, block_n=16,
                                  population=48)
    assert (cmp_, bad, mx) == (15, 0, 0.0)


def replica_scores(oracle, sd, zp, vocab, n_seeds, n_gens, pop, block):
    """batch_score / seq_score for one genome on the CPU: the same GP
    sessions stepped with the oracle's fitness."""
    mask = R.term_mask_from(vocab)
    sessions = [gp.Session(vocab, s, population=pop) for s in range(n_seeds)]

    def fits(gen):
        out = []
        for s, sess in enumerate(sessions):
            smp = gp.gen_durations(sd.durations, 0.2, 1, s * 10000 + gen)
            r = oracle.eval_pairs(sd, zp, sess.packed(), smp, 1, mask)
            out.append(np.array([float(row[0]) for row in r]))
        return out

    for g in range(n_gens):
        f = fits(g)
        if g < n_gens - 1:
            for s in range(n_seeds):
                sessions[s].step(f[s])
    f = fits(n_gens)
    res = []
    for s in range(n_seeds):
        rule = sessions[s].packed().subset([int(np.argmax(f[s]))])
        r = oracle.eval_pairs(sd, zp, rule, block, block.shape[0], mask)[0]
        acc = 0.0
        for v in r:
            acc += float(v)
        res.append(acc / block.shape[0])
    return np.array(res)


def test_batch_score_matches_cpu_replica(plain, oracle):
    w, ctx = plain
    zp = sidr.zstats(w.sd)
    genomes = [0b101, 0b1100000011, 0]
    n_seeds, n_gens, pop, block_n = 2, 2, 24, 8
    got, res = campaign.batch_score(ctx, UNIVERSE, genomes, n_seeds, n_gens, bmax=2,
                                    block_seed=123, block_n=block_n, population=pop)
    block = gp.gen_durations(w.sd.durations, 0.2, block_n, 123)
    for k, g in enumerate(genomes):
        vocab = R.NS_TERMINALS + [UNIVERSE[b] for b in range(len(UNIVERSE)) if g >> b & 1]
        exp = replica_scores(oracle, w.sd, zp, vocab, n_seeds, n_gens, pop, block)
        assert np.array_equal(bits(got[k]), bits(exp)), g
    seq = campaign.seq_score(ctx, UNIVERSE, genomes[1], n_seeds, n_gens, block_seed=123,
                             block_n=block_n, population=pop)
    assert np.array_equal(bits(seq), bits(got[1]))
    assert res.evaluations == len(genomes) * n_seeds * (pop * (n_gens + 1) + block_n)


def test_gen_trace_matches_cpu_replica(plain, oracle):
    w, ctx = plain
    zp = sidr.zstats(w.sd)
    extra = ["REACH2", "ATRISK", "ERC"]
    n_seeds, gens, pop, n_test, km = 2, 3, 24, 8, 150.0
    text, _ = campaign.gen_trace(ctx, "plain", extra, km, n_seeds=n_seeds, n_test=n_test,
                                 test_seed=99, population=pop, generations=gens)
    tr = json.loads(text)
    vocab = R.NS_TERMINALS + extra
    mask = R.term_mask_from(vocab)
    sessions = [gp.Session(vocab, s, population=pop, generations=gens) for s in range(n_seeds)]
    assert tr["instance"] == "plain" and tr["vocab_extra"] == extra
    test = gp.gen_durations(w.sd.durations, 0.2, n_test, 99)
    for g in range(gens + 1):
        for s, sess in enumerate(sessions):
            smp = gp.gen_durations(w.sd.durations, 0.2, 1, s * 10000 + g)
            f = np.array([float(r[0]) for r in oracle.eval_pairs(w.sd, zp, sess.packed(), smp, 1,
                                                                 mask)])
            b = int(np.argmax(f))
            text_b = sess.text()[b]
            if g < gens:
                e = tr["trace"][s][g]
                assert e["g"] == g and e["fit"] == round_half_even(f[b], 1)
                assert e["sz"] == len(R.compile_rule(text_b)[0])
                if g < gens - 1:
                    sess.step(f)
            else:
                fin = tr["finals"][s]
                assert fin["seed"] == s and fin["rule"] == text_b
                r = oracle.eval_pairs(w.sd, zp, sess.packed().subset([b]), test, n_test, mask)[0]
                got = 0.0
                for v in r:
                    got += float(v)
                got /= n_test
                assert fin["gain"] == round_half_even(100.0 * (got - km) / km, 2)


def best_entry(sess, f):
    b = int(np.argmax(f))
    return {"fit": round_half_even(f[b], 1), "sz": len(R.compile_rule(sess.text()[b])[0])}


@pytest.mark.parametrize("name", ["c101", "r101", "rc101", "pr01"])
def test_trace_reproduces_campaign_artefact(name, oracle):
    """The whole generation trace of the reference campaign (30 seeds x 1024
    rules x 51 generations, then the 30 finals on the held-out 1M x 500),
    regenerated and compared entry by entry.

    The reference made these traces with its GPU evaluator built with nvcc's
    default multiply-add contraction (its Makefile passes -O2 without
    -fmad=false), which differs from its CPU simulator on a few priorities,
    so a GP run can take another path there.  A seed that the regenerated
    trace does not follow must be explained: along the seed's trajectory
    this evaluator differs from the reference's GPU build only on rules
    where that build differs from the CPU simulator (the oracle), and there
    it equals the CPU simulator; and the reference's GPU build, driving the
    same GP, reproduces the artefact's trace for that seed."""
    sd, km, expected = campaign_case(name)
    exp = json.loads(expected)
    ctx = sidr.Context(sd, sidr.zstats(sd))
    text, _ = campaign.gen_trace(ctx, name, exp["vocab_extra"], km, n_seeds=30)
    got = json.loads(text)
    assert got["instance"] == exp["instance"] and got["vocab_extra"] == exp["vocab_extra"]
    diverged = {}
    for s in range(30):
        for g, (a, b) in enumerate(zip(got["trace"][s], exp["trace"][s])):
            if a != b:
                diverged[s] = g
                break
        else:
            assert got["finals"][s] == exp["finals"][s], s
    print(name, "seeds off the artefact's path (first generation):", diverged)
    assert len(diverged) <= 3
    if not diverged:
        assert text == expected
        ctx.close()
        return
    from oracle import REF_GPU_SO, ReferenceGPU
    if not os.path.exists(REF_GPU_SO):
        ctx.close()
        pytest.skip("the reference GPU build (oracle/_ref) is absent: divergence not explained")
    ref = ReferenceGPU()
    zp = sidr.zstats(sd)
    vocab = R.NS_TERMINALS + exp["vocab_extra"]
    mask = R.term_mask_from(vocab)
    for s, g_off in diverged.items():
        ours, theirs = gp.Session(vocab, s), gp.Session(vocab, s)
        disagreements = 0
        for g in range(51):
            smp = gp.gen_durations(sd.durations, 0.2, 1, s * 10000 + g)
            if g <= g_off:
                pk = ours.packed()
                f = ctx.evaluate(pk, smp, 1, mask)[:, 0]
                f_ref = ref.evaluate(sd, zp, pk, smp, 1, mask)[:, 0]
                idx = np.nonzero(bits(f) != bits(f_ref))[0]
                if idx.size:
                    cpu = np.array([r[0] for r in oracle.eval_pairs(sd, zp, pk.subset(list(idx)),
                                                                    smp, 1, mask)])
                    assert np.array_equal(bits(f[idx]), bits(cpu)), (s, g, idx)
                    disagreements += idx.size
                assert got["trace"][s][g]["fit"] == best_entry(ours, f)["fit"]
                ours.step(f)
            pt = theirs.packed()
            ft = ref.evaluate(sd, zp, pt, smp, 1, mask)[:, 0]
            e = exp["trace"][s][g]
            assert {"fit": e["fit"], "sz": e["sz"]} == best_entry(theirs, ft), (s, g)
            theirs.step(ft)
        assert disagreements > 0, s
    ctx.close()


@pytest.mark.parametrize("name", ["c101", "r101", "rc101", "pr01"])
def test_redeploy_seals_campaign_traces(name):
    sd, km, text = campaign_case(name)
    ctx = sidr.Context(sd, sidr.zstats(sd))
    r = campaign.redeploy(ctx, name, text, km)
    assert r["sealed"], r
    # every final, not only the best: its recorded gain is reproduced
    tr = json.loads(text)
    mask = R.term_mask_from(R.NS_TERMINALS + tr["vocab_extra"])
    rules = R.pack([f["rule"] for f in tr["finals"]])
    test = gp.gen_durations(sd.durations, 0.2, campaign.TEST_N, campaign.TEST_SEED)
    out = ctx.evaluate(rules, test, campaign.TEST_N, mask)
    for f, row in zip(tr["finals"], out):
        got = 0.0
        for v in row:
            got += float(v)
        got /= campaign.TEST_N
        assert round_half_even(100.0 * (got - km) / km, 2) == f["gain"], f["seed"]
    with pytest.raises(sidr.SidrError):
        campaign.redeploy(ctx, "other", text, km)
    ctx.close()


def test_trace_mean_train_and_choice():
    sd, km, text = campaign_case("c101")
    ctx = sidr.Context(sd, sidr.zstats(sd))
    mt, ho = campaign.trace_mean_train(ctx, text)
    tr = json.loads(text)
    fins = sorted(tr["finals"], key=lambda f: f["seed"])
    rules = R.pack([f["rule"] for f in fins])
    mask = R.term_mask_from(R.NS_TERMINALS + tr["vocab_extra"])
    train = gp.gen_durations(sd.durations, 0.2, campaign.TRAIN_N, campaign.TRAIN_SEED)
    out = ctx.evaluate(rules, train, campaign.TRAIN_N, mask)
    acc = 0.0
    for row in out:
        m = 0.0
        for v in row:
            m += float(v)
        acc += m / campaign.TRAIN_N
    assert bits(mt) == bits(acc / len(fins)) and ho == tr["mean_gain"]
    other = text.replace('"mean_gain": 1.39', '"mean_gain": 2.0')
    rep = campaign.choice(ctx, "c101", [text, other], ["a", "b"])
    assert "CROSS-VALIDATORY CHOICE (train-side): a" in rep
    assert "virtual best (labeled): b -> +2.00 | choice==VBS? False" in rep
    ctx.close()


def test_vocab_ga_head_reproduces_search_log():
    """The first generation of the reference's vocabulary GA on c101
    (universe = the 18-terminal menu, neutral seeds without the full set,
    proxies of 16 seeds x 51 inner generations on the TRAIN block): its
    header and 'gen 0' lines.  The confirmation is cut to one seed, which the
    compared lines do not depend on."""
    sd, _, _ = campaign_case("c101")
    head = [str(x) for x in np.load(os.path.join(GOLDEN, "campaign.npz"))["c101/search_head"]]
    ctx = sidr.Context(sd, sidr.zstats(sd))
    res = campaign.run_ga(R.EXTRA, "c101", ctx=ctx, seeds_neutral=1, nofull=1, gens=1, stag=10,
                          confirm=1, top=1, bmax=13, gp={"generations": 1})
    ctx.close()
    lines = [ln for ln in res.log.split("\n") if not ln.startswith("  batch ")]
    assert lines[0] == head[0].replace("gens 50", "gens 1")
    assert lines[1] == head[1]
