"""The seed-batched GP driver (sidr_gp_run_batched, the reference's
exhaust_batched) on the B200 evaluator, against a CPU replica: the same GP
sessions stepped with the oracle's fitness."""
import numpy as np
import pytest

from conftest import cuda_available

import sidr
from sidr import gp
from sidr import rules as R
from sidr import workload

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.uint64)


def test_run_batched_matches_cpu_replica(oracle):
    w = workload.plain_eval(P=2, S=1)
    zp = sidr.zstats(w.sd)
    terms = workload.MENU29
    n_seeds, first_seed, T, gens, pop, test_n = 3, 5, 2, 3, 48, 16
    cfg = dict(population=pop, generations=gens, train_samples=T, test_samples=test_n)
    ctx = sidr.Context(w.sd, zp)
    res = gp.run_batched(ctx, terms, w.mask, n_seeds, first_seed=first_seed, test_seed=777, **cfg)
    ctx.close()

    sessions = [gp.Session(terms, first_seed + s, **cfg) for s in range(n_seeds)]

    def fit_all(gen):
        out = []
        for s, sess in enumerate(sessions):
            smp = gp.gen_durations(w.sd.durations, 0.2, T, (first_seed + s) * 10000 + gen)
            r = oracle.eval_pairs(w.sd, zp, sess.packed(), smp, T, w.mask)
            out.append(np.array([sum(float(v) for v in row) / T for row in r]))
        return out

    for g in range(gens):
        fits = fit_all(g)
        for s in range(n_seeds):
            assert res.best_train[g, s] == fits[s].max(), (g, s)
        if g < gens - 1:
            for s in range(n_seeds):
                sessions[s].step(fits[s])
    fits = fit_all(gens)
    test = gp.gen_durations(w.sd.durations, 0.2, test_n, 777)
    for s in range(n_seeds):
        bi = int(np.argmax(fits[s]))  # first maximum, as the reference's strict >
        rule = sessions[s].packed().subset([bi])
        assert res.best_rules[s] == sessions[s].text()[bi]
        held = oracle.eval_pairs(w.sd, zp, rule, test, test_n, w.mask)[0]
        assert bits(res.best_test[s]) == bits(sum(float(v) for v in held) / test_n)
    assert res.evaluations == gens * n_seeds * pop * T + n_seeds * pop * T + n_seeds * test_n


def test_run_multi_equals_run_batched_per_instance():
    """Three instances of uneven size (25, 50 and 288 customers), two seeds
    each, evolved through one multi-instance launch per generation: every
    instance's best train fitness per generation, best rules and held-out
    scores equal the seed-batched driver's on that instance alone."""
    mw = workload.batched_uneven(K=4, rules_per_instance=1, S=1)
    sds = [mw.sds[0], mw.sds[1], mw.sds[3]]
    assert [sd.n for sd in sds] == [25, 50, 288]
    zps = [sidr.zstats(sd) for sd in sds]
    masks = [mw.masks[0]] * 3
    terms = workload.MENU29
    cfg = dict(population=32, generations=3, train_samples=3, test_samples=8)
    multi = gp.run_multi(sds, zps, terms, masks, 2, first_seed=11, test_seed=4321, shape=1, **cfg)
    auto = gp.run_multi(sds[:2], zps[:2], terms, masks[:2], 2, first_seed=11, test_seed=4321,
                        shape=-1, **cfg)
    for k, (sd, zp) in enumerate(zip(sds, zps)):
        ctx = sidr.Context(sd, zp)
        one = gp.run_batched(ctx, terms, masks[k], 2, first_seed=11, test_seed=4321, **cfg)
        ctx.close()
        assert np.array_equal(bits(multi.best_train[:, k, :]), bits(one.best_train)), k
        assert np.array_equal(bits(multi.best_test[k]), bits(one.best_test)), k
        assert multi.best_rules[2 * k:2 * k + 2] == one.best_rules, k
        if k < 2:
            assert np.array_equal(bits(auto.best_test[k]), bits(one.best_test)), k
    assert multi.evaluations == 3 * 2 * 32 * 3 * (3 + 1) + 3 * 2 * 8


def test_batched_checkpoint_resumes_exactly(tmp_path):
    """The seed-batched run stepped, checkpointed to a file, restored in a new
    object (after the first object is gone) and finished gives run_batched's
    results bit for bit, from a checkpoint taken before any generation, in the
    middle and after the last; malformed checkpoints and checkpoints of
    another instance are refused."""
    w = workload.plain_eval(P=2, S=1)
    zp = sidr.zstats(w.sd)
    terms = workload.MENU29
    n_seeds, first_seed, gens = 2, 3, 5
    cfg = dict(population=40, generations=gens, train_samples=3, test_samples=12)
    ctx = sidr.Context(w.sd, zp)
    try:
        full = gp.run_batched(ctx, terms, w.mask, n_seeds, first_seed=first_seed, test_seed=99, **cfg)
        for cut in (0, 2, gens):
            b = gp.Batched(ctx, terms, w.mask, n_seeds, first_seed=first_seed, test_seed=99, **cfg)
            b.step(cut)
            assert b.generation == cut
            path = tmp_path / f"run{cut}.ckpt"
            path.write_text(b.checkpoint())
            b.close()
            r = gp.Batched.restore(ctx, path.read_text())
            assert r.generation == cut
            assert r.checkpoint() == path.read_text()
            r.step(gens)  # stops at the last generation
            assert r.generation == gens
            res = r.finish()
            r.close()
            assert np.array_equal(bits(res.best_train), bits(full.best_train)), cut
            assert np.array_equal(bits(res.best_test), bits(full.best_test)), cut
            assert res.best_rules == full.best_rules, cut
            assert res.evaluations == full.evaluations, cut
        # refusals
        b = gp.Batched(ctx, terms, w.mask, n_seeds, first_seed=first_seed, test_seed=99, **cfg)
        b.step(1)
        text = b.checkpoint()
        with pytest.raises(sidr.SidrError):
            b.finish()  # generations left
        b.close()
        for broken in (text[: len(text) // 2], text.replace("generation 1\n", "generation 2\n"),
                       text.replace("sidr-gp-batched-checkpoint 1", "sidr-gp-batched-checkpoint 9"),
                       text + "extra\n"):
            with pytest.raises(sidr.SidrError):
                gp.Batched.restore(ctx, broken)
    finally:
        ctx.close()
    other = workload.gp_generation(P=1, S=1)
    ctx2 = sidr.Context(other.sd, sidr.zstats(other.sd))
    try:
        with pytest.raises(sidr.SidrError):
            gp.Batched.restore(ctx2, text)
    finally:
        ctx2.close()
