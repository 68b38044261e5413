"""Decision-situation capture, phenotypes and the surrogate-assisted GP on
the GPU (include/sidr_surrogate.h).

* capture: at every recorded decision, the rule's priorities recomputed from
  the captured terminal tables pick the customer the evaluator chose, the
  chosen customers' scores add up to the evaluator's rollout score, and the
  first decision's base terminals (SCORE..RemT at the depot, time 0) match a
  direct computation from the instance;
* phenotype: the kernel's ranks against a Python restatement;
* the driver with plain breeding equals the seed-batched GP driver
  generation by generation, and with the surrogate its reported fitness is
  simulated;
* the gain: offspring the trained model ranks highest are fitter, when
  simulated, than offspring picked at random."""
import math

import numpy as np
import pytest

from conftest import cuda_available

import sidr
from sidr import gp as GP
from sidr import rules as R
from sidr import surrogate as SG
from sidr import workload

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]


def eval_tree(ops, args, t):
    st = []
    for k, o in enumerate(ops):
        if o == -1:
            st.append(t[args[2 * k]])
        elif o == -2:
            st.append(args[2 * k] / 1000.0)
        else:
            b = st.pop()
            a = st.pop()
            if o == 0:
                r = a + b
            elif o == 1:
                r = a - b
            elif o == 2:
                r = a * b
            elif o == 3:
                r = 1.0 if abs(b) < 1e-10 else a / b
            elif o == 4:
                r = a if a < b else b
            elif o == 5:
                r = a if a > b else b
            else:
                raise ValueError("rmod not used here")
            st.append(r)
    v = st[0]
    return -1e300 if v != v else v


@pytest.fixture(scope="module")
def setup():
    w = workload.gp_generation(P=64, S=8)
    ctx = sidr.Context(w.sd, sidr.zstats(w.sd))
    yield w, ctx
    ctx.close()


def test_capture_reproduces_the_decisions(setup):
    w, ctx = setup
    for p in (0, 5, 17):
        rule = w.rules.subset([p])
        ops, args = rule.rule(0)
        terms, cust, info = SG.capture_situations(ctx, rule, w.sampled, w.mask, 80, 100)
        scores = ctx.evaluate(rule, w.sampled, w.S, w.mask)[0]
        sd = w.sd
        for s in range(w.S):
            total = 0.0
            for d in range(80):
                nc, chosen = info[s, d]
                if nc == 0:
                    continue
                pri = [eval_tree(ops, args, terms[s, d, c]) for c in range(nc)]
                best, bp = -1, -1e300
                for c in range(nc):
                    if pri[c] > bp:
                        bp, best = pri[c], c
                assert (cust[s, d, best] if best >= 0 else -1) == chosen, (p, s, d)
                if chosen >= 0:
                    total += sd.scores[chosen]
                if d == 0:  # at the depot at time 0
                    for c in range(nc):
                        i = cust[s, d, c]
                        ta = sd.dist[i + 1]
                        t = terms[s, d, c]
                        assert t[0] == sd.scores[i] and t[1] == sd.durations[i]
                        assert t[2] == sd.open_t[i] - 0.0 and t[3] == sd.close_t[i] - 0.0
                        assert t[4] == ta and t[5] == sd.dist_to_depot[i]
            assert np.array_equal(np.float64(total), scores[s]), (p, s)


def test_phenotype_matches_restatement(setup):
    w, ctx = setup
    smp = GP.gen_durations(w.sd.durations, 0.2, 16, 77)
    terms, cust, info = SG.capture_situations(ctx, w.rules.subset([3]), smp, w.mask, 64, 64)
    picks = [(s, d) for s in range(16) for d in range(64)
             if 2 <= info[s, d, 0] <= 64 and info[s, d, 1] >= 0]
    rng = np.random.default_rng(1)
    sel = [picks[i] for i in rng.choice(len(picks), 32, replace=False)]
    sit = np.stack([terms[s, d] for s, d in sel])
    nc = np.array([info[s, d, 0] for s, d in sel], np.int32)
    ref = np.array([list(cust[s, d, :info[s, d, 0]]).index(info[s, d, 1]) for s, d in sel], np.int32)
    feats = SG.phenotype(w.rules, sit, nc, ref)
    assert feats.shape == (w.rules.P, 40)
    for p in range(w.rules.P):
        ops, args = w.rules.rule(p)
        for j in range(32):
            pri = [eval_tree(ops, args, sit[j, c]) for c in range(nc[j])]
            pos = sum(1 for c in range(nc[j]) if c != ref[j] and
                      (pri[c] > pri[ref[j]] or (pri[c] == pri[ref[j]] and c < ref[j])))
            assert feats[p, j] == np.float32(pos / (nc[j] - 1)), (p, j)
        assert feats[p, 32] == np.float32(len(ops) / 255.0)


def test_plain_driver_equals_batched_gp(setup):
    w, ctx = setup
    cfg = dict(population=64, generations=4, train_samples=4, test_samples=16)
    plain = SG.sgp_run(ctx, workload.MENU29, w.mask, seed=3, test_seed=555, gp=cfg, use_surrogate=0)
    ref = GP.run_batched(ctx, workload.MENU29, w.mask, 1, first_seed=3, test_seed=555, **cfg)
    assert np.array_equal(plain["best_train"], ref.best_train[:, 0])
    assert plain["screened"] == 0 and plain["fallback"] == 0


def test_surrogate_run_reports_simulated_fitness(setup):
    w, ctx = setup
    cfg = dict(population=64, generations=5, train_samples=4, test_samples=16)
    res = SG.sgp_run(ctx, workload.MENU29, w.mask, seed=3, test_seed=555, gp=cfg, screen=512,
                     audit=32, train_steps=30, batch=128, rho_min=-1.0, capture_scenarios=4)
    assert res["screened"] == 4 and res["fallback"] == 0
    assert all(math.isfinite(r) for r in res["rho"][:4]) and math.isnan(res["rho"][4])
    # the last held-out score is the simulated score of the reported rule
    rule = R.pack([res["best_rule"]])
    test = GP.gen_durations(w.sd.durations, 0.2, 16, 555)
    out = ctx.evaluate(rule, test, 16, w.mask)[0]
    acc = 0.0
    for v in out:
        acc += float(v)
    assert acc / 16 == res["held_out"][-1]
    # a threshold no audit can reach: every generation breeds plainly
    res2 = SG.sgp_run(ctx, workload.MENU29, w.mask, seed=3, test_seed=555, gp=cfg, screen=512,
                      audit=32, train_steps=5, batch=128, rho_min=2.0, capture_scenarios=4)
    assert res2["screened"] == 0 and res2["fallback"] == 4


def test_mixed_screening_with_rank_targets(setup):
    """Half the slots screened (one child per situation ranking), the model
    trained on rank scores: every generation is screened, the reported
    fitness is still simulated, and settings out of range are refused."""
    w, ctx = setup
    cfg = dict(population=64, generations=4, train_samples=4, test_samples=16)
    res = SG.sgp_run(ctx, workload.MENU29, w.mask, seed=5, test_seed=556, gp=cfg, screen=512,
                     audit=32, train_steps=30, batch=128, rho_min=-1.0, capture_scenarios=4,
                     target=1, screen_fraction=0.5, distinct=1)
    assert res["screened"] == 3 and res["fallback"] == 0
    rule = R.pack([res["best_rule"]])
    test = GP.gen_durations(w.sd.durations, 0.2, 16, 556)
    out = ctx.evaluate(rule, test, 16, w.mask)[0]
    acc = 0.0
    for v in out:
        acc += float(v)
    assert acc / 16 == res["held_out"][-1]
    for bad in (dict(screen_fraction=1.5), dict(target=2), dict(selection=3), dict(distinct=2)):
        with pytest.raises(sidr.SidrError):
            SG.sgp_run(ctx, workload.MENU29, w.mask, seed=5, test_seed=556, gp=cfg, screen=512,
                       audit=32, **bad)


def test_screening_gain_over_random_offspring(setup):
    """Train the model on three simulated generations of one GP run, then
    take 4096 offspring bred by four other runs (their third generation):
    the 512 the model ranks highest have a higher simulated mean fitness than
    512 drawn at random."""
    w, ctx = setup
    smp = GP.gen_durations(w.sd.durations, 0.2, 16, 78)
    terms_, cust, info = SG.capture_situations(ctx, w.rules.subset([3]), smp, w.mask, 64, 64)
    picks = [(s, d) for s in range(16) for d in range(64)
             if 2 <= info[s, d, 0] <= 64 and info[s, d, 1] >= 0]
    rng = np.random.default_rng(4)
    sel = [picks[i] for i in rng.choice(len(picks), 32, replace=False)]
    sit = np.stack([terms_[s, d] for s, d in sel])
    nc = np.array([info[s, d, 0] for s, d in sel], np.int32)
    ref = np.array([list(cust[s, d, :info[s, d, 0]]).index(info[s, d, 1]) for s, d in sel], np.int32)
    block = GP.gen_durations(w.sd.durations, 0.2, 16, 4242)

    def run(seed, gens):
        sess = GP.Session(workload.MENU29, seed, population=1024)
        hist = []
        for g in range(gens):
            pk = sess.packed()
            f = ctx.evaluate(pk, block, 16, w.mask).mean(axis=1)
            hist.append((pk, f))
            sess.step(f)
        return sess, hist

    _, hist = run(5, 3)
    X = np.concatenate([SG.phenotype(pk, sit, nc, ref) for pk, _ in hist])
    Y = np.concatenate([f for _, f in hist])
    m = SG.MLP(seed=2)
    m.train(X, (Y - Y.mean()) / Y.std(), steps=200, batch=1024, lr=1e-3, seed=1)
    pool = [run(100 + k, 2)[0].packed() for k in range(4)]
    cand = R.pack_compiled([o.rule(i) for o in pool for i in range(o.P)])
    pred = m.predict(SG.phenotype(cand, sit, nc, ref))
    true = ctx.evaluate(cand, block, 16, w.mask).mean(axis=1)
    top = np.argsort(-pred, kind="stable")[:512]
    rand = rng.choice(cand.P, 512, replace=False)
    rk = lambda v: np.argsort(np.argsort(v))  # noqa: E731
    rho = np.corrcoef(rk(pred), rk(true))[0, 1]
    print("top-predicted mean", true[top].mean(), "random mean", true[rand].mean(), "rho", rho)
    assert true[top].mean() > true[rand].mean()
    m.close()


def _small_cfg():
    gp = dict(population=64, generations=4, train_samples=12, test_samples=20)
    sg = dict(screen=256, audit=24, train_steps=12, batch=128, history=2)
    return gp, sg


def test_sgp_multi_single_population_is_sgp_run():
    """With one instance and one seed the combined driver is sidr_sgp_run,
    value for value (the model's training is deterministic, and the
    multi-instance launch gives the single-instance scores)."""
    w = workload.gp_generation(P=1, S=1)
    zp = sidr.zstats(w.sd)
    gp, sg = _small_cfg()
    ctx = sidr.Context(w.sd, zp)
    one = SG.sgp_run(ctx, workload.MENU29, w.mask, seed=3, test_seed=1000000, gp=gp, **sg)
    ctx.close()
    multi = SG.sgp_run_multi([w.sd], [zp], workload.MENU29, [w.mask], 1, first_seed=3,
                             test_seed=1000000, shape=0, gp=gp, **sg)
    assert np.array_equal(multi["best_train"][:, 0, 0], one["best_train"])
    assert np.array_equal(multi["held_out"][:, 0, 0], one["held_out"])
    r1, r2 = multi["rho"][:, 0, 0], one["rho"]
    assert np.array_equal(np.isnan(r1), np.isnan(r2)) and np.array_equal(r1[~np.isnan(r1)], r2[~np.isnan(r2)])
    assert (multi["screened"], multi["fallback"]) == (one["screened"], one["fallback"])


def test_sgp_multi_matches_cpu_simulator(oracle):
    """The large combined run's driver at reduced counts: two 288-customer
    instances (12-cluster and uniform layouts, m = 4, H = 1000) x two GP seeds,
    surrogate screening on; the final best rule of every population, scored by
    the C oracle on its instance's held-out block, gives the driver's held-out
    score bit for bit, and the run is the same when repeated."""
    mw = workload.large_combined(K=2, seeds=1, rules_per_seed=1, S=1)
    zps = [sidr.zstats(sd) for sd in mw.sds]
    gp, sg = _small_cfg()
    runs = [SG.sgp_run_multi(mw.sds, zps, workload.MENU29, mw.masks, 2, first_seed=5,
                             test_seed=1000000, shape=-1, gp=gp, **sg) for _ in range(2)]
    a, b = runs
    for key in ("best_train", "held_out"):
        assert np.array_equal(a[key], b[key]), key
    assert a["best_rules"] == b["best_rules"]
    assert a["screened"] + a["fallback"] == 2 * 2 * (gp["generations"] - 1)
    for e, text in enumerate(a["best_rules"]):
        k = e // 2
        sd = mw.sds[k]
        rules = R.pack([text])
        test = R.gen_durations(sd.durations, sd.sigma, gp["test_samples"], 1000000)
        cpu = oracle.eval_pairs(sd, zps[k], rules, test, gp["test_samples"], mw.masks[k])
        assert cpu.sum() / gp["test_samples"] == a["held_out"][-1, k, e % 2], e


def _bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.uint64)


def test_surrogate_checkpoint_resumes_exactly(setup, tmp_path):
    """sidr_sgp_run_resumable: a run stopped after two generations (and
    again after one more), each time resumed from its checkpoint file in a
    new call, gives the uninterrupted run's outputs bit for bit -- model
    weights, Adam moments, history window, situations and GP state all come
    back exactly.  A checkpoint written with other settings is refused."""
    w, ctx = setup
    cfg = dict(population=64, generations=5, train_samples=4, test_samples=16)
    kw = dict(screen=512, audit=32, train_steps=30, batch=128, rho_min=0.3, capture_scenarios=4)
    full = SG.sgp_run(ctx, workload.MENU29, w.mask, seed=7, test_seed=557, gp=cfg, **kw)
    path = tmp_path / "sgp.ckpt"
    part = SG.sgp_run(ctx, workload.MENU29, w.mask, seed=7, test_seed=557, gp=cfg, checkpoint=path,
                      every=1, stop_after=2, **kw)
    assert not part["finished"] and path.exists()
    assert np.array_equal(_bits(part["best_train"][:2]), _bits(full["best_train"][:2]))
    part = SG.sgp_run(ctx, workload.MENU29, w.mask, seed=7, test_seed=557, gp=cfg, checkpoint=path,
                      every=1, stop_after=1, **kw)
    assert not part["finished"]
    with pytest.raises(sidr.SidrError):  # another seed
        SG.sgp_run(ctx, workload.MENU29, w.mask, seed=8, test_seed=557, gp=cfg, checkpoint=path, **kw)
    with pytest.raises(sidr.SidrError):  # another audit size
        SG.sgp_run(ctx, workload.MENU29, w.mask, seed=7, test_seed=557, gp=cfg, checkpoint=path,
                   **{**kw, "audit": 16})
    done = SG.sgp_run(ctx, workload.MENU29, w.mask, seed=7, test_seed=557, gp=cfg, checkpoint=path,
                      every=1, **kw)
    assert done["finished"]
    for key in ("best_train", "held_out", "rho"):
        assert np.array_equal(_bits(done[key]), _bits(full[key])), key
    assert done["best_rule"] == full["best_rule"]
    assert (done["screened"], done["fallback"], done["evaluations"]) == \
        (full["screened"], full["fallback"], full["evaluations"])
    assert full["screened"] + full["fallback"] == 4


def test_combined_run_checkpoint_resumes_exactly(tmp_path):
    """sidr_sgp_run_multi_resumable on two instances (50 and 100 customers) x
    two seeds: stopped after one generation and resumed from the checkpoint
    file in a new call, the run gives the uninterrupted run's outputs bit for
    bit (every population's GP session, each instance's model and fitness
    window come back); a checkpoint of other seeds is refused."""
    mw = workload.batched_uneven(K=3, rules_per_instance=1, S=1)
    sds, masks = mw.sds[1:3], mw.masks[1:3]
    zps = [sidr.zstats(sd) for sd in sds]
    gp, sg = _small_cfg()
    kw = dict(first_seed=2, test_seed=31, shape=0, gp=gp, **sg)
    full = SG.sgp_run_multi(sds, zps, workload.MENU29, masks, 2, **kw)
    path = tmp_path / "multi.ckpt"
    part = SG.sgp_run_multi(sds, zps, workload.MENU29, masks, 2, checkpoint=path, every=1,
                            stop_after=1, **kw)
    assert not part["finished"] and path.exists()
    with pytest.raises(sidr.SidrError):
        SG.sgp_run_multi(sds, zps, workload.MENU29, masks, 2, checkpoint=path,
                         **{**kw, "first_seed": 3})
    done = SG.sgp_run_multi(sds, zps, workload.MENU29, masks, 2, checkpoint=path, every=2, **kw)
    assert done["finished"]
    for key in ("best_train", "held_out", "rho"):
        assert np.array_equal(_bits(done[key]), _bits(full[key])), key
    assert done["best_rules"] == full["best_rules"]
    assert (done["screened"], done["fallback"], done["evaluations"]) == \
        (full["screened"], full["fallback"], full["evaluations"])
