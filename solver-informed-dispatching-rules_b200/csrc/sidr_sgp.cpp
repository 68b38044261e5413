// sidr_sgp.cpp -- the surrogate-assisted GP driver (include/sidr_surrogate.h):
// the GP of sidr_gp_core.hpp whose offspring are pre-screened by the MLP of
// sidr_surrogate.cu on their phenotypes, with the evaluator as the judge of
// every fitness and plain breeding whenever the model's audit rank
// correlation is too low.
#include <chrono>
#include <cmath>
#include <numeric>
#include <set>

#include "../../include/sidr_surrogate.h"
#include "sidr_gp_core.hpp"
#include "sidr_sgp_select.hpp"

using namespace sidr::gp;
using sidr::sgp::best_distinct;
using sidr::sgp::preselect;
using sidr::sgp::spearman;
using sidr::sgp::training_targets;

namespace {

double now_s() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

struct Packed {
    std::vector<int32_t> ops, args, off, len;
    sidr_rules_desc desc() {
        return sidr_rules_desc{ops.data(), args.data(), off.data(), len.data(), (int32_t)off.size(),
                               (int64_t)ops.size()};
    }
};

void pack_rules(const std::vector<Rule>& rules, const Vocab& v, Packed& pk) {
    for (const Rule& r : rules) {
        pk.off.push_back((int32_t)pk.ops.size());
        size_t k = 0;
        compile_at(r, k, v, pk.ops, pk.args, pk.ops.size());
        pk.len.push_back((int32_t)pk.ops.size() - pk.off.back());
    }
}


// The surrogate state of one instance: its decision situations, its model
// and the window of simulated fitness (all of its seeds) the model trains on.
struct InstanceSurrogate {
    std::vector<double> sit_terms;
    std::vector<int32_t> sit_nc, sit_ref;
    sidr_mlp* model = nullptr;
    std::vector<std::vector<float>> hist_x;
    std::vector<std::vector<double>> hist_t;
    InstanceSurrogate() = default;
    InstanceSurrogate(const InstanceSurrogate&) = delete;
    InstanceSurrogate& operator=(const InstanceSurrogate&) = delete;
    ~InstanceSurrogate() {
        if (model) sidr_mlp_destroy(model);
    }
};

// Decision situations of one instance: rollouts of `rule` on
// capture_scenarios scenarios (base seed seed*10000 + 7777), NS decisions of 2
// .. max_cand candidates drawn with Mt19937(seed*7919 + 17) -- the sampling of
// sidr_sgp_run.
sidr_status capture_for(sidr_ctx* ctx, const sidr_instance_desc* inst, const int64_t* mask,
                        const sidr_sgp_config* sc, uint64_t seed, Packed& rule, InstanceSurrogate& out) {
    const int n = inst->n, NS = sc->n_situations;
    sidr_rules_desc r = rule.desc();
    const int S = sc->capture_scenarios, D = 64, C = sc->max_cand;
    std::vector<double> smp((size_t)S * n), cap_terms((size_t)S * D * C * 61);
    std::vector<int32_t> cap_cust((size_t)S * D * C), cap_info((size_t)S * D * 2);
    sidr_gen_durations(n, inst->durations, 0.2, S, (long long)seed * 10000 + 7777, smp.data());
    sidr_status st = sidr_capture_situations(ctx, &r, smp.data(), S, mask, D, C, cap_terms.data(),
                                             cap_cust.data(), cap_info.data());
    if (st != SIDR_OK) return st;
    std::vector<int> pool;
    for (int q = 0; q < S * D; q++)
        if (cap_info[2 * q] >= 2 && cap_info[2 * q] <= C && cap_info[2 * q + 1] >= 0) pool.push_back(q);
    if ((int)pool.size() < NS) return gp_fail(SIDR_ERR_INVALID, "too few decision situations captured");
    Mt19937 srng(seed * 7919 + 17);
    const std::vector<size_t> pick = srng.sample(pool.size(), (size_t)NS);
    out.sit_terms.assign((size_t)NS * C * 61, 0.0);
    for (int j = 0; j < NS; j++) {
        const int q = pool[pick[j]];
        const int nc = cap_info[2 * q], chosen = cap_info[2 * q + 1];
        int ref = -1;
        for (int c = 0; c < nc; c++)
            if (cap_cust[(size_t)q * C + c] == chosen) ref = c;
        if (ref < 0) return gp_fail(SIDR_ERR_KERNEL, "captured choice not among the candidates");
        std::copy(cap_terms.begin() + (size_t)q * C * 61, cap_terms.begin() + (size_t)(q + 1) * C * 61,
                  out.sit_terms.begin() + (size_t)j * C * 61);
        out.sit_nc.push_back(nc);
        out.sit_ref.push_back(ref);
    }
    return SIDR_OK;
}

}  // namespace

extern "C" {

void sidr_sgp_default_config(sidr_sgp_config* c) {
    if (!c) return;
    c->screen = 8192;
    c->train_steps = 200;
    c->batch = 1024;
    c->lr = 1e-3f;
    c->audit = 128;
    c->rho_min = 0.8;
    c->history = 3;
    c->n_situations = SIDR_MLP_INPUTS - 8;
    c->capture_scenarios = 16;
    c->max_cand = 64;
    c->model_seed = 1;
    c->use_surrogate = 1;
    c->device = 0;
    c->selection = 0;
    c->target = 1;
    c->screen_fraction = 1.0;
    c->distinct = 1;
}

sidr_status sidr_sgp_run(sidr_ctx* ctx, const sidr_instance_desc* inst, const sidr_gp_config* cfg,
                         const sidr_sgp_config* sc, const char* terminals_csv, const int64_t* mask,
                         uint64_t seed, int64_t test_seed, double* best_train, double* held_out,
                         double* rho, double* gen_seconds, char* best_rule, int64_t rule_cap,
                         sidr_sgp_result* result) {
    std::string err;
    if (!ctx || !inst || !sc || !mask) return gp_fail(SIDR_ERR_INVALID, "null argument");
    if (!valid_config(cfg, err)) return gp_fail(SIDR_ERR_INVALID, err);
    if (sc->n_situations + 8 != SIDR_MLP_INPUTS)
        return gp_fail(SIDR_ERR_INVALID, "n_situations + 8 must equal the model's 40 inputs");
    if (sc->screen < cfg->population || sc->audit < 3 || sc->history < 1 || sc->batch < 1 ||
        sc->capture_scenarios < 1 || sc->max_cand < 2 || cfg->test_samples < 1)
        return gp_fail(SIDR_ERR_INVALID, "surrogate settings out of range");
    if (sc->selection < 0 || sc->selection > 1 || sc->target < 0 || sc->target > 1 ||
        !(sc->screen_fraction >= 0.0 && sc->screen_fraction <= 1.0) || sc->distinct < 0 || sc->distinct > 1)
        return gp_fail(SIDR_ERR_INVALID, "selection, target, screen_fraction or distinct out of range");
    std::vector<std::string> terms;
    if (!parse_terminals(terminals_csv, terms, err)) return gp_fail(SIDR_ERR_INVALID, err);
    const int n = inst->n, ps = cfg->population, T = cfg->train_samples, G = cfg->generations;
    const int NS = sc->n_situations, NF = SIDR_MLP_INPUTS;
    const double t_start = now_s();
    double t_eval = 0.0, t_model = 0.0;
    int64_t evals = 0;
    int screened = 0, fallback = 0;

    Gp gp(*cfg, seed);
    gp.vocab.terminals = terms;
    gp.vocab.n_funcs = cfg->with_rmod ? 7 : 6;
    gp.init();

    auto simulate = [&](const std::vector<Rule>& rules, long long block_seed, int S,
                        std::vector<double>& fit) -> sidr_status {
        Packed pk;
        pack_rules(rules, gp.vocab, pk);
        std::vector<double> smp((size_t)S * n);
        sidr_gen_durations(n, inst->durations, 0.2, S, block_seed, smp.data());
        sidr_rules_desc r = pk.desc();
        std::vector<double> out((size_t)r.P * S);
        const double t0 = now_s();
        const sidr_status st = sidr_evaluate(ctx, &r, smp.data(), S, mask, out.data());
        t_eval += now_s() - t0;
        evals += (int64_t)r.P * S;
        if (st != SIDR_OK) return gp_fail(st, std::string("evaluation: ") + sidr_last_error());
        fit.assign(r.P, 0.0);
        for (int p = 0; p < r.P; p++) {
            double acc = 0.0;
            for (int s = 0; s < S; s++) acc += out[(size_t)p * S + s];
            fit[p] = acc / S;
        }
        return SIDR_OK;
    };

    // decision situations and the model (created on first use)
    std::vector<double> sit_terms;
    std::vector<int32_t> sit_nc, sit_ref;
    sidr_mlp* model = nullptr;
    struct ModelGuard {
        sidr_mlp*& m;
        ~ModelGuard() {
            if (m) sidr_mlp_destroy(m);
        }
    } guard{model};
    auto features_of = [&](const std::vector<Rule>& rules, std::vector<float>& f) -> sidr_status {
        Packed pk;
        pack_rules(rules, gp.vocab, pk);
        sidr_rules_desc r = pk.desc();
        f.assign((size_t)r.P * NF, 0.0f);
        const double t0 = now_s();
        const sidr_status st = sidr_phenotype(&r, sit_terms.data(), sit_nc.data(), sit_ref.data(), NS,
                                              sc->max_cand, sc->device, f.data());
        t_model += now_s() - t0;
        return st;
    };
    std::vector<std::vector<float>> hist_x;
    std::vector<std::vector<double>> hist_t;

    std::vector<double> fit;
    for (int g = 0; g < G; g++) {
        sidr_status st = simulate(gp.pop, (long long)seed * 10000 + g, T, fit);
        if (st != SIDR_OK) return st;
        size_t bi = 0;
        for (size_t p = 1; p < fit.size(); p++)
            if (fit[p] > fit[bi]) bi = p;
        if (best_train) best_train[g] = fit[bi];
        {
            std::vector<double> ho;
            if ((st = simulate({gp.pop[bi]}, test_seed, cfg->test_samples, ho)) != SIDR_OK) return st;
            if (held_out) held_out[g] = ho[0];
        }
        if (rho) rho[g] = std::nan("");
        if (sc->use_surrogate && g == 0) {
            // situations from the first generation's best rule
            Packed pk;
            pack_rules({gp.pop[bi]}, gp.vocab, pk);
            InstanceSurrogate cap;
            const double t0 = now_s();
            st = capture_for(ctx, inst, mask, sc, seed, pk, cap);
            t_eval += now_s() - t0;
            if (st != SIDR_OK) return st;
            sit_terms.swap(cap.sit_terms);
            sit_nc.swap(cap.sit_nc);
            sit_ref.swap(cap.sit_ref);
            if ((st = sidr_mlp_create(sc->device, sc->model_seed, &model)) != SIDR_OK) return st;
        }
        if (sc->use_surrogate) {
            std::vector<float> f;
            if ((st = features_of(gp.pop, f)) != SIDR_OK) return st;
            hist_x.push_back(f);
            hist_t.push_back(fit);
        }
        if (g < G - 1) {
            bool screened_gen = false;
            if (sc->use_surrogate) {
                while ((int)hist_x.size() > sc->history * 2) {  // population + audit entries per generation
                    hist_x.erase(hist_x.begin());
                    hist_t.erase(hist_t.begin());
                }
                // train on the recent simulated fitness: standardised, or as
                // uniform scores of its ranks over the whole history
                std::vector<float> X;
                std::vector<double> all;
                for (size_t h = 0; h < hist_x.size(); h++) {
                    X.insert(X.end(), hist_x[h].begin(), hist_x[h].end());
                    all.insert(all.end(), hist_t[h].begin(), hist_t[h].end());
                }
                std::vector<float> Y = training_targets(all, sc->target);
                float loss = 0.0f;
                double t0 = now_s();
                st = sidr_mlp_train(model, X.data(), Y.data(), (int32_t)Y.size(), sc->train_steps, sc->batch,
                                    sc->lr, seed * 131 + g, &loss);
                t_model += now_s() - t0;
                if (st != SIDR_OK) return st;
                // screen: breed `screen` candidates, predict, audit a random sample
                std::vector<Rule> cand = gp.breed(fit, (size_t)sc->screen);
                std::vector<float> cf;
                if ((st = features_of(cand, cf)) != SIDR_OK) return st;
                std::vector<float> pred(cand.size());
                t0 = now_s();
                st = sidr_mlp_predict(model, cf.data(), (int32_t)cand.size(), pred.data());
                t_model += now_s() - t0;
                if (st != SIDR_OK) return st;
                const std::vector<size_t> aud = gp.rng.sample(cand.size(), (size_t)sc->audit);
                std::vector<Rule> aud_rules;
                for (size_t a : aud) aud_rules.push_back(cand[a]);
                std::vector<double> aud_fit;
                if ((st = simulate(aud_rules, (long long)seed * 10000 + g, T, aud_fit)) != SIDR_OK) return st;
                std::vector<double> aud_pred;
                std::vector<float> aud_x;
                for (size_t a : aud) {
                    aud_pred.push_back(pred[a]);
                    aud_x.insert(aud_x.end(), cf.begin() + a * NF, cf.begin() + (a + 1) * NF);
                }
                const double r_s = spearman(aud_pred, aud_fit);
                if (rho) rho[g] = r_s;
                hist_x.push_back(aud_x);
                hist_t.push_back(aud_fit);
                if (r_s >= sc->rho_min) {
                    // elites of the current population, then the screened offspring
                    std::vector<int> order(ps);
                    std::iota(order.begin(), order.end(), 0);
                    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return fit[a] > fit[b]; });
                    std::vector<Rule> next;
                    for (int e = 0; e < cfg->elitism && e < ps; e++) next.push_back(gp.pop[order[e]]);
                    const int slots = ps - (int)next.size();
                    const int need = (int)std::lround(sc->screen_fraction * slots);
                    std::vector<int> pick;
                    if (sc->selection == 1) {
                        // pre-selection: the best-predicted child of each group of
                        // screen/need consecutive (independently bred) children
                        pick = preselect(pred, need);
                    } else if (sc->distinct == 1) {
                        // the best-predicted children, one per ranking of the decision situations
                        pick = best_distinct<std::vector<float>>(pred, (size_t)need, [&](int c) {
                            return std::vector<float>(cf.begin() + (size_t)c * NF, cf.begin() + (size_t)c * NF + NS);
                        });
                    } else {
                        // the best-predicted distinct children
                        pick = best_distinct<Rule>(pred, (size_t)need, [&](int c) { return cand[c]; });
                    }
                    for (int c : pick) next.push_back(cand[c]);
                    if ((int)next.size() < ps) {
                        // the slots left to plain breeding
                        std::vector<Rule> plain = gp.breed(fit, (size_t)(ps - (int)next.size()));
                        for (Rule& r : plain) next.push_back(std::move(r));
                    }
                    gp.pop.swap(next);
                    screened_gen = true;
                    screened++;
                } else {
                    fallback++;
                }
            }
            if (!screened_gen) gp.step(fit);
        }
        if (gen_seconds) gen_seconds[g] = now_s() - t_start;
    }
    // the last generation's best rule
    size_t bi = 0;
    for (size_t p = 1; p < fit.size(); p++)
        if (fit[p] > fit[bi]) bi = p;
    std::string text;
    size_t k = 0;
    prefix_at(gp.pop[bi], k, gp.vocab, text);
    if (best_rule && rule_cap > (int64_t)text.size()) std::memcpy(best_rule, text.c_str(), text.size() + 1);
    if (result) {
        result->eval_seconds = t_eval;
        result->model_seconds = t_model;
        result->host_seconds = now_s() - t_start - t_eval - t_model;
        result->evaluations = evals;
        result->generations_screened = screened;
        result->generations_fallback = fallback;
    }
    return SIDR_OK;
}

}  // extern "C"


// ----------------------------------------------------------------------------
// Many instances x many seeds (sidr_sgp_run_multi).

extern "C" sidr_status sidr_sgp_run_multi(const sidr_instance_desc* insts, const double* zps, int32_t K,
                                          const sidr_gp_config* cfg, const sidr_sgp_config* sc,
                                          const char* terminals_csv, const int64_t* masks, int32_t n_seeds,
                                          int64_t first_seed, int64_t test_seed, int32_t shape,
                                          double* best_train, double* held_out, double* rho,
                                          char* best_rules, int64_t rules_cap, sidr_sgp_result* result) {
    std::string err;
    if (!insts || !zps || !masks || !sc) return gp_fail(SIDR_ERR_INVALID, "null argument");
    if (K < 1 || n_seeds < 1) return gp_fail(SIDR_ERR_INVALID, "K < 1 or n_seeds < 1");
    if ((int64_t)K * n_seeds > 16383) return gp_fail(SIDR_ERR_INVALID, "K * n_seeds > 16383");
    if (shape < -1 || shape >= SIDR_MULTI_SHAPES) return gp_fail(SIDR_ERR_INVALID, "shape out of range");
    if (!valid_config(cfg, err)) return gp_fail(SIDR_ERR_INVALID, err);
    if (sc->n_situations + 8 != SIDR_MLP_INPUTS)
        return gp_fail(SIDR_ERR_INVALID, "n_situations + 8 must equal the model's 40 inputs");
    if (sc->screen < cfg->population || sc->audit < 3 || sc->history < 1 || sc->batch < 1 ||
        sc->capture_scenarios < 1 || sc->max_cand < 2 || cfg->test_samples < 1)
        return gp_fail(SIDR_ERR_INVALID, "surrogate settings out of range");
    if (sc->selection < 0 || sc->selection > 1 || sc->target < 0 || sc->target > 1 ||
        !(sc->screen_fraction >= 0.0 && sc->screen_fraction <= 1.0) || sc->distinct < 0 || sc->distinct > 1)
        return gp_fail(SIDR_ERR_INVALID, "selection, target, screen_fraction or distinct out of range");
    for (int k = 0; k < K; k++)
        if (insts[k].n < 1 || !insts[k].durations)
            return gp_fail(SIDR_ERR_INVALID, "instance " + std::to_string(k) + ": no customers or no durations");
    std::vector<std::string> terms;
    if (!parse_terminals(terminals_csv, terms, err)) return gp_fail(SIDR_ERR_INVALID, err);
    const int S = n_seeds, E = K * S, ps = cfg->population, T = cfg->train_samples, G = cfg->generations;
    const int NS = sc->n_situations, NF = SIDR_MLP_INPUTS;
    const double t_start = now_s();
    double t_eval = 0.0, t_model = 0.0;
    int64_t evals = 0;
    int screened = 0, fallback = 0, chosen = shape;

    // population e = k * S + s: instance k, GP seed first_seed + s
    std::vector<Gp> gps;
    gps.reserve(E);
    for (int e = 0; e < E; e++) {
        gps.emplace_back(*cfg, (uint64_t)(first_seed + e % S));
        gps.back().vocab.terminals = terms;
        gps.back().vocab.n_funcs = cfg->with_rmod ? 7 : 6;
        gps.back().init();
    }
    auto seed_of = [&](int e) { return (long long)(first_seed + e % S); };

    // One multi-instance launch: rule sets[q] of population q (its leaf labels
    // are interned in that population's own vocabulary) on instance inst_of[q]
    // with the scenario block blocks[q] of Tn scenarios; per-rule means.
    auto simulate = [&](const std::vector<const std::vector<Rule>*>& sets, const std::vector<int>& inst_of,
                        const std::vector<std::vector<double>>& blocks, int Tn,
                        std::vector<std::vector<double>>& fit) -> sidr_status {
        const int Q = (int)sets.size();
        Packed pk;
        std::vector<int32_t> owner;
        std::vector<sidr_instance_desc> d(Q);
        std::vector<double> z((size_t)Q * 10), flat;
        std::vector<int64_t> mk((size_t)Q * 61), offs(Q);
        for (int q = 0; q < Q; q++) {
            const int k = inst_of[q];
            pack_rules(*sets[q], gps[q].vocab, pk);
            owner.insert(owner.end(), sets[q]->size(), q);
            d[q] = insts[k];
            std::copy(zps + 10 * (size_t)k, zps + 10 * (size_t)k + 10, z.begin() + 10 * (size_t)q);
            std::copy(masks + 61 * (size_t)k, masks + 61 * (size_t)k + 61, mk.begin() + 61 * (size_t)q);
            offs[q] = (int64_t)flat.size();
            flat.insert(flat.end(), blocks[q].begin(), blocks[q].end());
        }
        sidr_rules_desc r = pk.desc();
        std::vector<double> out((size_t)r.P * Tn);
        const double t0 = now_s();
        sidr_multi* m = nullptr;
        sidr_status st = sidr_multi_create(d.data(), z.data(), Q, &r, owner.data(), flat.data(),
                                           (int64_t)flat.size(), offs.data(), Tn, mk.data(), sc->device, &m);
        if (st == SIDR_OK) st = chosen < 0 ? sidr_multi_autotune(m, 1, &chosen, nullptr) : sidr_multi_set_shape(m, chosen);
        if (st == SIDR_OK) st = sidr_multi_run(m, nullptr);
        if (st == SIDR_OK) st = sidr_multi_read(m, out.data());
        const std::string why = st == SIDR_OK ? std::string() : std::string(sidr_last_error());
        sidr_multi_destroy(m);
        t_eval += now_s() - t0;
        evals += (int64_t)r.P * Tn;
        if (st != SIDR_OK) return gp_fail(st, "evaluation: " + why);
        fit.assign(Q, {});
        size_t p = 0;
        for (int q = 0; q < Q; q++) {
            fit[q].assign(sets[q]->size(), 0.0);
            for (size_t i = 0; i < sets[q]->size(); i++, p++) {
                double acc = 0.0;
                for (int s = 0; s < Tn; s++) acc += out[p * Tn + s];
                fit[q][i] = acc / Tn;
            }
        }
        return SIDR_OK;
    };
    auto train_blocks = [&](int g) {
        std::vector<std::vector<double>> blocks(E);
        for (int e = 0; e < E; e++) {
            const int n = insts[e / S].n;
            blocks[e].resize((size_t)T * n);
            sidr_gen_durations(n, insts[e / S].durations, 0.2, T, seed_of(e) * 10000 + g, blocks[e].data());
        }
        return blocks;
    };
    std::vector<std::vector<double>> test_blocks(K);
    for (int k = 0; k < K; k++) {
        test_blocks[k].resize((size_t)cfg->test_samples * insts[k].n);
        sidr_gen_durations(insts[k].n, insts[k].durations, 0.2, cfg->test_samples, test_seed,
                           test_blocks[k].data());
    }
    std::vector<int> inst_of_e(E);
    for (int e = 0; e < E; e++) inst_of_e[e] = e / S;

    std::vector<InstanceSurrogate> sur(K);
    // phenotypes of rules bred by population e, on its instance's situations
    auto features_of = [&](int e, const std::vector<Rule>& rules, std::vector<float>& f) -> sidr_status {
        const int k = e / S;
        Packed pk;
        pack_rules(rules, gps[e].vocab, pk);
        sidr_rules_desc r = pk.desc();
        f.assign((size_t)r.P * NF, 0.0f);
        const double t0 = now_s();
        const sidr_status st = sidr_phenotype(&r, sur[k].sit_terms.data(), sur[k].sit_nc.data(),
                                              sur[k].sit_ref.data(), NS, sc->max_cand, sc->device, f.data());
        t_model += now_s() - t0;
        return st;
    };

    std::vector<std::vector<double>> fits;
    for (int g = 0; g < G; g++) {
        std::vector<const std::vector<Rule>*> sets(E);
        for (int e = 0; e < E; e++) sets[e] = &gps[e].pop;
        const std::vector<std::vector<double>> blocks = train_blocks(g);
        sidr_status st = simulate(sets, inst_of_e, blocks, T, fits);
        if (st != SIDR_OK) return st;
        // each population's best rule: train fitness and the held-out block
        std::vector<size_t> best(E, 0);
        std::vector<std::vector<Rule>> champions(E);
        for (int e = 0; e < E; e++) {
            for (size_t p = 1; p < fits[e].size(); p++)
                if (fits[e][p] > fits[e][best[e]]) best[e] = p;
            if (best_train) best_train[(size_t)g * E + e] = fits[e][best[e]];
            champions[e] = {gps[e].pop[best[e]]};
            if (rho) rho[(size_t)g * E + e] = std::nan("");
        }
        if (g == G - 1 && best_rules) {  // the last generation's best rules as prefix text
            std::string text;
            for (int e = 0; e < E; e++) {
                size_t k = 0;
                prefix_at(champions[e][0], k, gps[e].vocab, text);
                text += '\n';
            }
            if (rules_cap <= (int64_t)text.size())
                return gp_fail(SIDR_ERR_INVALID, "best_rules buffer too small");
            std::memcpy(best_rules, text.c_str(), text.size() + 1);
        }
        {
            std::vector<const std::vector<Rule>*> bsets(E);
            std::vector<std::vector<double>> tb(E);
            for (int e = 0; e < E; e++) {
                bsets[e] = &champions[e];
                tb[e] = test_blocks[e / S];
            }
            std::vector<std::vector<double>> ho;
            if ((st = simulate(bsets, inst_of_e, tb, cfg->test_samples, ho)) != SIDR_OK) return st;
            if (held_out)
                for (int e = 0; e < E; e++) held_out[(size_t)g * E + e] = ho[e][0];
        }
        if (!sc->use_surrogate) {
            if (g < G - 1)
                for (int e = 0; e < E; e++) gps[e].step(fits[e]);
            continue;
        }
        if (g == 0) {
            // per instance: situations from the best rule of its first seed, and a model
            for (int k = 0; k < K; k++) {
                const int e = k * S;
                sidr_ctx* ctx = nullptr;
                if ((st = sidr_ctx_create(&insts[k], zps + 10 * (size_t)k, sc->device, &ctx)) != SIDR_OK) return st;
                Packed one;
                pack_rules(champions[e], gps[e].vocab, one);
                const double t0 = now_s();
                st = capture_for(ctx, &insts[k], masks + 61 * (size_t)k, sc, (uint64_t)seed_of(e), one, sur[k]);
                t_eval += now_s() - t0;
                sidr_ctx_destroy(ctx);
                if (st != SIDR_OK) return st;
                if ((st = sidr_mlp_create(sc->device, sc->model_seed + (uint64_t)k, &sur[k].model)) != SIDR_OK)
                    return st;
            }
        }
        for (int e = 0; e < E; e++) {
            std::vector<float> f;
            if ((st = features_of(e, gps[e].pop, f)) != SIDR_OK) return st;
            sur[e / S].hist_x.push_back(std::move(f));
            sur[e / S].hist_t.push_back(fits[e]);
        }
        if (g == G - 1) break;
        // per instance: train its model on the window of all its seeds' simulated fitness
        for (int k = 0; k < K; k++) {
            InstanceSurrogate& u = sur[k];
            while ((int)u.hist_x.size() > sc->history * 2 * S) {  // population + audit entries per seed
                u.hist_x.erase(u.hist_x.begin());
                u.hist_t.erase(u.hist_t.begin());
            }
            std::vector<float> X;
            std::vector<double> all;
            for (size_t h = 0; h < u.hist_x.size(); h++) {
                X.insert(X.end(), u.hist_x[h].begin(), u.hist_x[h].end());
                all.insert(all.end(), u.hist_t[h].begin(), u.hist_t[h].end());
            }
            const std::vector<float> Y = training_targets(all, sc->target);
            float loss = 0.0f;
            const uint64_t tseed = ((uint64_t)first_seed * 131 + (uint64_t)g) ^ ((uint64_t)k * 0x9e3779b97f4a7c15ull);
            const double t0 = now_s();
            st = sidr_mlp_train(u.model, X.data(), Y.data(), (int32_t)Y.size(), sc->train_steps, sc->batch,
                                sc->lr, tseed, &loss);
            t_model += now_s() - t0;
            if (st != SIDR_OK) return st;
        }
        // per population: breed, predict, and pick the audit sample
        std::vector<std::vector<Rule>> cand(E), aud_rules(E);
        std::vector<std::vector<float>> cf(E), pred(E);
        std::vector<std::vector<size_t>> aud(E);
        for (int e = 0; e < E; e++) {
            const int k = e / S;
            cand[e] = gps[e].breed(fits[e], (size_t)sc->screen);
            if ((st = features_of(e, cand[e], cf[e])) != SIDR_OK) return st;
            pred[e].resize(cand[e].size());
            const double t0 = now_s();
            st = sidr_mlp_predict(sur[k].model, cf[e].data(), (int32_t)cand[e].size(), pred[e].data());
            t_model += now_s() - t0;
            if (st != SIDR_OK) return st;
            aud[e] = gps[e].rng.sample(cand[e].size(), (size_t)sc->audit);
            for (size_t a : aud[e]) aud_rules[e].push_back(cand[e][a]);
        }
        // every audit in one launch, each on its population's train block
        std::vector<const std::vector<Rule>*> asets(E);
        for (int e = 0; e < E; e++) asets[e] = &aud_rules[e];
        std::vector<std::vector<double>> aud_fit;
        if ((st = simulate(asets, inst_of_e, blocks, T, aud_fit)) != SIDR_OK) return st;
        for (int e = 0; e < E; e++) {
            const int k = e / S;
            std::vector<double> aud_pred;
            std::vector<float> aud_x;
            for (size_t a : aud[e]) {
                aud_pred.push_back(pred[e][a]);
                aud_x.insert(aud_x.end(), cf[e].begin() + a * NF, cf[e].begin() + (a + 1) * NF);
            }
            const double r_s = spearman(aud_pred, aud_fit[e]);
            if (rho) rho[(size_t)g * E + e] = r_s;
            sur[k].hist_x.push_back(std::move(aud_x));
            sur[k].hist_t.push_back(aud_fit[e]);
            if (!(r_s >= sc->rho_min)) {
                fallback++;
                gps[e].step(fits[e]);
                continue;
            }
            // elites, then the screened offspring, then plain breeding for the slots left
            std::vector<int> order(ps);
            std::iota(order.begin(), order.end(), 0);
            std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return fits[e][a] > fits[e][b]; });
            std::vector<Rule> next;
            for (int i = 0; i < cfg->elitism && i < ps; i++) next.push_back(gps[e].pop[order[i]]);
            const int slots = ps - (int)next.size();
            const int need = (int)std::lround(sc->screen_fraction * slots);
            std::vector<int> pick;
            const std::vector<float>& pe = pred[e];
            const std::vector<float>& fe = cf[e];
            if (sc->selection == 1) {
                pick = preselect(pe, need);
            } else if (sc->distinct == 1) {
                pick = best_distinct<std::vector<float>>(pe, (size_t)need, [&](int c) {
                    return std::vector<float>(fe.begin() + (size_t)c * NF, fe.begin() + (size_t)c * NF + NS);
                });
            } else {
                pick = best_distinct<Rule>(pe, (size_t)need, [&](int c) { return cand[e][c]; });
            }
            for (int c : pick) next.push_back(cand[e][c]);
            if ((int)next.size() < ps) {
                std::vector<Rule> plain = gps[e].breed(fits[e], (size_t)(ps - (int)next.size()));
                for (Rule& r : plain) next.push_back(std::move(r));
            }
            gps[e].pop.swap(next);
            screened++;
        }
    }
    if (result) {
        result->eval_seconds = t_eval;
        result->model_seconds = t_model;
        result->host_seconds = now_s() - t_start - t_eval - t_model;
        result->evaluations = evals;
        result->generations_screened = screened;
        result->generations_fallback = fallback;
    }
    return SIDR_OK;
}
