// sidr_sgp.cpp -- the surrogate-assisted GP driver (include/sidr_surrogate.h):
// the GP of sidr_gp_core.hpp whose offspring are pre-screened by the MLP of
// sidr_surrogate.cu on their phenotypes, with the evaluator deciding
// every fitness and plain breeding whenever the model's audit rank
// correlation is too low.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <numeric>
#include <set>
#include <sstream>
#include <type_traits>

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


// ---------------------------------------------------------------- checkpoints
// Text of the surrogate driver's state between two generations.  Doubles and
// floats travel as the hexadecimal digits of their bits, so NaN audit values
// and every weight come back exactly.

constexpr const char* kSgpHeader = "sidr-sgp-checkpoint 1";

std::string hex64(double v) {
    uint64_t u;
    std::memcpy(&u, &v, 8);
    char b[24];
    std::snprintf(b, sizeof b, "%016llx", (unsigned long long)u);
    return b;
}
std::string hex32(float v) {
    uint32_t u;
    std::memcpy(&u, &v, 4);
    char b[16];
    std::snprintf(b, sizeof b, "%08x", u);
    return b;
}
bool unhex64(const std::string& t, double& v) {
    if (t.size() != 16) return false;
    char* end = nullptr;
    const uint64_t u = std::strtoull(t.c_str(), &end, 16);
    if (!end || *end) return false;
    std::memcpy(&v, &u, 8);
    return true;
}
bool unhex32(const std::string& t, float& v) {
    if (t.size() != 8) return false;
    char* end = nullptr;
    const uint32_t u = (uint32_t)std::strtoul(t.c_str(), &end, 16);
    if (!end || *end) return false;
    std::memcpy(&v, &u, 4);
    return true;
}

// A named list of values, 8 per line: "<key> <count>" then the lines.
template <class T>
void put_list(std::string& out, const char* key, const std::vector<T>& v) {
    out += std::string(key) + " " + std::to_string(v.size()) + "\n";
    for (size_t i = 0; i < v.size(); i++) {
        if constexpr (std::is_same<T, double>::value) out += hex64(v[i]);
        else if constexpr (std::is_same<T, float>::value) out += hex32(v[i]);
        else out += std::to_string(v[i]);
        out += (i % 8 == 7 || i + 1 == v.size()) ? "\n" : " ";
    }
}

template <class T>
bool get_list(std::istream& in, const char* key, std::vector<T>& v, size_t limit = (size_t)1 << 28) {
    std::string line, word;
    if (!std::getline(in, line)) return false;
    std::istringstream ls(line);
    long long cnt = -1;
    if (!(ls >> word >> cnt) || word != key || cnt < 0 || (size_t)cnt > limit) return false;
    v.clear();
    v.reserve((size_t)cnt);
    while ((long long)v.size() < cnt) {
        if (!std::getline(in, line)) return false;
        std::istringstream vs(line);
        std::string tok;
        while (vs >> tok) {
            T x{};
            if constexpr (std::is_same<T, double>::value) {
                if (!unhex64(tok, x)) return false;
            } else if constexpr (std::is_same<T, float>::value) {
                if (!unhex32(tok, x)) return false;
            } else {
                char* end = nullptr;
                const long long q = std::strtoll(tok.c_str(), &end, 10);
                if (!end || *end) return false;
                x = (T)q;
            }
            v.push_back(x);
        }
    }
    return (long long)v.size() == cnt;
}

std::string sgp_config_text(const sidr_sgp_config& c) {
    return "sgp " + std::to_string(c.screen) + " " + std::to_string(c.train_steps) + " " +
           std::to_string(c.batch) + " " + hex32(c.lr) + " " + std::to_string(c.audit) + " " + hex64(c.rho_min) +
           " " + std::to_string(c.history) + " " + std::to_string(c.n_situations) + " " +
           std::to_string(c.capture_scenarios) + " " + std::to_string(c.max_cand) + " " +
           std::to_string(c.model_seed) + " " + std::to_string(c.use_surrogate) + " " +
           std::to_string(c.selection) + " " + std::to_string(c.target) + " " + hex64(c.screen_fraction) + " " +
           std::to_string(c.distinct);
}

// Everything the driver carries from one generation to the next.
struct SgpState {
    int64_t next = 0;  // the generation to run next
    double t_eval = 0.0, t_model = 0.0, elapsed = 0.0;
    int64_t evals = 0;
    int64_t screened = 0, fallback = 0;
    std::vector<double> best_train, held_out, rho, gen_seconds;  // [next]
    std::vector<double> sit_terms;
    std::vector<int32_t> sit_nc, sit_ref;
    std::vector<float> model;  // sidr_mlp_state; empty without a model
    int64_t model_step = 0;
    std::vector<std::vector<float>> hist_x;
    std::vector<std::vector<double>> hist_t;
    std::string gp_text;  // sidr::gp::state_text
};

std::string sgp_state_text(const SgpState& st, uint64_t seed, int64_t test_seed, const sidr_instance_desc& inst,
                           const int64_t* mask, const sidr_sgp_config& sc) {
    std::string t = std::string(kSgpHeader) + "\n";
    char hb[32];
    std::snprintf(hb, sizeof hb, "%016llx", (unsigned long long)instance_hash(inst));
    t += "run " + std::to_string(seed) + " " + std::to_string(test_seed) + " " + std::to_string(inst.n) + " " +
         hb + "\n";
    t += "mask";
    for (int k = 0; k < 61; k++) t += " " + std::to_string(mask[k]);
    t += "\n" + sgp_config_text(sc) + "\n";
    t += "next " + std::to_string(st.next) + "\n";
    t += "counters " + hex64(st.t_eval) + " " + hex64(st.t_model) + " " + hex64(st.elapsed) + " " +
         std::to_string(st.evals) + " " + std::to_string(st.screened) + " " + std::to_string(st.fallback) + "\n";
    put_list(t, "best_train", st.best_train);
    put_list(t, "held_out", st.held_out);
    put_list(t, "rho", st.rho);
    put_list(t, "gen_seconds", st.gen_seconds);
    put_list(t, "sit_terms", st.sit_terms);
    put_list(t, "sit_nc", st.sit_nc);
    put_list(t, "sit_ref", st.sit_ref);
    t += "model_step " + std::to_string(st.model_step) + "\n";
    put_list(t, "model", st.model);
    t += "history " + std::to_string(st.hist_x.size()) + "\n";
    for (size_t h = 0; h < st.hist_x.size(); h++) {
        put_list(t, "x", st.hist_x[h]);
        put_list(t, "t", st.hist_t[h]);
    }
    const size_t lines = (size_t)std::count(st.gp_text.begin(), st.gp_text.end(), '\n');
    t += "gp " + std::to_string(lines) + "\n" + st.gp_text;
    return t;
}

sidr_status sgp_state_parse(const std::string& text, uint64_t seed, int64_t test_seed,
                            const sidr_instance_desc& inst, const int64_t* mask, const sidr_sgp_config& sc,
                            SgpState& st) {
    auto bad = [](const std::string& what) { return gp_fail(SIDR_ERR_INVALID, "surrogate checkpoint: " + what); };
    std::istringstream in(text);
    std::string line;
    if (!std::getline(in, line) || line != kSgpHeader) return bad("not a surrogate GP checkpoint of version 1");
    char hb[32];
    std::snprintf(hb, sizeof hb, "%016llx", (unsigned long long)instance_hash(inst));
    if (!std::getline(in, line) ||
        line != "run " + std::to_string(seed) + " " + std::to_string(test_seed) + " " + std::to_string(inst.n) +
                    " " + hb)
        return bad("written for another seed, test seed or instance");
    std::string want = "mask";
    for (int k = 0; k < 61; k++) want += " " + std::to_string(mask[k]);
    if (!std::getline(in, line) || line != want) return bad("written for another terminal mask");
    if (!std::getline(in, line) || line != sgp_config_text(sc)) return bad("written with other surrogate settings");
    long long next = -1;
    if (!std::getline(in, line) || std::sscanf(line.c_str(), "next %lld", &next) != 1 || next < 1)
        return bad("malformed generation line");
    st.next = next;
    {
        if (!std::getline(in, line)) return bad("no counters");
        std::istringstream ls(line);
        std::string w, a, b, c;
        long long ev, sc_, fb;
        if (!(ls >> w >> a >> b >> c >> ev >> sc_ >> fb) || w != "counters" || !unhex64(a, st.t_eval) ||
            !unhex64(b, st.t_model) || !unhex64(c, st.elapsed) || ev < 0 || sc_ < 0 || fb < 0)
            return bad("malformed counters");
        st.evals = ev;
        st.screened = sc_;
        st.fallback = fb;
    }
    if (!get_list(in, "best_train", st.best_train) || !get_list(in, "held_out", st.held_out) ||
        !get_list(in, "rho", st.rho) || !get_list(in, "gen_seconds", st.gen_seconds))
        return bad("malformed per-generation outputs");
    const size_t g = (size_t)next;
    if (st.best_train.size() != g || st.held_out.size() != g || st.rho.size() != g || st.gen_seconds.size() != g)
        return bad("per-generation outputs differ from the generation count");
    if (!get_list(in, "sit_terms", st.sit_terms) || !get_list(in, "sit_nc", st.sit_nc) ||
        !get_list(in, "sit_ref", st.sit_ref))
        return bad("malformed decision situations");
    long long ms = -1;
    if (!std::getline(in, line) || std::sscanf(line.c_str(), "model_step %lld", &ms) != 1 || ms < 0)
        return bad("malformed model step");
    st.model_step = ms;
    if (!get_list(in, "model", st.model)) return bad("malformed model state");
    long long nh = -1;
    if (!std::getline(in, line) || std::sscanf(line.c_str(), "history %lld", &nh) != 1 || nh < 0 || nh > 4096)
        return bad("malformed history");
    st.hist_x.assign((size_t)nh, {});
    st.hist_t.assign((size_t)nh, {});
    for (long long h = 0; h < nh; h++)
        if (!get_list(in, "x", st.hist_x[h]) || !get_list(in, "t", st.hist_t[h]) ||
            st.hist_x[h].size() != st.hist_t[h].size() * SIDR_MLP_INPUTS)
            return bad("malformed history entry");
    long long lines = -1;
    if (!std::getline(in, line) || std::sscanf(line.c_str(), "gp %lld", &lines) != 1 || lines < 1)
        return bad("malformed GP header");
    st.gp_text.clear();
    for (long long k = 0; k < lines; k++) {
        if (!std::getline(in, line)) return bad("GP state truncated");
        st.gp_text += line + "\n";
    }
    if (std::getline(in, line) && !line.empty()) return bad("trailing text");
    if (sc.use_surrogate) {
        const size_t C = (size_t)sc.max_cand, NS = (size_t)sc.n_situations;
        if (st.sit_nc.size() != NS || st.sit_ref.size() != NS || st.sit_terms.size() != NS * C * 61)
            return bad("decision situations of another size");
        for (size_t j = 0; j < NS; j++)
            if (st.sit_nc[j] < 2 || st.sit_nc[j] > (int32_t)C || st.sit_ref[j] < 0 || st.sit_ref[j] >= st.sit_nc[j])
                return bad("decision situation out of range");
    }
    return SIDR_OK;
}

// Writes text to path through a temporary file renamed over it, so that an
// interrupted write leaves the previous checkpoint in place.
sidr_status write_atomically(const char* path, const std::string& text) {
    const std::string tmp = std::string(path) + ".tmp";
    FILE* f = std::fopen(tmp.c_str(), "wb");
    if (!f) return gp_fail(SIDR_ERR_INVALID, "cannot write " + tmp);
    const bool ok = std::fwrite(text.data(), 1, text.size(), f) == text.size();
    if (std::fclose(f) != 0 || !ok) return gp_fail(SIDR_ERR_INVALID, "cannot write " + tmp);
    if (std::rename(tmp.c_str(), path) != 0) return gp_fail(SIDR_ERR_INVALID, std::string("cannot replace ") + path);
    return SIDR_OK;
}

bool read_file(const char* path, std::string& out) {
    FILE* f = std::fopen(path, "rb");
    if (!f) return false;
    char buf[1 << 16];
    size_t k;
    out.clear();
    while ((k = std::fread(buf, 1, sizeof buf, f)) > 0) out.append(buf, k);
    std::fclose(f);
    return true;
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
    return sidr_sgp_run_resumable(ctx, inst, cfg, sc, terminals_csv, mask, seed, test_seed, nullptr, 0, -1,
                                  nullptr, best_train, held_out, rho, gen_seconds, best_rule, rule_cap, result);
}

sidr_status sidr_sgp_run_resumable(sidr_ctx* ctx, const sidr_instance_desc* inst, const sidr_gp_config* cfg,
                                   const sidr_sgp_config* sc, const char* terminals_csv, const int64_t* mask,
                                   uint64_t seed, int64_t test_seed, const char* checkpoint_path, int32_t every,
                                   int32_t stop_after, int32_t* finished, double* best_train, double* held_out,
                                   double* rho, double* gen_seconds, char* best_rule, int64_t rule_cap,
                                   sidr_sgp_result* result) {
    std::string err;
    if (finished) *finished = 0;
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
    double t_start = now_s();
    double t_eval = 0.0, t_model = 0.0;
    int64_t evals = 0;
    int screened = 0, fallback = 0;
    // per-generation outputs of the whole run (a resumed run starts with the checkpoint's)
    std::vector<double> out_bt, out_ho, out_rho, out_gs;

    // a checkpoint at checkpoint_path: the state after generation next - 1
    SgpState resume;
    bool resuming = false;
    if (checkpoint_path) {
        std::string text;
        if (read_file(checkpoint_path, text)) {
            const sidr_status st = sgp_state_parse(text, seed, test_seed, *inst, mask, *sc, resume);
            if (st != SIDR_OK) return st;
            if (resume.next >= G) return gp_fail(SIDR_ERR_INVALID, "surrogate checkpoint: beyond the run's end");
            resuming = true;
        }
    }

    Gp gp(*cfg, seed);
    gp.vocab.terminals = terms;
    gp.vocab.n_funcs = cfg->with_rmod ? 7 : 6;
    if (resuming) {
        std::unique_ptr<Gp> saved;
        int64_t steps = -1;
        const sidr_status st = sidr::gp::state_parse(resume.gp_text, saved, steps);
        if (st != SIDR_OK) return st;
        if (!same_config(saved->cfg, *cfg) || saved->vocab.terminals != terms)
            return gp_fail(SIDR_ERR_INVALID, "surrogate checkpoint: written for another GP configuration");
        gp = *saved;
        t_eval = resume.t_eval;
        t_model = resume.t_model;
        t_start = now_s() - resume.elapsed;
        evals = resume.evals;
        screened = (int)resume.screened;
        fallback = (int)resume.fallback;
        out_bt = resume.best_train;
        out_ho = resume.held_out;
        out_rho = resume.rho;
        out_gs = resume.gen_seconds;
    } else {
        gp.init();
    }

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
    int g0 = 0;
    if (resuming) {
        g0 = (int)resume.next;
        sit_terms.swap(resume.sit_terms);
        sit_nc.swap(resume.sit_nc);
        sit_ref.swap(resume.sit_ref);
        hist_x.swap(resume.hist_x);
        hist_t.swap(resume.hist_t);
        if (sc->use_surrogate) {
            sidr_status st = sidr_mlp_create(sc->device, sc->model_seed, &model);
            int64_t cnt = 0;
            if (st == SIDR_OK) st = sidr_mlp_state(model, 0, nullptr, &cnt, nullptr);
            if (st == SIDR_OK && cnt != (int64_t)resume.model.size())
                return gp_fail(SIDR_ERR_INVALID, "surrogate checkpoint: model state of another size");
            if (st == SIDR_OK) st = sidr_mlp_state(model, 1, resume.model.data(), &cnt, &resume.model_step);
            if (st != SIDR_OK) return st;
        }
    }
    // the state after generation g, for the next call to resume from
    auto save = [&](int g) -> sidr_status {
        SgpState cur;
        cur.next = g + 1;
        cur.t_eval = t_eval;
        cur.t_model = t_model;
        cur.elapsed = now_s() - t_start;
        cur.evals = evals;
        cur.screened = screened;
        cur.fallback = fallback;
        cur.best_train = out_bt;
        cur.held_out = out_ho;
        cur.rho = out_rho;
        cur.gen_seconds = out_gs;
        cur.sit_terms = sit_terms;
        cur.sit_nc = sit_nc;
        cur.sit_ref = sit_ref;
        if (model) {
            int64_t cnt = 0;
            sidr_status st = sidr_mlp_state(model, 0, nullptr, &cnt, nullptr);
            cur.model.resize((size_t)cnt);
            if (st == SIDR_OK) st = sidr_mlp_state(model, 0, cur.model.data(), &cnt, &cur.model_step);
            if (st != SIDR_OK) return st;
        }
        cur.hist_x = hist_x;
        cur.hist_t = hist_t;
        cur.gp_text = sidr::gp::state_text(gp, g + 1);
        return write_atomically(checkpoint_path, sgp_state_text(cur, seed, test_seed, *inst, mask, *sc));
    };
    auto copy_out = [&]() {
        for (size_t g = 0; g < out_bt.size(); g++) {
            if (best_train) best_train[g] = out_bt[g];
            if (held_out) held_out[g] = out_ho[g];
            if (rho) rho[g] = out_rho[g];
            if (gen_seconds) gen_seconds[g] = out_gs[g];
        }
        if (result) {
            result->eval_seconds = t_eval;
            result->model_seconds = t_model;
            result->host_seconds = now_s() - t_start - t_eval - t_model;
            result->evaluations = evals;
            result->generations_screened = screened;
            result->generations_fallback = fallback;
        }
    };

    std::vector<double> fit;
    int ran = 0;  // generations run by this call
    for (int g = g0; g < G; g++) {
        sidr_status st = simulate(gp.pop, (long long)seed * 10000 + g, T, fit);
        if (st != SIDR_OK) return st;
        size_t bi = 0;
        for (size_t p = 1; p < fit.size(); p++)
            if (fit[p] > fit[bi]) bi = p;
        out_bt.push_back(fit[bi]);
        {
            std::vector<double> ho;
            if ((st = simulate({gp.pop[bi]}, test_seed, cfg->test_samples, ho)) != SIDR_OK) return st;
            out_ho.push_back(ho[0]);
        }
        out_rho.push_back(std::nan(""));
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
                out_rho[g] = r_s;
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
        out_gs.push_back(now_s() - t_start);
        ran++;
        if (checkpoint_path && g < G - 1) {
            const bool stop = stop_after >= 0 && ran >= stop_after;
            if (stop || (every > 0 && (g + 1) % every == 0))
                if ((st = save(g)) != SIDR_OK) return st;
            if (stop) {
                copy_out();
                return SIDR_OK;  // *finished stays 0
            }
        }
    }
    // the last generation's best rule
    size_t bi = 0;
    for (size_t p = 1; p < fit.size(); p++)
        if (fit[p] > fit[bi]) bi = p;
    std::string text;
    size_t k = 0;
    prefix_at(gp.pop[bi], k, gp.vocab, text);
    if (best_rule && rule_cap > (int64_t)text.size()) std::memcpy(best_rule, text.c_str(), text.size() + 1);
    copy_out();
    if (finished) *finished = 1;
    return SIDR_OK;
}

}  // extern "C"


// ----------------------------------------------------------------------------
// Many instances x many seeds (sidr_sgp_run_multi).

namespace {

constexpr const char* kSgpMultiHeader = "sidr-sgp-multi-checkpoint 1";

// The combined driver's state between two generations.
struct SgpMultiState {
    int64_t next = 0;
    double t_eval = 0.0, t_model = 0.0, elapsed = 0.0;
    int64_t evals = 0, screened = 0, fallback = 0, chosen = -1;
    std::vector<double> best_train, held_out, rho;  // [next][E]
    struct Inst {
        std::vector<double> sit_terms;
        std::vector<int32_t> sit_nc, sit_ref;
        std::vector<float> model;
        int64_t model_step = 0;
        std::vector<std::vector<float>> hist_x;
        std::vector<std::vector<double>> hist_t;
    };
    std::vector<Inst> inst;       // [K]
    std::vector<std::string> gp;  // [E] sidr::gp::state_text
};

std::string multi_run_line(int K, int S, int64_t first_seed, int64_t test_seed, const sidr_instance_desc* insts) {
    std::string t = "run " + std::to_string(K) + " " + std::to_string(S) + " " + std::to_string(first_seed) + " " +
                    std::to_string(test_seed);
    for (int k = 0; k < K; k++) {
        char hb[32];
        std::snprintf(hb, sizeof hb, " %d:%016llx", insts[k].n, (unsigned long long)instance_hash(insts[k]));
        t += hb;
    }
    return t;
}

std::string multi_mask_line(int K, const int64_t* masks) {
    std::string t = "masks";
    for (int64_t i = 0; i < (int64_t)K * 61; i++) t += " " + std::to_string(masks[i]);
    return t;
}

std::string sgp_multi_text(const SgpMultiState& st, const std::string& run_line, const std::string& mask_line,
                           const sidr_sgp_config& sc) {
    std::string t = std::string(kSgpMultiHeader) + "\n" + run_line + "\n" + mask_line + "\n" + sgp_config_text(sc) +
                    "\n";
    t += "next " + std::to_string(st.next) + "\n";
    t += "counters " + hex64(st.t_eval) + " " + hex64(st.t_model) + " " + hex64(st.elapsed) + " " +
         std::to_string(st.evals) + " " + std::to_string(st.screened) + " " + std::to_string(st.fallback) + " " +
         std::to_string(st.chosen) + "\n";
    put_list(t, "best_train", st.best_train);
    put_list(t, "held_out", st.held_out);
    put_list(t, "rho", st.rho);
    for (const SgpMultiState::Inst& u : st.inst) {
        put_list(t, "sit_terms", u.sit_terms);
        put_list(t, "sit_nc", u.sit_nc);
        put_list(t, "sit_ref", u.sit_ref);
        t += "model_step " + std::to_string(u.model_step) + "\n";
        put_list(t, "model", u.model);
        t += "history " + std::to_string(u.hist_x.size()) + "\n";
        for (size_t h = 0; h < u.hist_x.size(); h++) {
            put_list(t, "x", u.hist_x[h]);
            put_list(t, "t", u.hist_t[h]);
        }
    }
    for (const std::string& g : st.gp)
        t += "gp " + std::to_string(std::count(g.begin(), g.end(), '\n')) + "\n" + g;
    return t;
}

sidr_status sgp_multi_parse(const std::string& text, const std::string& run_line, const std::string& mask_line,
                            const sidr_sgp_config& sc, int K, int E, SgpMultiState& st) {
    auto bad = [](const std::string& what) {
        return gp_fail(SIDR_ERR_INVALID, "combined-run checkpoint: " + what);
    };
    std::istringstream in(text);
    std::string line;
    if (!std::getline(in, line) || line != kSgpMultiHeader) return bad("not a combined-run checkpoint of version 1");
    if (!std::getline(in, line) || line != run_line) return bad("written for other instances, seeds or test seed");
    if (!std::getline(in, line) || line != mask_line) return bad("written for other terminal masks");
    if (!std::getline(in, line) || line != sgp_config_text(sc)) return bad("written with other surrogate settings");
    long long next = -1;
    if (!std::getline(in, line) || std::sscanf(line.c_str(), "next %lld", &next) != 1 || next < 1)
        return bad("malformed generation line");
    st.next = next;
    {
        if (!std::getline(in, line)) return bad("no counters");
        std::istringstream ls(line);
        std::string w, a, b, c;
        long long ev, sc_, fb, ch;
        if (!(ls >> w >> a >> b >> c >> ev >> sc_ >> fb >> ch) || w != "counters" || !unhex64(a, st.t_eval) ||
            !unhex64(b, st.t_model) || !unhex64(c, st.elapsed) || ev < 0 || sc_ < 0 || fb < 0 || ch < -1 ||
            ch >= SIDR_MULTI_SHAPES)
            return bad("malformed counters");
        st.evals = ev;
        st.screened = sc_;
        st.fallback = fb;
        st.chosen = ch;
    }
    if (!get_list(in, "best_train", st.best_train) || !get_list(in, "held_out", st.held_out) ||
        !get_list(in, "rho", st.rho))
        return bad("malformed per-generation outputs");
    const size_t want = (size_t)next * (size_t)E;
    if (st.best_train.size() != want || st.held_out.size() != want || st.rho.size() != want)
        return bad("per-generation outputs differ from generations x populations");
    st.inst.assign((size_t)K, {});
    for (SgpMultiState::Inst& u : st.inst) {
        if (!get_list(in, "sit_terms", u.sit_terms) || !get_list(in, "sit_nc", u.sit_nc) ||
            !get_list(in, "sit_ref", u.sit_ref))
            return bad("malformed decision situations");
        long long ms = -1;
        if (!std::getline(in, line) || std::sscanf(line.c_str(), "model_step %lld", &ms) != 1 || ms < 0)
            return bad("malformed model step");
        u.model_step = ms;
        if (!get_list(in, "model", u.model)) return bad("malformed model state");
        long long nh = -1;
        if (!std::getline(in, line) || std::sscanf(line.c_str(), "history %lld", &nh) != 1 || nh < 0 ||
            nh > (1 << 20))
            return bad("malformed history");
        u.hist_x.assign((size_t)nh, {});
        u.hist_t.assign((size_t)nh, {});
        for (long long h = 0; h < nh; h++)
            if (!get_list(in, "x", u.hist_x[h]) || !get_list(in, "t", u.hist_t[h]) ||
                u.hist_x[h].size() != u.hist_t[h].size() * SIDR_MLP_INPUTS)
                return bad("malformed history entry");
        if (sc.use_surrogate) {
            const size_t C = (size_t)sc.max_cand, NS = (size_t)sc.n_situations;
            if (u.sit_nc.size() != NS || u.sit_ref.size() != NS || u.sit_terms.size() != NS * C * 61)
                return bad("decision situations of another size");
            for (size_t j = 0; j < NS; j++)
                if (u.sit_nc[j] < 2 || u.sit_nc[j] > (int32_t)C || u.sit_ref[j] < 0 || u.sit_ref[j] >= u.sit_nc[j])
                    return bad("decision situation out of range");
        }
    }
    st.gp.assign((size_t)E, {});
    for (std::string& g : st.gp) {
        long long lines = -1;
        if (!std::getline(in, line) || std::sscanf(line.c_str(), "gp %lld", &lines) != 1 || lines < 1)
            return bad("malformed GP header");
        for (long long k = 0; k < lines; k++) {
            if (!std::getline(in, line)) return bad("GP state truncated");
            g += line + "\n";
        }
    }
    if (std::getline(in, line) && !line.empty()) return bad("trailing text");
    return SIDR_OK;
}

}  // namespace

extern "C" sidr_status sidr_sgp_run_multi(const sidr_instance_desc* insts, const double* zps, int32_t K,
                                          const sidr_gp_config* cfg, const sidr_sgp_config* sc,
                                          const char* terminals_csv, const int64_t* masks, int32_t n_seeds,
                                          int64_t first_seed, int64_t test_seed, int32_t shape,
                                          double* best_train, double* held_out, double* rho,
                                          char* best_rules, int64_t rules_cap, sidr_sgp_result* result) {
    return sidr_sgp_run_multi_resumable(insts, zps, K, cfg, sc, terminals_csv, masks, n_seeds, first_seed,
                                        test_seed, shape, nullptr, 0, -1, nullptr, best_train, held_out, rho,
                                        best_rules, rules_cap, result);
}

extern "C" sidr_status sidr_sgp_run_multi_resumable(
    const sidr_instance_desc* insts, const double* zps, int32_t K, const sidr_gp_config* cfg,
    const sidr_sgp_config* sc, const char* terminals_csv, const int64_t* masks, int32_t n_seeds, int64_t first_seed,
    int64_t test_seed, int32_t shape, const char* checkpoint_path, int32_t every, int32_t stop_after,
    int32_t* finished, double* best_train, double* held_out, double* rho, char* best_rules, int64_t rules_cap,
    sidr_sgp_result* result) {
    std::string err;
    if (finished) *finished = 0;
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
    double t_start = now_s();
    double t_eval = 0.0, t_model = 0.0;
    int64_t evals = 0;
    int screened = 0, fallback = 0, chosen = shape;
    // per-generation outputs [g][E] of the whole run (a resumed run starts with the checkpoint's)
    std::vector<double> out_bt, out_ho, out_rho;

    const std::string run_line = multi_run_line(K, S, first_seed, test_seed, insts);
    const std::string mask_line = multi_mask_line(K, masks);
    SgpMultiState resume;
    bool resuming = false;
    if (checkpoint_path) {
        std::string text;
        if (read_file(checkpoint_path, text)) {
            const sidr_status st = sgp_multi_parse(text, run_line, mask_line, *sc, K, E, resume);
            if (st != SIDR_OK) return st;
            if (resume.next >= G) return gp_fail(SIDR_ERR_INVALID, "combined-run checkpoint: beyond the run's end");
            resuming = true;
        }
    }

    // population e = k * S + s: instance k, GP seed first_seed + s
    std::vector<Gp> gps;
    gps.reserve(E);
    for (int e = 0; e < E; e++) {
        gps.emplace_back(*cfg, (uint64_t)(first_seed + e % S));
        gps.back().vocab.terminals = terms;
        gps.back().vocab.n_funcs = cfg->with_rmod ? 7 : 6;
        if (resuming) {
            std::unique_ptr<Gp> saved;
            int64_t steps = -1;
            const sidr_status st = sidr::gp::state_parse(resume.gp[e], saved, steps);
            if (st != SIDR_OK) return st;
            if (!same_config(saved->cfg, *cfg) || saved->vocab.terminals != terms)
                return gp_fail(SIDR_ERR_INVALID, "combined-run checkpoint: written for another GP configuration");
            gps.back() = *saved;
        } else {
            gps.back().init();
        }
    }
    if (resuming) {
        t_eval = resume.t_eval;
        t_model = resume.t_model;
        t_start = now_s() - resume.elapsed;
        evals = resume.evals;
        screened = (int)resume.screened;
        fallback = (int)resume.fallback;
        chosen = resume.chosen >= 0 ? (int)resume.chosen : shape;
        out_bt = resume.best_train;
        out_ho = resume.held_out;
        out_rho = resume.rho;
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
        if (st == SIDR_OK) st = chosen < 0 ? sidr_multi_autotune_sampled(m, 1, 16, &chosen, nullptr) : sidr_multi_set_shape(m, chosen);
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
    if (resuming) {
        for (int k = 0; k < K; k++) {
            SgpMultiState::Inst& u = resume.inst[k];
            sur[k].sit_terms.swap(u.sit_terms);
            sur[k].sit_nc.swap(u.sit_nc);
            sur[k].sit_ref.swap(u.sit_ref);
            sur[k].hist_x.swap(u.hist_x);
            sur[k].hist_t.swap(u.hist_t);
            if (!sc->use_surrogate) continue;
            sidr_status st = sidr_mlp_create(sc->device, sc->model_seed + (uint64_t)k, &sur[k].model);
            int64_t cnt = 0;
            if (st == SIDR_OK) st = sidr_mlp_state(sur[k].model, 0, nullptr, &cnt, nullptr);
            if (st == SIDR_OK && cnt != (int64_t)u.model.size())
                return gp_fail(SIDR_ERR_INVALID, "combined-run checkpoint: model state of another size");
            if (st == SIDR_OK) st = sidr_mlp_state(sur[k].model, 1, u.model.data(), &cnt, &u.model_step);
            if (st != SIDR_OK) return st;
        }
    }
    // the state after generation g, for the next call to resume from
    auto save = [&](int g) -> sidr_status {
        SgpMultiState cur;
        cur.next = g + 1;
        cur.t_eval = t_eval;
        cur.t_model = t_model;
        cur.elapsed = now_s() - t_start;
        cur.evals = evals;
        cur.screened = screened;
        cur.fallback = fallback;
        cur.chosen = chosen;
        cur.best_train = out_bt;
        cur.held_out = out_ho;
        cur.rho = out_rho;
        cur.inst.resize((size_t)K);
        for (int k = 0; k < K; k++) {
            SgpMultiState::Inst& u = cur.inst[k];
            u.sit_terms = sur[k].sit_terms;
            u.sit_nc = sur[k].sit_nc;
            u.sit_ref = sur[k].sit_ref;
            u.hist_x = sur[k].hist_x;
            u.hist_t = sur[k].hist_t;
            if (sur[k].model) {
                int64_t cnt = 0;
                sidr_status st = sidr_mlp_state(sur[k].model, 0, nullptr, &cnt, nullptr);
                u.model.resize((size_t)cnt);
                if (st == SIDR_OK) st = sidr_mlp_state(sur[k].model, 0, u.model.data(), &cnt, &u.model_step);
                if (st != SIDR_OK) return st;
            }
        }
        for (int e = 0; e < E; e++) cur.gp.push_back(sidr::gp::state_text(gps[e], g + 1));
        return write_atomically(checkpoint_path, sgp_multi_text(cur, run_line, mask_line, *sc));
    };
    auto copy_out = [&]() {
        for (size_t i = 0; i < out_bt.size(); i++) {
            if (best_train) best_train[i] = out_bt[i];
            if (held_out) held_out[i] = out_ho[i];
            if (rho) rho[i] = out_rho[i];
        }
        if (result) {
            result->eval_seconds = t_eval;
            result->model_seconds = t_model;
            result->host_seconds = now_s() - t_start - t_eval - t_model;
            result->evaluations = evals;
            result->generations_screened = screened;
            result->generations_fallback = fallback;
        }
    };
    // after generation g: a checkpoint, and the end of this call when it has run stop_after generations
    int ran = 0;
    auto after_generation = [&](int g, bool& stop) -> sidr_status {
        ran++;
        stop = false;
        if (!checkpoint_path || g >= G - 1) return SIDR_OK;
        stop = stop_after >= 0 && ran >= stop_after;
        if (stop || (every > 0 && (g + 1) % every == 0)) return save(g);
        return SIDR_OK;
    };
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
    const int g0 = resuming ? (int)resume.next : 0;
    for (int g = g0; g < G; g++) {
        out_bt.resize((size_t)(g + 1) * E);
        out_ho.resize((size_t)(g + 1) * E);
        out_rho.resize((size_t)(g + 1) * E);
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
            out_bt[(size_t)g * E + e] = fits[e][best[e]];
            champions[e] = {gps[e].pop[best[e]]};
            out_rho[(size_t)g * E + e] = std::nan("");
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
            for (int e = 0; e < E; e++) out_ho[(size_t)g * E + e] = ho[e][0];
        }
        if (!sc->use_surrogate) {
            if (g < G - 1)
                for (int e = 0; e < E; e++) gps[e].step(fits[e]);
            bool stop = false;
            if ((st = after_generation(g, stop)) != SIDR_OK) return st;
            if (stop) {
                copy_out();
                return SIDR_OK;
            }
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
            out_rho[(size_t)g * E + e] = r_s;
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
        bool stop = false;
        if ((st = after_generation(g, stop)) != SIDR_OK) return st;
        if (stop) {
            copy_out();
            return SIDR_OK;
        }
    }
    copy_out();
    if (finished) *finished = 1;
    return SIDR_OK;
}
