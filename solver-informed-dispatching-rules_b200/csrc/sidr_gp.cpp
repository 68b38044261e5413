// sidr_gp.cpp -- the host GP loop driving the evaluator (include/sidr_gp.h).
#include <algorithm>
#include <chrono>
#include <memory>
#include <sstream>

#include "sidr_gp_core.hpp"

using namespace sidr::gp;

struct sidr_gp_session {
    Gp gp;
    int64_t generation = 0;  // gp_step calls so far
    sidr_gp_session(const sidr_gp_config& c, uint64_t seed) : gp(c, seed) {}
};

// A seed-batched run (exhaust_batched) taken one generation at a time: the
// sessions of its seeds, the generations evaluated so far and what they gave.
struct sidr_gp_batched {
    sidr_ctx* ctx = nullptr;
    int n = 0;                        // customers of the instance
    uint64_t inst_hash = 0;           // of the instance's arrays (checkpoints name their instance)
    std::vector<double> durations;    // expected service times (scenario sampling)
    sidr_gp_config cfg{};
    std::vector<int64_t> mask;        // the 61-slot terminal mask
    int64_t first_seed = 0, test_seed = 0;
    std::vector<std::unique_ptr<sidr_gp_session>> seeds;
    int64_t gen = 0;                  // generations evaluated (and bred from, but the last)
    std::vector<double> best_train;   // [gen][seeds]
    double t_eval = 0.0, t_host = 0.0;
    int64_t evals = 0;

    // One grouped evaluation of every population on its own train block
    // (base seed seed*10000 + gen): per-rule mean fitness per population.
    sidr_status grouped_fit(int gen_no, std::vector<std::vector<double>>& fits);
};

namespace {

constexpr const char* kCheckpointHeader = "sidr-gp-checkpoint 1";
constexpr const char* kBatchedHeader = "sidr-gp-batched-checkpoint 1";

double seconds_now() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

std::string hexf(double v) {
    char buf[64];
    std::snprintf(buf, sizeof buf, "%a", v);
    return buf;
}

// A rule in prefix codes is well formed when it is one complete tree of
// known functions and leaf labels.
bool rule_ok(const Rule& r, int n_funcs, size_t n_labels) {
    if (r.empty()) return false;
    long need = 1;
    for (size_t k = 0; k < r.size(); k++) {
        if (need <= 0) return false;
        const int32_t c = r[k];
        if (c >= 0) {
            if (c >= n_funcs) return false;
            need += 1;
        } else {
            if ((size_t)(-(int64_t)c - 1) >= n_labels) return false;
            need -= 1;
        }
    }
    return need == 0;
}

}  // namespace

namespace sidr {
namespace gp {

std::string state_text(const Gp& g, int64_t generation) {
    const sidr_gp_config& c = g.cfg;
    std::string t = std::string(kCheckpointHeader) + "\n";
    t += "config " + std::to_string(c.population) + " " + std::to_string(c.generations) + " " +
         std::to_string(c.max_depth) + " " + std::to_string(c.min_depth) + " " + std::to_string(c.tournament) +
         " " + std::to_string(c.elitism) + " " + hexf(c.crossover_rate) + " " + hexf(c.mutation_rate) + " " +
         hexf(c.reproduction_rate) + " " + std::to_string(c.train_samples) + " " +
         std::to_string(c.test_samples) + " " + std::to_string(c.with_rmod) + "\n";
    t += "generation " + std::to_string(generation) + "\n";
    t += "terminals " + std::to_string(g.vocab.terminals.size()) + "\n";
    for (const std::string& x : g.vocab.terminals) t += x + "\n";
    t += "labels " + std::to_string(g.vocab.labels.size()) + "\n";
    for (const std::string& x : g.vocab.labels) t += x + "\n";
    t += "rng " + g.rng.state() + "\n";
    t += "population " + std::to_string(g.pop.size()) + "\n";
    for (const Rule& r : g.pop) {
        t += std::to_string(r.size());
        for (int32_t v : r) t += " " + std::to_string(v);
        t += "\n";
    }
    return t;
}

sidr_status state_parse(const std::string& text, std::unique_ptr<Gp>& out, int64_t& generation_out) {
    std::istringstream in(text);
    std::string line, word;
    auto bad = [](const std::string& what) { return gp_fail(SIDR_ERR_INVALID, "checkpoint: " + what); };
    if (!std::getline(in, line) || line != kCheckpointHeader) return bad("not a GP checkpoint of version 1");
    sidr_gp_config c;
    std::string cx, mu, rp;
    if (!std::getline(in, line)) return bad("no config line");
    {
        std::istringstream ls(line);
        if (!(ls >> word) || word != "config" ||
            !(ls >> c.population >> c.generations >> c.max_depth >> c.min_depth >> c.tournament >> c.elitism >>
              cx >> mu >> rp >> c.train_samples >> c.test_samples >> c.with_rmod))
            return bad("malformed config line");
        c.crossover_rate = std::strtod(cx.c_str(), nullptr);
        c.mutation_rate = std::strtod(mu.c_str(), nullptr);
        c.reproduction_rate = std::strtod(rp.c_str(), nullptr);
    }
    std::string err;
    if (!valid_config(&c, err)) return bad(err);
    int64_t generation = -1;
    if (!std::getline(in, line) || std::sscanf(line.c_str(), "generation %lld", (long long*)&generation) != 1 ||
        generation < 0)
        return bad("malformed generation line");
    auto read_list = [&](const char* key, std::vector<std::string>& items) -> bool {
        long long cnt = -1;
        if (!std::getline(in, line)) return false;
        std::istringstream ls(line);
        if (!(ls >> word) || word != key || !(ls >> cnt) || cnt < 0 || cnt > (1 << 24)) return false;
        items.clear();
        for (long long i = 0; i < cnt; i++) {
            if (!std::getline(in, line) || line.empty()) return false;
            items.push_back(line);
        }
        return true;
    };
    std::vector<std::string> terms, labels;
    if (!read_list("terminals", terms)) return bad("malformed terminals");
    std::string csv;
    for (size_t i = 0; i < terms.size(); i++) csv += (i ? "," : "") + terms[i];
    std::vector<std::string> parsed;
    if (!parse_terminals(csv.c_str(), parsed, err) || parsed != terms) return bad("terminals: " + err);
    if (!read_list("labels", labels)) return bad("malformed labels");
    std::unique_ptr<Gp> g(new Gp(c, 0));
    g->vocab.terminals = terms;
    g->vocab.n_funcs = c.with_rmod ? 7 : 6;
    for (const std::string& l : labels)
        if (g->vocab.leaf(l) != (int)g->vocab.labels.size() - 1) return bad("repeated label " + l);
    if (!std::getline(in, line) || line.compare(0, 4, "rng ") != 0 || !g->rng.set_state(line.substr(4)))
        return bad("malformed generator state");
    long long np = -1;
    if (!std::getline(in, line) || std::sscanf(line.c_str(), "population %lld", &np) != 1 ||
        np != c.population)
        return bad("population size differs from the config");
    for (long long i = 0; i < np; i++) {
        if (!std::getline(in, line)) return bad("population truncated");
        std::istringstream ls(line);
        long long len = -1;
        if (!(ls >> len) || len < 1 || len > (1 << 20)) return bad("malformed rule");
        Rule r((size_t)len);
        for (long long k = 0; k < len; k++)
            if (!(ls >> r[(size_t)k])) return bad("malformed rule");
        if (ls >> word) return bad("rule " + std::to_string(i) + ": more codes than its length");
        if (!rule_ok(r, g->vocab.n_funcs, labels.size())) return bad("rule " + std::to_string(i) + " is not a tree");
        g->pop.push_back(std::move(r));
    }
    out = std::move(g);
    generation_out = generation;
    return SIDR_OK;
}

}  // namespace gp
}  // namespace sidr

sidr_status sidr_gp_batched::grouped_fit(int gen_no, std::vector<std::vector<double>>& fits) {
    const int n_seeds = (int)seeds.size(), ps = cfg.population, T = cfg.train_samples;
    std::vector<int32_t> ops, args, off, len;
    for (auto& g : seeds) g->gp.packed(ops, args, off, len);
    std::vector<double> grouped((size_t)n_seeds * T * n);
    for (int s = 0; s < n_seeds; s++)
        sidr_gen_durations(n, durations.data(), 0.2, T, (first_seed + s) * 10000 + gen_no,
                           grouped.data() + (size_t)s * T * n);
    sidr_rules_desc r{ops.data(), args.data(), off.data(), len.data(), (int32_t)off.size(), (int64_t)ops.size()};
    std::vector<double> out((size_t)r.P * T);
    const double e0 = seconds_now();
    const sidr_status st = sidr_evaluate_grouped(ctx, &r, grouped.data(), n_seeds, T, ps, mask.data(), out.data());
    t_eval += seconds_now() - e0;
    evals += (int64_t)r.P * T;
    if (st != SIDR_OK) return gp_fail(st, std::string("evaluation: ") + sidr_last_error());
    fits.assign(n_seeds, std::vector<double>(ps));
    for (int s = 0; s < n_seeds; s++)
        for (int p = 0; p < ps; p++) {
            double acc = 0.0;
            for (int t = 0; t < T; t++) acc += out[((size_t)s * ps + p) * T + t];
            fits[s][p] = acc / T;
        }
    return SIDR_OK;
}

extern "C" {

void sidr_gp_default_config(sidr_gp_config* c) {
    if (!c) return;
    c->population = 1024;
    c->generations = 51;
    c->max_depth = 8;
    c->min_depth = 2;
    c->tournament = 7;
    c->elitism = 10;
    c->crossover_rate = 0.80;
    c->mutation_rate = 0.15;
    c->reproduction_rate = 0.05;
    c->train_samples = 1;
    c->test_samples = 500;
    c->with_rmod = 0;
}

sidr_status sidr_gp_create(const sidr_gp_config* cfg, const char* terminals_csv, uint64_t seed,
                           sidr_gp_session** out) {
    if (!out) return gp_fail(SIDR_ERR_INVALID, "out is null");
    *out = nullptr;
    std::string err;
    if (!valid_config(cfg, err)) return gp_fail(SIDR_ERR_INVALID, err);
    std::vector<std::string> terms;
    if (!parse_terminals(terminals_csv, terms, err)) return gp_fail(SIDR_ERR_INVALID, err);
    sidr_gp_session* s = new sidr_gp_session(*cfg, seed);
    s->gp.vocab.terminals = terms;
    s->gp.vocab.n_funcs = cfg->with_rmod ? 7 : 6;
    s->gp.init();
    *out = s;
    return SIDR_OK;
}

void sidr_gp_destroy(sidr_gp_session* s) { delete s; }

int64_t sidr_gp_population_text(const sidr_gp_session* s, char* buf, int64_t cap) {
    if (!s) return -1;
    const std::string t = s->gp.text();
    if (buf && cap > (int64_t)t.size()) std::memcpy(buf, t.c_str(), t.size() + 1);
    return (int64_t)t.size() + 1;
}

sidr_status sidr_gp_population_packed(const sidr_gp_session* s, int32_t* ops, int32_t* args,
                                      int32_t* offsets, int32_t* lengths, int64_t* n_nodes) {
    if (!s || !n_nodes) return gp_fail(SIDR_ERR_INVALID, "null argument");
    std::vector<int32_t> o, a, off, len;
    s->gp.packed(o, a, off, len);
    *n_nodes = (int64_t)o.size();
    if (ops && args && offsets && lengths) {
        std::memcpy(ops, o.data(), o.size() * 4);
        std::memcpy(args, a.data(), a.size() * 4);
        std::memcpy(offsets, off.data(), off.size() * 4);
        std::memcpy(lengths, len.data(), len.size() * 4);
    }
    return SIDR_OK;
}

sidr_status sidr_gp_step(sidr_gp_session* s, const double* fitness) {
    if (!s || !fitness) return gp_fail(SIDR_ERR_INVALID, "null argument");
    std::vector<double> f(fitness, fitness + s->gp.pop.size());
    s->gp.step(f);
    s->generation++;
    return SIDR_OK;
}

int64_t sidr_gp_generation(const sidr_gp_session* s) { return s ? s->generation : -1; }

int64_t sidr_gp_checkpoint(const sidr_gp_session* s, char* buf, int64_t cap) {
    if (!s) return -1;
    const std::string t = sidr::gp::state_text(s->gp, s->generation);
    if (buf && cap > (int64_t)t.size()) std::memcpy(buf, t.c_str(), t.size() + 1);
    return (int64_t)t.size() + 1;
}

sidr_status sidr_gp_restore(const char* checkpoint, sidr_gp_session** out) {
    if (!out || !checkpoint) return gp_fail(SIDR_ERR_INVALID, "null argument");
    *out = nullptr;
    std::unique_ptr<Gp> g;
    int64_t generation = -1;
    const sidr_status st = sidr::gp::state_parse(checkpoint, g, generation);
    if (st != SIDR_OK) return st;
    std::unique_ptr<sidr_gp_session> s(new sidr_gp_session(g->cfg, 0));
    s->gp = *g;
    s->generation = generation;
    *out = s.release();
    return SIDR_OK;
}

sidr_status sidr_gen_durations(int32_t n, const double* durations, double sigma, int32_t S,
                               int64_t base_seed, double* out) {
    if (n < 0 || S < 0 || (n > 0 && (!durations || !out))) return gp_fail(SIDR_ERR_INVALID, "bad argument");
    for (int s = 0; s < S; s++) {
        Mt19937 rng((uint64_t)(base_seed + s));  // one fresh generator per scenario
        for (int i = 0; i < n; i++) {
            const double e = durations[i];
            double v = 0.0;
            if (e > 0.0) {  // zero-duration visits draw nothing
                v = rng.gauss(e, sigma * e);
                v = v > 0.0 ? v : 0.0;
            }
            out[(size_t)s * n + i] = v;
        }
    }
    return SIDR_OK;
}

sidr_status sidr_gp_batched_create(sidr_ctx* ctx, const sidr_instance_desc* inst, const sidr_gp_config* cfg,
                                   const char* terminals_csv, const int64_t* term_mask, int32_t n_seeds,
                                   int64_t first_seed, int64_t test_seed, sidr_gp_batched** out) {
    if (!out) return gp_fail(SIDR_ERR_INVALID, "out is null");
    *out = nullptr;
    std::string err;
    if (!ctx || !inst || !term_mask) return gp_fail(SIDR_ERR_INVALID, "null argument");
    if (!valid_config(cfg, err)) return gp_fail(SIDR_ERR_INVALID, err);
    if (n_seeds < 1) return gp_fail(SIDR_ERR_INVALID, "n_seeds < 1");
    if (inst->n < 1 || !inst->durations) return gp_fail(SIDR_ERR_INVALID, "instance without customers");
    std::vector<std::string> terms;
    if (!parse_terminals(terminals_csv, terms, err)) return gp_fail(SIDR_ERR_INVALID, err);
    std::unique_ptr<sidr_gp_batched> b(new sidr_gp_batched());
    b->ctx = ctx;
    b->n = inst->n;
    b->inst_hash = instance_hash(*inst);
    b->durations.assign(inst->durations, inst->durations + inst->n);
    b->cfg = *cfg;
    b->mask.assign(term_mask, term_mask + 61);
    b->first_seed = first_seed;
    b->test_seed = test_seed;
    for (int s = 0; s < n_seeds; s++) {
        sidr_gp_session* g = nullptr;
        const sidr_status st = sidr_gp_create(cfg, terminals_csv, (uint64_t)(first_seed + s), &g);
        if (st != SIDR_OK) return st;
        b->seeds.emplace_back(g);
    }
    *out = b.release();
    return SIDR_OK;
}

sidr_status sidr_gp_batched_step(sidr_gp_batched* b, int32_t generations) {
    if (!b || generations < 0) return gp_fail(SIDR_ERR_INVALID, "null run or generations < 0");
    const double t0 = seconds_now();
    const double e0 = b->t_eval;
    std::vector<std::vector<double>> fits;
    for (int k = 0; k < generations && b->gen < b->cfg.generations; k++) {
        const int gen = (int)b->gen;
        const sidr_status st = b->grouped_fit(gen, fits);
        if (st != SIDR_OK) return st;
        for (size_t s = 0; s < b->seeds.size(); s++) {
            double best = fits[s][0];
            for (double f : fits[s]) best = f > best ? f : best;
            b->best_train.push_back(best);
        }
        if (gen < b->cfg.generations - 1)
            for (size_t s = 0; s < b->seeds.size(); s++) sidr_gp_step(b->seeds[s].get(), fits[s].data());
        b->gen++;
    }
    b->t_host += seconds_now() - t0 - (b->t_eval - e0);
    return SIDR_OK;
}

int64_t sidr_gp_batched_generation(const sidr_gp_batched* b) { return b ? b->gen : -1; }

int64_t sidr_gp_batched_checkpoint(const sidr_gp_batched* b, char* buf, int64_t cap) {
    if (!b) return -1;
    std::string t = std::string(kBatchedHeader) + "\n";
    t += "seeds " + std::to_string(b->seeds.size()) + " " + std::to_string(b->first_seed) + " " +
         std::to_string(b->test_seed) + "\n";
    char hb[32];
    std::snprintf(hb, sizeof hb, "%016llx", (unsigned long long)b->inst_hash);
    t += "instance " + std::to_string(b->n) + " " + hb + "\n";
    t += "mask";
    for (int64_t v : b->mask) t += " " + std::to_string(v);
    t += "\n";
    t += "generation " + std::to_string(b->gen) + "\n";
    t += "counters " + hexf(b->t_eval) + " " + hexf(b->t_host) + " " + std::to_string(b->evals) + "\n";
    t += "best_train " + std::to_string(b->best_train.size()) + "\n";
    for (double v : b->best_train) t += hexf(v) + "\n";
    for (size_t s = 0; s < b->seeds.size(); s++) {
        const int64_t len = sidr_gp_checkpoint(b->seeds[s].get(), nullptr, 0);
        std::string st((size_t)len, '\0');
        sidr_gp_checkpoint(b->seeds[s].get(), &st[0], len);
        st.resize((size_t)len - 1);
        const size_t lines = (size_t)std::count(st.begin(), st.end(), '\n');
        t += "session " + std::to_string(s) + " " + std::to_string(lines) + "\n" + st;
    }
    if (buf && cap > (int64_t)t.size()) std::memcpy(buf, t.c_str(), t.size() + 1);
    return (int64_t)t.size() + 1;
}

sidr_status sidr_gp_batched_restore(sidr_ctx* ctx, const sidr_instance_desc* inst, const char* checkpoint,
                                    sidr_gp_batched** out) {
    if (!out) return gp_fail(SIDR_ERR_INVALID, "out is null");
    *out = nullptr;
    if (!ctx || !inst || !checkpoint) return gp_fail(SIDR_ERR_INVALID, "null argument");
    if (inst->n < 1 || !inst->durations) return gp_fail(SIDR_ERR_INVALID, "instance without customers");
    auto bad = [](const std::string& what) { return gp_fail(SIDR_ERR_INVALID, "batched checkpoint: " + what); };
    std::istringstream in(checkpoint);
    std::string line;
    if (!std::getline(in, line) || line != kBatchedHeader) return bad("not a seed-batched GP checkpoint of version 1");
    std::unique_ptr<sidr_gp_batched> b(new sidr_gp_batched());
    b->ctx = ctx;
    long long ns = -1, n = -1, gen = -1, evals = -1, nb = -1;
    char hb[32] = {0};
    if (!std::getline(in, line) ||
        std::sscanf(line.c_str(), "seeds %lld %lld %lld", &ns, (long long*)&b->first_seed,
                    (long long*)&b->test_seed) != 3 || ns < 1 || ns > (1 << 20))
        return bad("malformed seeds line");
    if (!std::getline(in, line) || std::sscanf(line.c_str(), "instance %lld %31s", &n, hb) != 2)
        return bad("malformed instance line");
    b->n = (int)n;
    b->inst_hash = std::strtoull(hb, nullptr, 16);
    if (n != inst->n || b->inst_hash != instance_hash(*inst))
        return bad("written for another instance");
    b->durations.assign(inst->durations, inst->durations + inst->n);
    {
        if (!std::getline(in, line)) return bad("no mask line");
        std::istringstream ls(line);
        std::string word;
        if (!(ls >> word) || word != "mask") return bad("malformed mask line");
        long long v;
        while (ls >> v) b->mask.push_back(v);
        if (b->mask.size() != 61) return bad("mask of " + std::to_string(b->mask.size()) + " flags");
    }
    if (!std::getline(in, line) || std::sscanf(line.c_str(), "generation %lld", &gen) != 1 || gen < 0)
        return bad("malformed generation line");
    b->gen = gen;
    {
        if (!std::getline(in, line)) return bad("no counters line");
        std::istringstream ls(line);
        std::string word, te, th;
        if (!(ls >> word >> te >> th >> evals) || word != "counters" || evals < 0) return bad("malformed counters");
        b->t_eval = std::strtod(te.c_str(), nullptr);
        b->t_host = std::strtod(th.c_str(), nullptr);
        b->evals = evals;
    }
    if (!std::getline(in, line) || std::sscanf(line.c_str(), "best_train %lld", &nb) != 1 || nb != gen * ns)
        return bad("best-train count differs from generation x seeds");
    for (long long i = 0; i < nb; i++) {
        if (!std::getline(in, line) || line.empty()) return bad("best-train values truncated");
        char* end = nullptr;
        b->best_train.push_back(std::strtod(line.c_str(), &end));
        if (!end || *end) return bad("malformed best-train value");
    }
    for (long long s = 0; s < ns; s++) {
        long long idx = -1, lines = -1;
        if (!std::getline(in, line) || std::sscanf(line.c_str(), "session %lld %lld", &idx, &lines) != 2 ||
            idx != s || lines < 1 || lines > (1 << 24))
            return bad("malformed session header");
        std::string text;
        for (long long k = 0; k < lines; k++) {
            if (!std::getline(in, line)) return bad("session " + std::to_string(s) + " truncated");
            text += line + "\n";
        }
        sidr_gp_session* g = nullptr;
        const sidr_status st = sidr_gp_restore(text.c_str(), &g);
        if (st != SIDR_OK) return st;
        b->seeds.emplace_back(g);
        // every session has stepped once per generation but the last
        const int64_t want = std::min<int64_t>(gen, g->gp.cfg.generations - 1);
        if (g->generation != want) return bad("session " + std::to_string(s) + " is at another generation");
        if (s == 0) {
            b->cfg = g->gp.cfg;
        } else if (!same_config(b->cfg, g->gp.cfg) ||
                   g->gp.vocab.terminals != b->seeds[0]->gp.vocab.terminals) {
            return bad("sessions of different configurations");
        }
    }
    if (gen > b->cfg.generations) return bad("generation beyond the run's end");
    if (std::getline(in, line) && !line.empty()) return bad("trailing text");
    *out = b.release();
    return SIDR_OK;
}

sidr_status sidr_gp_batched_finish(sidr_gp_batched* b, double* best_test, double* best_train, char* best_rules,
                                   int64_t rules_cap, sidr_gp_result* result) {
    if (!b) return gp_fail(SIDR_ERR_INVALID, "null run");
    if (b->gen != b->cfg.generations)
        return gp_fail(SIDR_ERR_INVALID, "the run has " + std::to_string(b->cfg.generations - b->gen) +
                                             " generations left");
    const double t0 = seconds_now();
    const double e0 = b->t_eval;
    const int n_seeds = (int)b->seeds.size(), ps = b->cfg.population, n = b->n;
    // final train block, best rule per population, held-out scoring
    std::vector<std::vector<double>> fits;
    sidr_status st = b->grouped_fit(b->cfg.generations, fits);
    if (st != SIDR_OK) return st;
    std::string rules_text;
    std::vector<int32_t> ops, args, off, len;
    for (int s = 0; s < n_seeds; s++) {
        const Gp& g = b->seeds[s]->gp;
        int bi = 0;
        for (int p = 1; p < ps; p++)
            if (fits[s][p] > fits[s][bi]) bi = p;
        g.packed(ops, args, off, len, (size_t)bi, 1);
        size_t k = 0;
        prefix_at(g.pop[bi], k, g.vocab, rules_text);
        rules_text += '\n';
    }
    if (b->cfg.test_samples > 0) {
        const int TS = b->cfg.test_samples;
        std::vector<double> test((size_t)TS * n);
        sidr_gen_durations(n, b->durations.data(), 0.2, TS, b->test_seed, test.data());
        sidr_rules_desc r{ops.data(), args.data(), off.data(), len.data(), (int32_t)off.size(),
                          (int64_t)ops.size()};
        std::vector<double> out((size_t)r.P * TS);
        const double q0 = seconds_now();
        st = sidr_evaluate(b->ctx, &r, test.data(), TS, b->mask.data(), out.data());
        b->t_eval += seconds_now() - q0;
        b->evals += (int64_t)r.P * TS;
        if (st != SIDR_OK) return gp_fail(st, std::string("held-out evaluation: ") + sidr_last_error());
        for (int s = 0; s < n_seeds; s++) {
            double acc = 0.0;
            for (int t = 0; t < TS; t++) acc += out[(size_t)s * TS + t];
            if (best_test) best_test[s] = acc / TS;
        }
    }
    if (best_train) std::memcpy(best_train, b->best_train.data(), b->best_train.size() * sizeof(double));
    if (best_rules && rules_cap > (int64_t)rules_text.size())
        std::memcpy(best_rules, rules_text.c_str(), rules_text.size() + 1);
    b->t_host += seconds_now() - t0 - (b->t_eval - e0);
    if (result) {
        result->eval_seconds = b->t_eval;
        result->host_seconds = b->t_host;
        result->evaluations = b->evals;
    }
    return SIDR_OK;
}

void sidr_gp_batched_destroy(sidr_gp_batched* b) { delete b; }

sidr_status sidr_gp_run_batched(sidr_ctx* ctx, const sidr_instance_desc* inst,
                                const sidr_gp_config* cfg, const char* terminals_csv,
                                const int64_t* term_mask, int32_t n_seeds, int64_t first_seed,
                                int64_t test_seed, double* best_test, double* best_train,
                                char* best_rules, int64_t rules_cap, sidr_gp_result* result) {
    sidr_gp_batched* b = nullptr;
    sidr_status st = sidr_gp_batched_create(ctx, inst, cfg, terminals_csv, term_mask, n_seeds, first_seed,
                                            test_seed, &b);
    std::unique_ptr<sidr_gp_batched> own(b);
    if (st == SIDR_OK) st = sidr_gp_batched_step(b, cfg->generations);
    if (st == SIDR_OK) st = sidr_gp_batched_finish(b, best_test, best_train, best_rules, rules_cap, result);
    return st;
}

sidr_status sidr_gp_run_multi(const sidr_instance_desc* insts, const double* zps, int32_t K,
                              const sidr_gp_config* cfg, const char* terminals_csv, const int64_t* masks,
                              int32_t n_seeds, int64_t first_seed, int64_t test_seed, int32_t shape,
                              int32_t device, double* best_test, double* best_train, char* best_rules,
                              int64_t rules_cap, sidr_gp_result* result) {
    using clock = std::chrono::steady_clock;
    std::string err;
    if (!insts || !zps || !masks) return gp_fail(SIDR_ERR_INVALID, "null argument");
    if (K < 1 || n_seeds < 1) return gp_fail(SIDR_ERR_INVALID, "K < 1 or n_seeds < 1");
    if ((int64_t)K * n_seeds > 32767) return gp_fail(SIDR_ERR_INVALID, "K * n_seeds > 32767");
    if (shape < -1 || shape >= SIDR_MULTI_SHAPES) return gp_fail(SIDR_ERR_INVALID, "shape out of range");
    if (!valid_config(cfg, err)) return gp_fail(SIDR_ERR_INVALID, err);
    for (int k = 0; k < K; k++)
        if (insts[k].n < 1 || !insts[k].durations)
            return gp_fail(SIDR_ERR_INVALID, "instance " + std::to_string(k) + ": no customers or no durations");
    std::vector<std::string> terms;
    if (!parse_terminals(terminals_csv, terms, err)) return gp_fail(SIDR_ERR_INVALID, err);
    const int ps = cfg->population, T = cfg->train_samples, E = K * n_seeds;
    double t_eval = 0.0;
    int64_t evals = 0;
    int chosen = shape;
    const auto t0 = clock::now();
    // population e = k * n_seeds + s: instance k, seed first_seed + s
    std::vector<Gp> gps;
    gps.reserve(E);
    for (int e = 0; e < E; e++) {
        gps.emplace_back(*cfg, (uint64_t)(first_seed + e % n_seeds));
        gps.back().vocab.terminals = terms;
        gps.back().vocab.n_funcs = cfg->with_rmod ? 7 : 6;
        gps.back().init();
    }
    // One multi-instance launch: entry q is instance ek[q] with the scenario
    // block blocks[q] ([Tn][n]); rule p belongs to entry owner[p]; out [P][Tn].
    auto launch = [&](const std::vector<int>& ek, const std::vector<std::vector<double>>& blocks, int Tn,
                      std::vector<int32_t>& ops, std::vector<int32_t>& args, std::vector<int32_t>& off,
                      std::vector<int32_t>& len, const std::vector<int32_t>& owner,
                      std::vector<double>& out) -> sidr_status {
        const int Q = (int)ek.size();
        std::vector<sidr_instance_desc> d(Q);
        std::vector<double> z((size_t)Q * 10), flat;
        std::vector<int64_t> mk((size_t)Q * 61), offs(Q);
        for (int q = 0; q < Q; q++) {
            d[q] = insts[ek[q]];
            std::copy(zps + 10 * (size_t)ek[q], zps + 10 * (size_t)ek[q] + 10, z.begin() + 10 * (size_t)q);
            std::copy(masks + 61 * (size_t)ek[q], masks + 61 * (size_t)ek[q] + 61, mk.begin() + 61 * (size_t)q);
            offs[q] = (int64_t)flat.size();
            flat.insert(flat.end(), blocks[q].begin(), blocks[q].end());
        }
        sidr_rules_desc r{ops.data(), args.data(), off.data(), len.data(), (int32_t)off.size(),
                          (int64_t)ops.size()};
        out.assign((size_t)r.P * Tn, 0.0);
        const auto e0 = clock::now();
        sidr_multi* m = nullptr;
        sidr_status st = sidr_multi_create(d.data(), z.data(), Q, &r, owner.data(), flat.data(),
                                           (int64_t)flat.size(), offs.data(), Tn, mk.data(), device, &m);
        if (st == SIDR_OK) st = chosen < 0 ? sidr_multi_autotune_sampled(m, 1, 16, &chosen, nullptr) : sidr_multi_set_shape(m, chosen);
        if (st == SIDR_OK) st = sidr_multi_run(m, nullptr);
        if (st == SIDR_OK) st = sidr_multi_read(m, out.data());
        const std::string why = st == SIDR_OK ? std::string() : std::string(sidr_last_error());
        sidr_multi_destroy(m);
        t_eval += std::chrono::duration<double>(clock::now() - e0).count();
        evals += (int64_t)r.P * Tn;
        if (st != SIDR_OK) return gp_fail(st, "evaluation: " + why);
        return SIDR_OK;
    };
    // every population on its own train block (base seed seed*10000 + gen) of its instance
    std::vector<std::vector<double>> fits(E, std::vector<double>(ps));
    auto train_fit = [&](int gen) -> sidr_status {
        std::vector<int32_t> ops, args, off, len, owner;
        std::vector<std::vector<double>> blocks(E);
        std::vector<int> ek(E);
        for (int e = 0; e < E; e++) {
            const int k = e / n_seeds, sd = e % n_seeds, n = insts[k].n;
            gps[e].packed(ops, args, off, len);
            owner.insert(owner.end(), ps, e);
            ek[e] = k;
            blocks[e].resize((size_t)T * n);
            sidr_gen_durations(n, insts[k].durations, 0.2, T, (first_seed + sd) * 10000 + gen, blocks[e].data());
        }
        std::vector<double> out;
        const sidr_status st = launch(ek, blocks, T, ops, args, off, len, owner, out);
        if (st != SIDR_OK) return st;
        for (int e = 0; e < E; e++)
            for (int p = 0; p < ps; p++) {
                double acc = 0.0;
                for (int t = 0; t < T; t++) acc += out[((size_t)e * ps + p) * T + t];
                fits[e][p] = acc / T;
            }
        return SIDR_OK;
    };
    for (int gen = 0; gen < cfg->generations; gen++) {
        const sidr_status st = train_fit(gen);
        if (st != SIDR_OK) return st;
        for (int e = 0; e < E; e++) {
            double b = fits[e][0];
            for (int p = 1; p < ps; p++) b = fits[e][p] > b ? fits[e][p] : b;
            if (best_train) best_train[(size_t)gen * E + e] = b;
        }
        if (gen < cfg->generations - 1)
            for (int e = 0; e < E; e++) gps[e].step(fits[e]);
    }
    // final train block, best rule per population, held-out scoring on each instance's test block
    sidr_status st = train_fit(cfg->generations);
    if (st != SIDR_OK) return st;
    std::string rules_text;
    std::vector<int32_t> ops, args, off, len, owner;
    for (int e = 0; e < E; e++) {
        int bi = 0;
        for (int p = 1; p < ps; p++)
            if (fits[e][p] > fits[e][bi]) bi = p;
        gps[e].packed(ops, args, off, len, (size_t)bi, 1);
        owner.push_back(e / n_seeds);
        size_t k = 0;
        prefix_at(gps[e].pop[bi], k, gps[e].vocab, rules_text);
        rules_text += '\n';
    }
    if (cfg->test_samples > 0) {
        const int TS = cfg->test_samples;
        std::vector<std::vector<double>> blocks(K);
        std::vector<int> ek(K);
        for (int k = 0; k < K; k++) {
            ek[k] = k;
            blocks[k].resize((size_t)TS * insts[k].n);
            sidr_gen_durations(insts[k].n, insts[k].durations, 0.2, TS, test_seed, blocks[k].data());
        }
        std::vector<double> out;
        if ((st = launch(ek, blocks, TS, ops, args, off, len, owner, out)) != SIDR_OK) return st;
        for (int e = 0; e < E; e++) {
            double acc = 0.0;
            for (int t = 0; t < TS; t++) acc += out[(size_t)e * TS + t];
            if (best_test) best_test[e] = acc / TS;
        }
    }
    if (best_rules && rules_cap > (int64_t)rules_text.size())
        std::memcpy(best_rules, rules_text.c_str(), rules_text.size() + 1);
    if (result) {
        result->eval_seconds = t_eval;
        result->host_seconds = std::chrono::duration<double>(clock::now() - t0).count() - t_eval;
        result->evaluations = evals;
    }
    return SIDR_OK;
}

}  // extern "C"
