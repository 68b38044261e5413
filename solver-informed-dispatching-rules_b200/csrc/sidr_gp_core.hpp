// sidr_gp_core.hpp -- the host GP's building blocks, shared by the GP driver
// (sidr_gp.cpp) and the campaign drivers (sidr_campaign.cpp).
//
// Rules are flat prefix-order arrays of nodes: a function node (opcode 0..6,
// two children) is followed by its left subtree, then its right subtree.  The
// subtree at pre-order position k spans [k, end(k)), so the reference's
// pre-order point numbering (engine/gp.hpp:99-118), subtree extraction and
// replacement are index ranges.  Every random draw goes through Mt19937, the
// same stream as the reference's Python-compatible generator (engine/rng.hpp).
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "../../include/sidr_gp.h"
#include "sidr_host.hpp"

namespace sidr {
namespace gp {

// ------------------------------------------------------------------ MT19937

class Mt19937 {
  public:
    explicit Mt19937(uint64_t seed) {
        // init_by_array over the 32-bit words of the seed, least significant
        // first; a single zero word for seed 0 (engine/rng.hpp:27-52)
        uint32_t key[2];
        int klen = 0;
        if (seed == 0) key[klen++] = 0;
        while (seed) {
            key[klen++] = (uint32_t)(seed & 0xffffffffu);
            seed >>= 32;
        }
        mt_[0] = 19650218u;
        for (int i = 1; i < kN; i++) mt_[i] = 1812433253u * (mt_[i - 1] ^ (mt_[i - 1] >> 30)) + (uint32_t)i;
        int i = 1, j = 0;
        for (int k = kN > klen ? kN : klen; k; k--) {
            mt_[i] = (mt_[i] ^ ((mt_[i - 1] ^ (mt_[i - 1] >> 30)) * 1664525u)) + key[j] + (uint32_t)j;
            if (++i >= kN) {
                mt_[0] = mt_[kN - 1];
                i = 1;
            }
            if (++j >= klen) j = 0;
        }
        for (int k = kN - 1; k; k--) {
            mt_[i] = (mt_[i] ^ ((mt_[i - 1] ^ (mt_[i - 1] >> 30)) * 1566083941u)) - (uint32_t)i;
            if (++i >= kN) {
                mt_[0] = mt_[kN - 1];
                i = 1;
            }
        }
        mt_[0] = 0x80000000u;
        mti_ = kN;
    }

    uint32_t next() {
        if (mti_ >= kN) {
            for (int k = 0; k < kN; k++) {
                const uint32_t y = (mt_[k] & 0x80000000u) | (mt_[(k + 1) % kN] & 0x7fffffffu);
                mt_[k] = mt_[(k + kM) % kN] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
            }
            mti_ = 0;
        }
        uint32_t y = mt_[mti_++];
        y ^= y >> 11;
        y ^= (y << 7) & 0x9d2c5680u;
        y ^= (y << 15) & 0xefc60000u;
        y ^= y >> 18;
        return y;
    }

    double random() {  // 53-bit double in [0,1) (engine/rng.hpp:78-81)
        const uint32_t a = next() >> 5, b = next() >> 6;
        return (a * 67108864.0 + b) * (1.0 / 9007199254740992.0);
    }

    uint64_t randbelow(uint64_t n) {  // rejection on the top bit_length(n) bits
        if (n == 0) return 0;
        int k = 0;
        for (uint64_t v = n; v; v >>= 1) k++;
        uint64_t r = next() >> (32 - k);
        while (r >= n) r = next() >> (32 - k);
        return r;
    }

    int64_t randint(int64_t a, int64_t b) { return a + (int64_t)randbelow((uint64_t)(b - a + 1)); }

    // k distinct indices of [0, n) (engine/rng.hpp:97-120)
    std::vector<size_t> sample(size_t n, size_t k) {
        std::vector<size_t> out(k);
        size_t setsize = 21;
        if (k > 5) setsize += (size_t)std::pow(4.0, std::ceil(std::log((double)(k * 3)) / std::log(4.0)));
        if (n <= setsize) {
            std::vector<size_t> pool(n);
            for (size_t i = 0; i < n; i++) pool[i] = i;
            for (size_t i = 0; i < k; i++) {
                const size_t j = (size_t)randbelow(n - i);
                out[i] = pool[j];
                pool[j] = pool[n - i - 1];
            }
        } else {
            std::unordered_set<size_t> taken;
            for (size_t i = 0; i < k; i++) {
                size_t j = (size_t)randbelow(n);
                while (taken.count(j)) j = (size_t)randbelow(n);
                taken.insert(j);
                out[i] = j;
            }
        }
        return out;
    }

    // Box-Muller with the spare value cached (engine/rng.hpp:135-147)
    double gauss(double mu, double sigma) {
        double z;
        if (has_spare_) {
            z = spare_;
            has_spare_ = false;
        } else {
            const double x2pi = random() * (2.0 * 3.14159265358979323846);
            const double g2rad = std::sqrt(-2.0 * std::log(1.0 - random()));
            z = std::cos(x2pi) * g2rad;
            spare_ = std::sin(x2pi) * g2rad;
            has_spare_ = true;
        }
        return mu + z * sigma;
    }

    // The generator's whole state as text (624 words, position, cached
    // Box-Muller value as a hexadecimal float), and back.
    std::string state() const {
        std::string out = std::to_string(mti_) + " " + (has_spare_ ? "1 " : "0 ");
        char buf[64];
        std::snprintf(buf, sizeof buf, "%a", spare_);
        out += buf;
        for (int k = 0; k < kN; k++) out += " " + std::to_string(mt_[k]);
        return out;
    }
    bool set_state(const std::string& text) {
        const char* p = text.c_str();
        char* e = nullptr;
        const long mti = std::strtol(p, &e, 10);
        if (e == p || mti < 0 || mti > kN + 1) return false;
        p = e;
        const long hs = std::strtol(p, &e, 10);
        if (e == p || (hs != 0 && hs != 1)) return false;
        p = e;
        const double sp = std::strtod(p, &e);
        if (e == p) return false;
        p = e;
        uint32_t mt[kN];
        for (int k = 0; k < kN; k++) {
            const unsigned long long v = std::strtoull(p, &e, 10);
            if (e == p || v > 0xffffffffull) return false;
            mt[k] = (uint32_t)v;
            p = e;
        }
        while (*p == ' ') p++;
        if (*p) return false;
        std::memcpy(mt_, mt, sizeof mt);
        mti_ = (int)mti;
        has_spare_ = hs == 1;
        spare_ = sp;
        return true;
    }

  private:
    static constexpr int kN = 624, kM = 397;
    uint32_t mt_[kN];
    int mti_ = kN + 1;
    bool has_spare_ = false;
    double spare_ = 0.0;
};

// ------------------------------------------------------------- vocabulary

inline const char* const kTermNames[61] = {
    "SCORE", "DUR", "TO", "TC", "TA", "TR", "TSV", "TFV", "SL", "RemT", "NS", "REGRET",
    "NSROB", "MAXN", "REACH2", "NSTW", "RAND", "FRAGCNT", "FRAGSCORE", "DOWNSLACK", "PBUST",
    "REACH1", "REACH3", "REACH5", "SAT", "VFRAC", "NFEAS", "VEH", "HARVEST", "BOLSAO",
    "ATRISK", "ZTC", "ZREACH", "ZWLOSS", "ZATRISK", "ZD2D", "C1", "C2", "C3", "C4", "C5",
    "REACH2ROB", "RELCOST", "NETREACH", "SKIPLOSS", "FRAGILITY", "SROB", "REACH3ROB",
    "REACH5ROB", "NSA2", "NSA05", "FEASCORE", "NFEASROB", "NSROB05", "NSROB2", "NNFWD",
    "NNK3", "NNCHAIN3", "SAVINGS", "DETOUR", "SCORERANK"};
inline const char* const kFuncNames[7] = {"+", "-", "*", "/", "min", "max", "rmod"};

// engine/vocab.hpp:73-81 (slot map and aliases)
inline int term_slot(const std::string& label) {
    for (int s = 0; s < 61; s++)
        if (label == kTermNames[s]) return s;
    if (label == "D2D") return 5;
    if (label == "SLACK") return 8;
    if (label == "WLOSS") return 11;
    return -1;
}

// A node: code >= 0 is a function opcode (two children); code < 0 is leaf
// label -code-1 of the session's label table.
using Rule = std::vector<int32_t>;

struct Vocab {
    std::vector<std::string> terminals;  // the configured terminal set
    int n_funcs = 6;
    std::vector<std::string> labels;     // leaf labels (terminals, then ERC texts)
    std::unordered_map<std::string, int> label_id;

    int leaf(const std::string& s) {
        auto it = label_id.find(s);
        if (it != label_id.end()) return it->second;
        const int id = (int)labels.size();
        labels.push_back(s);
        label_id.emplace(s, id);
        return id;
    }
};

inline size_t subtree_end(const Rule& r, size_t k) {
    int need = 1;
    while (need > 0) {
        need += (r[k] >= 0 ? 2 : 0) - 1;
        k++;
    }
    return k;
}

inline int depth_at(const Rule& r, size_t& k) {
    const int32_t c = r[k++];
    if (c < 0) return 0;
    const int a = depth_at(r, k);
    const int b = depth_at(r, k);
    return 1 + (a > b ? a : b);
}

inline int depth(const Rule& r) {
    size_t k = 0;
    return depth_at(r, k);
}

inline void prefix_at(const Rule& r, size_t& k, const Vocab& v, std::string& out) {
    const int32_t c = r[k++];
    if (c < 0) {
        out += v.labels[-c - 1];
        return;
    }
    out += "(";
    out += kFuncNames[c];
    out += " ";
    prefix_at(r, k, v, out);
    out += " ";
    prefix_at(r, k, v, out);
    out += ")";
}

// Post-order flatten (engine/vocab.hpp:99-126) appended to ops/args; returns
// the node's index within its rule (ops entries from `base` on).
inline int32_t compile_at(const Rule& r, size_t& k, const Vocab& v, std::vector<int32_t>& ops,
                   std::vector<int32_t>& args, size_t base) {
    const int32_t c = r[k++];
    if (c < 0) {
        const std::string& lab = v.labels[-c - 1];
        const int s = term_slot(lab);
        if (s >= 0) {
            ops.push_back(-1);
            args.push_back(s);
        } else {
            ops.push_back(-2);
            args.push_back((int32_t)std::llround(std::strtod(lab.c_str(), nullptr) * 1000.0));
        }
        args.push_back(0);
        return (int32_t)(ops.size() - 1 - base);
    }
    const int32_t left = compile_at(r, k, v, ops, args, base);
    const int32_t right = compile_at(r, k, v, ops, args, base);
    ops.push_back(c);
    args.push_back(left);
    args.push_back(right);
    return (int32_t)(ops.size() - 1 - base);
}

// ------------------------------------------------------------ GP operators

struct Gp {
    sidr_gp_config cfg;
    Vocab vocab;
    Mt19937 rng;
    std::vector<Rule> pop;

    Gp(const sidr_gp_config& c, uint64_t seed) : cfg(c), rng(seed) {}

    // pick_terminal (engine/gp.hpp:37-45)
    void terminal(Rule& out) {
        const std::string& t = vocab.terminals[rng.randbelow(vocab.terminals.size())];
        if (t == "ERC") {
            char buf[32];
            std::snprintf(buf, sizeof buf, "%.3f", rng.random());
            out.push_back(-vocab.leaf(buf) - 1);
            return;
        }
        out.push_back(-vocab.leaf(t) - 1);
    }

    void full(Rule& out, int d) {  // generate_full (:47-53)
        if (d <= 0) {
            terminal(out);
            return;
        }
        out.push_back((int32_t)rng.randbelow(vocab.n_funcs));
        full(out, d - 1);
        full(out, d - 1);
    }

    void grow(Rule& out, int d) {  // generate_grow (:55-63)
        if (d <= 0) {
            terminal(out);
            return;
        }
        const double nt = (double)vocab.terminals.size(), nf = (double)vocab.n_funcs;
        if (rng.random() < nt / (nt + nf)) {
            terminal(out);
            return;
        }
        out.push_back((int32_t)rng.randbelow(vocab.n_funcs));
        grow(out, d - 1);
        grow(out, d - 1);
    }

    void init() {  // ramped_half_and_half (:67-77)
        pop.clear();
        const int nd = cfg.max_depth - cfg.min_depth + 1;
        for (int i = 0; i < cfg.population; i++) {
            Rule r;
            const int d = cfg.min_depth + i % nd;
            if ((i / nd) % 2 == 0) full(r, d);
            else grow(r, d);
            pop.push_back(std::move(r));
        }
    }

    // select_crossover_point (:120-131): Koza 90/10 internal/leaf choice
    size_t point(const Rule& r) {
        std::vector<size_t> internals, leaves;
        for (size_t k = 0; k < r.size(); k++) (r[k] >= 0 ? internals : leaves).push_back(k);
        if (!internals.empty() && (leaves.empty() || rng.random() < 0.9))
            return internals[rng.randbelow(internals.size())];
        if (!leaves.empty()) return leaves[rng.randbelow(leaves.size())];
        return internals[rng.randbelow(internals.size())];
    }

    static Rule replaced(const Rule& r, size_t at, const Rule& with, size_t w0, size_t w1) {
        const size_t e = subtree_end(r, at);
        Rule out;
        out.reserve(r.size() - (e - at) + (w1 - w0));
        out.insert(out.end(), r.begin(), r.begin() + at);
        out.insert(out.end(), with.begin() + w0, with.begin() + w1);
        out.insert(out.end(), r.begin() + e, r.end());
        return out;
    }

    // subtree_crossover (:133-144)
    void crossover(const Rule& p1, const Rule& p2, Rule& c1, Rule& c2) {
        const size_t a = point(p1), b = point(p2);
        const size_t ae = subtree_end(p1, a), be = subtree_end(p2, b);
        c1 = replaced(p1, a, p2, b, be);
        c2 = replaced(p2, b, p1, a, ae);
        if (depth(c1) > cfg.max_depth) c1 = p1;
        if (depth(c2) > cfg.max_depth) c2 = p2;
    }

    // subtree_mutation (:146-153)
    Rule mutate(const Rule& ind) {
        const size_t at = point(ind);
        const int d = (int)rng.randint(cfg.min_depth, cfg.max_depth);
        Rule sub;
        grow(sub, d);
        Rule m = replaced(ind, at, sub, 0, sub.size());
        if (depth(m) > cfg.max_depth) return ind;
        return m;
    }

    // tournament_selection (:157-166)
    const Rule& tournament(const std::vector<double>& fit) {
        const size_t k = std::min((size_t)cfg.tournament, pop.size());
        const std::vector<size_t> c = rng.sample(pop.size(), k);
        size_t best = c[0];
        for (size_t t = 1; t < c.size(); t++)
            if (fit[c[t]] > fit[best]) best = c[t];
        return pop[best];
    }

    // gp_step (:170-194)
    void step(const std::vector<double>& fit) {
        std::vector<int> order(pop.size());
        for (size_t i = 0; i < pop.size(); i++) order[i] = (int)i;
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return fit[a] > fit[b]; });
        std::vector<Rule> next;
        next.reserve(cfg.population);
        for (int e = 0; e < cfg.elitism && e < (int)order.size(); e++) next.push_back(pop[order[e]]);
        while ((int)next.size() < cfg.population) {
            const double r = rng.random();
            if (r < cfg.crossover_rate) {
                const Rule& p1 = tournament(fit);
                const Rule& p2 = tournament(fit);
                Rule c1, c2;
                crossover(p1, p2, c1, c2);
                next.push_back(std::move(c1));
                if ((int)next.size() < cfg.population) next.push_back(std::move(c2));
            } else if (r < cfg.crossover_rate + cfg.mutation_rate) {
                const Rule& p = tournament(fit);
                next.push_back(mutate(p));
            } else {
                next.push_back(tournament(fit));
            }
        }
        next.resize(cfg.population);
        pop.swap(next);
    }

    // gp_step's breeding loop (engine/gp.hpp:178-192) on its own: `count`
    // children of the current population (crossover pairs, mutation,
    // reproduction, each parent by tournament), no elites.
    std::vector<Rule> breed(const std::vector<double>& fit, size_t count) {
        std::vector<Rule> next;
        next.reserve(count);
        while (next.size() < count) {
            const double r = rng.random();
            if (r < cfg.crossover_rate) {
                const Rule& p1 = tournament(fit);
                const Rule& p2 = tournament(fit);
                Rule c1, c2;
                crossover(p1, p2, c1, c2);
                next.push_back(std::move(c1));
                if (next.size() < count) next.push_back(std::move(c2));
            } else if (r < cfg.crossover_rate + cfg.mutation_rate) {
                const Rule& p = tournament(fit);
                next.push_back(mutate(p));
            } else {
                next.push_back(tournament(fit));
            }
        }
        return next;
    }

    std::string text() const {
        std::string out;
        for (const Rule& r : pop) {
            size_t k = 0;
            prefix_at(r, k, vocab, out);
            out += '\n';
        }
        return out;
    }

    void packed(std::vector<int32_t>& ops, std::vector<int32_t>& args, std::vector<int32_t>& offsets,
                std::vector<int32_t>& lengths, size_t first = 0, size_t count = SIZE_MAX) const {
        const size_t last = std::min(pop.size(), count == SIZE_MAX ? pop.size() : first + count);
        for (size_t p = first; p < last; p++) {
            offsets.push_back((int32_t)ops.size());
            size_t k = 0;
            compile_at(pop[p], k, vocab, ops, args, ops.size());
            lengths.push_back((int32_t)ops.size() - offsets.back());
        }
    }
};

// Records the failure for sidr_last_error() and returns its status.
inline sidr_status gp_fail(sidr_status s, const std::string& m) {
    sidr::set_last_error(m);
    return s;
}

inline bool parse_terminals(const char* csv, std::vector<std::string>& out, std::string& err) {
    out.clear();
    if (!csv) {
        err = "terminal set is null";
        return false;
    }
    std::string cur;
    for (const char* p = csv;; ++p) {
        if (*p == ',' || *p == '\0') {
            if (!cur.empty()) {
                if (cur != "ERC" && term_slot(cur) < 0) {
                    err = "unknown terminal " + cur;
                    return false;
                }
                out.push_back(cur);
            }
            cur.clear();
            if (*p == '\0') break;
        } else if (*p != ' ') {
            cur += *p;
        }
    }
    if (out.empty()) {
        err = "empty terminal set";
        return false;
    }
    return true;
}

inline bool same_config(const sidr_gp_config& a, const sidr_gp_config& b) {
    return a.population == b.population && a.generations == b.generations && a.max_depth == b.max_depth &&
           a.min_depth == b.min_depth && a.tournament == b.tournament && a.elitism == b.elitism &&
           a.crossover_rate == b.crossover_rate && a.mutation_rate == b.mutation_rate &&
           a.reproduction_rate == b.reproduction_rate && a.train_samples == b.train_samples &&
           a.test_samples == b.test_samples && a.with_rmod == b.with_rmod;
}

// FNV-1a over the instance's size, limits and arrays: a checkpoint resumes
// only on the instance it was written for.
inline uint64_t instance_hash(const sidr_instance_desc& d) {
    uint64_t h = 1469598103934665603ull;
    auto mix = [&](const void* p, size_t bytes) {
        const unsigned char* c = static_cast<const unsigned char*>(p);
        for (size_t i = 0; i < bytes; i++) h = (h ^ c[i]) * 1099511628211ull;
    };
    mix(&d.n, sizeof d.n);
    mix(&d.m, sizeof d.m);
    mix(&d.tmax, sizeof d.tmax);
    const size_t n = d.n > 0 ? (size_t)d.n : 0;
    for (const double* a : {d.scores, d.durations, d.open_t, d.close_t, d.dist_to_depot})
        if (a) mix(a, n * sizeof(double));
    if (d.dist) mix(d.dist, (n + 1) * (n + 1) * sizeof(double));
    return h;
}

// A GP's whole state as the text of sidr_gp_checkpoint (config, step count,
// terminal set, leaf labels, generator state, population), and back;
// state_parse refuses malformed text (SIDR_ERR_INVALID).  In sidr_gp.cpp.
std::string state_text(const Gp& g, int64_t generation);
sidr_status state_parse(const std::string& text, std::unique_ptr<Gp>& out, int64_t& generation);

inline bool valid_config(const sidr_gp_config* c, std::string& err) {
    if (!c) {
        err = "config is null";
        return false;
    }
    if (c->population < 1 || c->generations < 1 || c->min_depth < 0 || c->max_depth < c->min_depth ||
        c->max_depth > 8 || c->tournament < 1 || c->elitism < 0 || c->train_samples < 1 ||
        c->test_samples < 0) {
        err = "config out of range (population, generations >= 1; 0 <= min_depth <= max_depth <= 8)";
        return false;
    }
    return true;
}

}  // namespace gp
}  // namespace sidr
