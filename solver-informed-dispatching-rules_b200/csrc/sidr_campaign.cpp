// sidr_campaign.cpp -- the campaign drivers of include/sidr_campaign.h: the
// vocabulary GA (s4_selection/ga.cu), the generation trace
// (s3_generation/gen_trace.cu), redeploy sealing (s4_selection/redeploy.cu)
// and the train-side score of the cross-validatory choice
// (s4_selection/choice.cu), on the host GP of sidr_gp_core.hpp and the B200
// evaluator.
#include <algorithm>
#include <array>
#include <atomic>
#include <cctype>
#include <charconv>
#include <chrono>
#include <cstdarg>
#include <map>
#include <memory>
#include <set>
#include <thread>

#include "../../include/sidr_campaign.h"
#include "sidr_gp_core.hpp"

using namespace sidr::gp;

namespace {

double now_s() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

// Runs f(i) for i in [0, n) on the host's cores.  Every call is independent
// (one population each), so the result does not depend on the schedule.
template <class F>
void parallel_for(int n, F&& f) {
    const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
    const int nt = std::min(n, hw);
    if (nt <= 1) {
        for (int i = 0; i < n; i++) f(i);
        return;
    }
    std::atomic<int> next{0};
    std::vector<std::thread> ts;
    for (int t = 0; t < nt; t++)
        ts.emplace_back([&] {
            for (int i = next++; i < n; i = next++) f(i);
        });
    for (auto& t : ts) t.join();
}

// printf into a growing string (the programs' stdout).
struct Log {
    std::string text;
    void operator()(const char* fmt, ...) __attribute__((format(printf, 2, 3))) {
        char buf[1024];
        va_list ap;
        va_start(ap, fmt);
        const int k = std::vsnprintf(buf, sizeof buf, fmt, ap);
        va_end(ap);
        if (k > 0) text.append(buf, std::min(k, (int)sizeof buf - 1));
    }
};

// term_mask_from (engine/sim_host.hpp:85-94): ERC skipped.
std::vector<int64_t> mask_of(const std::vector<std::string>& terms) {
    std::vector<int64_t> m(61, 0);
    for (const auto& t : terms)
        if (t != "ERC") m[term_slot(t)] = 1;
    return m;
}

// The terminal sets of a genome family: base + universe[b] for each set bit b
// (s4_selection/ga.cu:90-95).
struct Universe {
    std::vector<std::string> base, uni;
    int nb = 0;

    std::vector<std::string> vocab_of(uint32_t g) const {
        std::vector<std::string> v = base;
        for (int b = 0; b < nb; b++)
            if (g >> b & 1u) v.push_back(uni[b]);
        return v;
    }
    std::string name_of(uint32_t g) const {  // ga.cu:96-101
        std::string s;
        for (int b = 0; b < nb; b++)
            if (g >> b & 1u) s += (s.empty() ? "" : ",") + uni[b];
        return s.empty() ? std::string("(base)") : s;
    }
};

sidr_status load_universe(const char* base_csv, const char* universe_csv, Universe& u) {
    std::string err;
    if (!parse_terminals(base_csv, u.base, err)) return gp_fail(SIDR_ERR_INVALID, "base set: " + err);
    if (!parse_terminals(universe_csv, u.uni, err)) return gp_fail(SIDR_ERR_INVALID, "universe: " + err);
    u.nb = (int)u.uni.size();
    if (u.nb > 30) return gp_fail(SIDR_ERR_INVALID, "universe holds more than 30 terminals");
    return SIDR_OK;
}

int nbits(uint32_t g) { return __builtin_popcount(g); }

double mean_of(const std::vector<double>& v) {
    double a = 0.0;
    for (double x : v) a += x;
    return a / v.size();
}

// Per-population means of a grouped result: out[(g*ps + p)*T + t].
void population_means(const std::vector<double>& out, int groups, int ps, int T,
                      std::vector<std::vector<double>>& f) {
    f.assign(groups, std::vector<double>(ps));
    for (int g = 0; g < groups; g++)
        for (int p = 0; p < ps; p++) {
            double acc = 0.0;
            for (int t = 0; t < T; t++) acc += out[((size_t)g * ps + p) * T + t];
            f[g][p] = acc / T;
        }
}

size_t best_index(const std::vector<double>& f) {  // strict >, first index
    size_t b = 0;
    for (size_t p = 1; p < f.size(); p++)
        if (f[p] > f[b]) b = p;
    return b;
}

struct Packed {
    std::vector<int32_t> ops, args, off, len;
    sidr_rules_desc desc() {
        return sidr_rules_desc{ops.data(), args.data(), off.data(), len.data(), (int32_t)off.size(),
                               (int64_t)ops.size()};
    }
};

void pack_rule(const Gp& g, size_t p, Packed& pk) { g.packed(pk.ops, pk.args, pk.off, pk.len, p, 1); }

// Every population's rules, compiled on the host's cores, concatenated in
// population order (offsets as if packed one after another).
void pack_all(const std::vector<std::unique_ptr<Gp>>& pops, Packed& pk) {
    std::vector<Packed> part(pops.size());
    parallel_for((int)pops.size(), [&](int i) { pops[i]->packed(part[i].ops, part[i].args, part[i].off, part[i].len); });
    for (const Packed& q : part) {
        const int32_t base = (int32_t)pk.ops.size();
        for (int32_t o : q.off) pk.off.push_back(o + base);
        pk.len.insert(pk.len.end(), q.len.begin(), q.len.end());
        pk.ops.insert(pk.ops.end(), q.ops.begin(), q.ops.end());
        pk.args.insert(pk.args.end(), q.args.begin(), q.args.end());
    }
}

std::vector<double> durations_block(const sidr_instance_desc* inst, int S, long long seed) {
    std::vector<double> v((size_t)S * inst->n);
    sidr_gen_durations(inst->n, inst->durations, 0.2, S, seed, v.data());
    return v;
}

std::unique_ptr<Gp> new_population(const sidr_gp_config& cfg, uint64_t seed,
                                   const std::vector<std::string>& terms) {
    std::unique_ptr<Gp> g(new Gp(cfg, seed));
    g->vocab.terminals = terms;
    g->vocab.n_funcs = cfg.with_rmod ? 7 : 6;
    return g;
}

// ----------------------------------------------------------- batch_score

struct Scorer {
    sidr_ctx* ctx;
    const sidr_instance_desc* inst;
    sidr_gp_config cfg;
    const Universe& u;
    long long block_seed;
    int block_n;
    double t_eval = 0.0;
    int64_t n_evals = 0;

    sidr_status grouped_masks(Packed& pk, const std::vector<double>& grouped, int G, int T,
                              int group_size, int mask_group, const std::vector<int64_t>& masks,
                              std::vector<double>& out) {
        sidr_rules_desc r = pk.desc();
        out.assign((size_t)r.P * T, 0.0);
        const double t0 = now_s();
        const sidr_status st = sidr_evaluate_grouped_masks(ctx, &r, grouped.data(), G, T, group_size,
                                                           mask_group, masks.data(), out.data());
        t_eval += now_s() - t0;
        n_evals += (int64_t)r.P * T;
        if (st != SIDR_OK) return gp_fail(st, std::string("evaluation: ") + sidr_last_error());
        return SIDR_OK;
    }

    // One chunk of genomes in lockstep (s4_selection/ga.cu:116-203).
    sidr_status chunk(const uint32_t* gs, int kb, int n, int ng, double* res) {
        const int ps = cfg.population, T = cfg.train_samples, nn = inst->n;
        std::vector<int64_t> mask_flat;
        std::vector<std::unique_ptr<Gp>> pops;  // [kb][n]
        for (int k = 0; k < kb; k++) {
            const std::vector<std::string> voc = u.vocab_of(gs[k]);
            const std::vector<int64_t> m = mask_of(voc);
            mask_flat.insert(mask_flat.end(), m.begin(), m.end());
            for (int s = 0; s < n; s++) pops.push_back(new_population(cfg, (uint64_t)s, voc));
        }
        parallel_for((int)pops.size(), [&](int i) { pops[i]->init(); });
        std::vector<std::vector<double>> f;
        auto gfit = [&](int gen_id) -> sidr_status {
            Packed pk;
            pack_all(pops, pk);
            // the train block of seed s repeats for every genome
            std::vector<double> grouped((size_t)kb * n * T * nn);
            for (int s = 0; s < n; s++) {
                const std::vector<double> one = durations_block(inst, T, (long long)s * 10000 + gen_id);
                for (int k = 0; k < kb; k++)
                    std::copy(one.begin(), one.end(), grouped.begin() + ((size_t)k * n + s) * T * nn);
            }
            std::vector<double> out;
            const sidr_status st = grouped_masks(pk, grouped, kb * n, T, ps, n * ps, mask_flat, out);
            if (st != SIDR_OK) return st;
            population_means(out, kb * n, ps, T, f);
            return SIDR_OK;
        };
        for (int gen = 0; gen < ng; gen++) {
            const sidr_status st = gfit(gen);
            if (st != SIDR_OK) return st;
            if (gen < ng - 1) parallel_for((int)pops.size(), [&](int i) { pops[i]->step(f[i]); });
        }
        sidr_status st = gfit(ng);
        if (st != SIDR_OK) return st;
        Packed fin;
        for (size_t i = 0; i < pops.size(); i++) pack_rule(*pops[i], best_index(f[i]), fin);
        const std::vector<double> blk = durations_block(inst, block_n, block_seed);
        std::vector<double> blk_rep;
        for (int k = 0; k < kb; k++) blk_rep.insert(blk_rep.end(), blk.begin(), blk.end());
        std::vector<double> out;
        if ((st = grouped_masks(fin, blk_rep, kb, block_n, n, n, mask_flat, out)) != SIDR_OK) return st;
        for (int k = 0; k < kb; k++)
            for (int s = 0; s < n; s++) {
                double acc = 0.0;
                for (int t = 0; t < block_n; t++) acc += out[((size_t)k * n + s) * block_n + t];
                res[(size_t)k * n + s] = acc / block_n;
            }
        return SIDR_OK;
    }

    // seq_score (s4_selection/ga.cu:208-258).
    sidr_status sequential(uint32_t g, int n, int ng, double* res) {
        const int ps = cfg.population, T = cfg.train_samples, nn = inst->n;
        const std::vector<std::string> voc = u.vocab_of(g);
        const std::vector<int64_t> tm = mask_of(voc);
        std::vector<std::unique_ptr<Gp>> pops;
        for (int s = 0; s < n; s++) {
            pops.push_back(new_population(cfg, (uint64_t)s, voc));
            pops.back()->init();
        }
        std::vector<std::vector<double>> f;
        auto gfit = [&](int gen_id) -> sidr_status {
            Packed pk;
            pack_all(pops, pk);
            std::vector<double> grouped((size_t)n * T * nn);
            for (int s = 0; s < n; s++) {
                const std::vector<double> one = durations_block(inst, T, (long long)s * 10000 + gen_id);
                std::copy(one.begin(), one.end(), grouped.begin() + (size_t)s * T * nn);
            }
            sidr_rules_desc r = pk.desc();
            std::vector<double> out((size_t)r.P * T);
            const double t0 = now_s();
            const sidr_status st =
                sidr_evaluate_grouped(ctx, &r, grouped.data(), n, T, ps, tm.data(), out.data());
            t_eval += now_s() - t0;
            n_evals += (int64_t)r.P * T;
            if (st != SIDR_OK) return gp_fail(st, std::string("evaluation: ") + sidr_last_error());
            population_means(out, n, ps, T, f);
            return SIDR_OK;
        };
        for (int gen = 0; gen < ng; gen++) {
            const sidr_status st = gfit(gen);
            if (st != SIDR_OK) return st;
            if (gen < ng - 1)
                for (int s = 0; s < n; s++) pops[s]->step(f[s]);
        }
        sidr_status st = gfit(ng);
        if (st != SIDR_OK) return st;
        Packed fin;
        for (int s = 0; s < n; s++) pack_rule(*pops[s], best_index(f[s]), fin);
        const std::vector<double> blk = durations_block(inst, block_n, block_seed);
        sidr_rules_desc r = fin.desc();
        std::vector<double> out((size_t)n * block_n);
        const double t0 = now_s();
        st = sidr_evaluate(ctx, &r, blk.data(), block_n, tm.data(), out.data());
        t_eval += now_s() - t0;
        n_evals += (int64_t)n * block_n;
        if (st != SIDR_OK) return gp_fail(st, std::string("evaluation: ") + sidr_last_error());
        for (int s = 0; s < n; s++) {
            double acc = 0.0;
            for (int t = 0; t < block_n; t++) acc += out[(size_t)s * block_n + t];
            res[s] = acc / block_n;
        }
        return SIDR_OK;
    }
};

sidr_status check_common(sidr_ctx* ctx, const sidr_instance_desc* inst, const sidr_gp_config* cfg,
                         int n_seeds, int n_gens, int block_n) {
    std::string err;
    if (!ctx || !inst) return gp_fail(SIDR_ERR_INVALID, "null context or instance");
    if (!valid_config(cfg, err)) return gp_fail(SIDR_ERR_INVALID, err);
    if (n_seeds < 1 || n_gens < 0 || block_n < 1)
        return gp_fail(SIDR_ERR_INVALID, "n_seeds >= 1, n_gens >= 0 and block_n >= 1 are required");
    return SIDR_OK;
}

// ------------------------------------------------------------------- JSON

// A small JSON reader for the trace files (objects, arrays, strings,
// numbers, true/false/null), enough for engine/json.hpp's uses here.
struct JVal {
    enum Kind { NUL, BOOL, NUM, STR, ARR, OBJ } kind = NUL;
    double num = 0.0;
    std::string str;
    std::vector<JVal> arr;
    std::vector<std::pair<std::string, JVal>> obj;

    const JVal* get(const std::string& k) const {
        for (const auto& kv : obj)
            if (kv.first == k) return &kv.second;
        return nullptr;
    }
};

struct JParser {
    const char* p;
    const char* e;
    std::string err;

    void ws() {
        while (p < e && (*p == ' ' || *p == '\n' || *p == '\r' || *p == '\t')) p++;
    }
    bool fail(const char* m) {
        if (err.empty()) err = m;
        return false;
    }
    bool string(std::string& out) {
        if (p >= e || *p != '"') return fail("expected a string");
        p++;
        while (p < e && *p != '"') {
            char c = *p++;
            if (c == '\\') {
                if (p >= e) return fail("bad escape");
                const char x = *p++;
                switch (x) {
                case 'n': c = '\n'; break;
                case 't': c = '\t'; break;
                case 'r': c = '\r'; break;
                case 'b': c = '\b'; break;
                case 'f': c = '\f'; break;
                case 'u': {
                    if (e - p < 4) return fail("bad escape");
                    const unsigned v = (unsigned)std::strtoul(std::string(p, 4).c_str(), nullptr, 16);
                    p += 4;
                    if (v < 0x80) {
                        c = (char)v;
                    } else if (v < 0x800) {
                        out += (char)(0xc0 | (v >> 6));
                        c = (char)(0x80 | (v & 0x3f));
                    } else {
                        out += (char)(0xe0 | (v >> 12));
                        out += (char)(0x80 | ((v >> 6) & 0x3f));
                        c = (char)(0x80 | (v & 0x3f));
                    }
                    break;
                }
                default: c = x;
                }
            }
            out += c;
        }
        if (p >= e) return fail("unterminated string");
        p++;
        return true;
    }
    bool value(JVal& v, int depth) {
        if (depth > 64) return fail("nesting too deep");
        ws();
        if (p >= e) return fail("unexpected end");
        if (*p == '{' || *p == '[') {
            const bool obj = *p == '{';
            const char close = obj ? '}' : ']';
            v.kind = obj ? JVal::OBJ : JVal::ARR;
            p++;
            ws();
            if (p < e && *p == close) {
                p++;
                return true;
            }
            for (;;) {
                ws();
                if (obj) {
                    std::string k;
                    if (!string(k)) return false;
                    ws();
                    if (p >= e || *p != ':') return fail("expected ':'");
                    p++;
                    v.obj.emplace_back(k, JVal());
                    if (!value(v.obj.back().second, depth + 1)) return false;
                } else {
                    v.arr.emplace_back();
                    if (!value(v.arr.back(), depth + 1)) return false;
                }
                ws();
                if (p < e && *p == ',') {
                    p++;
                    continue;
                }
                if (p < e && *p == close) {
                    p++;
                    return true;
                }
                return fail("expected ',' or a closing bracket");
            }
        }
        if (*p == '"') {
            v.kind = JVal::STR;
            return string(v.str);
        }
        if (e - p >= 4 && std::strncmp(p, "true", 4) == 0) {
            v.kind = JVal::BOOL;
            v.num = 1.0;
            p += 4;
            return true;
        }
        if (e - p >= 5 && std::strncmp(p, "false", 5) == 0) {
            v.kind = JVal::BOOL;
            p += 5;
            return true;
        }
        if (e - p >= 4 && std::strncmp(p, "null", 4) == 0) {
            p += 4;
            return true;
        }
        const char* q = p;
        while (q < e && (std::isdigit((unsigned char)*q) || *q == '-' || *q == '+' || *q == '.' ||
                         *q == 'e' || *q == 'E'))
            q++;
        if (q == p) return fail("unexpected character");
        v.kind = JVal::NUM;
        v.num = std::strtod(std::string(p, q).c_str(), nullptr);
        p = q;
        return true;
    }
};

sidr_status parse_json(const char* text, JVal& out) {
    if (!text) return gp_fail(SIDR_ERR_INVALID, "trace text is null");
    JParser jp{text, text + std::strlen(text), {}};
    if (!jp.value(out, 0)) return gp_fail(SIDR_ERR_INVALID, "trace JSON: " + jp.err);
    return SIDR_OK;
}

// ------------------------------------------------------------ JSON writing

// engine/jwrite.hpp: decimal rounding half to even, integral doubles with a
// trailing ".0", others as the shortest round-trip text.
double round_half_even(double x, int k) {
    const double m = std::pow(10.0, k);
    const double v = x * m;
    const double f = std::floor(v);
    const double diff = v - f;
    double r;
    if (diff > 0.5) r = f + 1;
    else if (diff < 0.5) r = f;
    else r = (std::fmod(f, 2.0) == 0.0) ? f : f + 1;
    return r / m;
}

std::string jnum(double x) {
    if (x == (long long)x && std::abs(x) < 1e15) return std::to_string((long long)x) + ".0";
    char buf[32];
    auto r = std::to_chars(buf, buf + sizeof buf, x);
    return std::string(buf, r.ptr);
}

std::string jstr(const std::string& s) {
    std::string o = "\"";
    for (char c : s) {
        if (c == '"' || c == '\\') {
            o += '\\';
            o += c;
        } else if (c == '\n') {
            o += "\\n";
        } else {
            o += c;
        }
    }
    return o + "\"";
}

std::string jlist(const std::vector<std::string>& parts) {
    std::string o = "[";
    for (size_t i = 0; i < parts.size(); i++) o += (i ? ", " : "") + parts[i];
    return o + "]";
}

std::string jstrlist(const std::vector<std::string>& v) {
    std::vector<std::string> p;
    for (const auto& s : v) p.push_back(jstr(s));
    return jlist(p);
}

// The extra terminals a rule uses (s3_generation/gen_trace.cu:36-47): its
// distinct leaf labels outside the base set, numbers left out, sorted.
std::vector<std::string> extras_of(const Rule& r, const Vocab& v, const std::set<std::string>& base) {
    std::set<std::string> toks;
    for (int32_t c : r)
        if (c < 0) toks.insert(v.labels[-c - 1]);
    std::vector<std::string> out;
    for (const auto& x : toks) {
        if (base.count(x)) continue;
        std::string d = x;
        d.erase(std::remove(d.begin(), d.end(), '.'), d.end());
        const bool num =
            !d.empty() && std::all_of(d.begin(), d.end(), [](char c) { return c >= '0' && c <= '9'; });
        if (!num) out.push_back(x);
    }
    return out;
}

// ------------------------------------------------------------ prefix rules

// parse_prefix (engine/tree.hpp:69-95) straight into compile_rmod's
// post-order encoding (engine/vocab.hpp:99-126): a terminal label -> (-1,
// slot), any other leaf -> (-2, llround(strtod(label) * 1000)), an operator
// with its two operands -> (opcode, left, right).
struct PrefixCompiler {
    std::vector<std::string> toks;
    size_t pos = 0;
    std::vector<int32_t> ops, args;
    std::string err;

    int32_t node(int depth) {
        if (depth > 64 || pos >= toks.size()) {
            err = "malformed prefix rule";
            return -1;
        }
        const std::string& tok = toks[pos];
        if (tok == "(") {
            pos++;
            if (pos >= toks.size()) {
                err = "malformed prefix rule";
                return -1;
            }
            const std::string sym = toks[pos++];
            int code = -1;
            for (int k = 0; k < 7; k++)
                if (sym == kFuncNames[k]) code = k;
            if (code < 0) {
                err = "unknown operator " + sym;
                return -1;
            }
            std::vector<int32_t> kids;
            while (pos < toks.size() && toks[pos] != ")") {
                kids.push_back(node(depth + 1));
                if (!err.empty()) return -1;
            }
            if (pos >= toks.size() || kids.size() != 2) {
                err = "operator " + sym + " needs two operands";
                return -1;
            }
            pos++;
            ops.push_back(code);
            args.push_back(kids[0]);
            args.push_back(kids[1]);
            return (int32_t)ops.size() - 1;
        }
        if (tok == ")") {
            err = "malformed prefix rule";
            return -1;
        }
        pos++;
        const int s = term_slot(tok);
        if (s >= 0) {
            ops.push_back(-1);
            args.push_back(s);
        } else {
            ops.push_back(-2);
            args.push_back((int32_t)std::llround(std::strtod(tok.c_str(), nullptr) * 1000.0));
        }
        args.push_back(0);
        return (int32_t)ops.size() - 1;
    }

    bool run(const std::string& s) {
        std::string t;
        for (char c : s) {
            if (c == '(') t += " ( ";
            else if (c == ')') t += " ) ";
            else t += c;
        }
        size_t i = 0;
        while (i < t.size()) {
            while (i < t.size() && std::isspace((unsigned char)t[i])) i++;
            size_t j = i;
            while (j < t.size() && !std::isspace((unsigned char)t[j])) j++;
            if (j > i) toks.push_back(t.substr(i, j - i));
            i = j;
        }
        node(0);
        if (err.empty() && pos != toks.size()) err = "trailing text after the rule";
        return err.empty();
    }
};

sidr_status compile_prefix(const std::string& text, Packed& pk) {
    PrefixCompiler pc;
    if (!pc.run(text)) return gp_fail(SIDR_ERR_RULE, pc.err + ": " + text.substr(0, 80));
    pk.off.push_back((int32_t)pk.ops.size());
    pk.len.push_back((int32_t)pc.ops.size());
    pk.ops.insert(pk.ops.end(), pc.ops.begin(), pc.ops.end());
    pk.args.insert(pk.args.end(), pc.args.begin(), pc.args.end());
    return SIDR_OK;
}

sidr_status vocab_of_trace(const JVal& tr, const std::vector<std::string>& base,
                           std::vector<std::string>& vocab) {
    const JVal* ex = tr.get("vocab_extra");
    if (!ex || ex->kind != JVal::ARR) return gp_fail(SIDR_ERR_INVALID, "trace has no vocab_extra list");
    vocab = base;
    for (const JVal& x : ex->arr) {
        if (x.kind != JVal::STR || (x.str != "ERC" && term_slot(x.str) < 0))
            return gp_fail(SIDR_ERR_INVALID, "unknown terminal in vocab_extra");
        vocab.push_back(x.str);
    }
    return SIDR_OK;
}

sidr_status copy_text(const std::string& s, char* buf, int64_t cap, int64_t* len) {
    if (len) *len = (int64_t)s.size() + 1;
    if (buf && cap > 0) {
        if (cap <= (int64_t)s.size()) return gp_fail(SIDR_ERR_TOO_LARGE, "output buffer too small");
        std::memcpy(buf, s.c_str(), s.size() + 1);
    }
    return SIDR_OK;
}

// ------------------------------------------------------ vocabulary search
//
// The search over terminal subsets of s4_selection/ga.cu:288-523 in three
// parts: a score store holding every evaluated genome's per-seed scores at the
// two budgets (proxy and confirmation) and mirroring them in the resumable
// cache file; a ranked hierarchy of 13 genomes; and the search, which breeds
// one offspring along every parent/supporter link of the hierarchy per
// generation.  Genomes are bit sets over the universe (bit b = universe[b]).
// The search's generator draws in the reference's order (pool padding, then
// per link: nb crossover draws and nb mutation draws), and its log lines and
// cache file have the reference's text, so runs are comparable line for line.

// Per-seed scores of genomes at the two evaluation budgets.
class ScoreStore {
public:
    enum Budget { kProxy = 0, kConfirm = 1 };

    explicit ScoreStore(std::string header) : header_(std::move(header)) {}
    ~ScoreStore() {
        if (file_) std::fclose(file_);
    }
    ScoreStore(const ScoreStore&) = delete;
    ScoreStore& operator=(const ScoreStore&) = delete;

    // Loads the entries of a cache file written under the same header (lines
    // cut short are dropped: those genomes are evaluated again), then keeps
    // the file open for appending; a file under another header is rewritten.
    // Returns the number of entries loaded.
    long attach(const char* path) {
        long loaded = 0;
        if (std::FILE* in = std::fopen(path, "r")) {
            std::string row;
            bool first = true, same_header = false;
            while (read_row(in, row)) {
                if (first) {
                    same_header = row == header_;
                    first = false;
                    if (!same_header) break;
                    continue;
                }
                loaded += parse_row(row) ? 1 : 0;
            }
            std::fclose(in);
        }
        file_ = std::fopen(path, loaded > 0 ? "a" : "w");
        if (file_ && loaded == 0) std::fprintf(file_, "%s\n", header_.c_str());
        return loaded;
    }

    bool has(Budget b, uint32_t g) const { return tab_[b].count(g) != 0; }
    const std::vector<double>& at(Budget b, uint32_t g) const { return tab_[b].at(g); }
    double mean(Budget b, uint32_t g) const { return mean_of(tab_[b].at(g)); }

    void put(Budget b, uint32_t g, std::vector<double> v) {
        if (file_) {
            std::fprintf(file_, "%c %x %d", b == kProxy ? 'P' : 'C', g, (int)v.size());
            for (double x : v) std::fprintf(file_, " %a", x);
            std::fputc('\n', file_);
        }
        tab_[b][g] = std::move(v);
    }
    void sync() {
        if (file_) std::fflush(file_);
    }

private:
    static bool read_row(std::FILE* in, std::string& row) {
        row.clear();
        int c;
        while ((c = std::fgetc(in)) != EOF && c != '\n') row += (char)c;
        return !(c == EOF && row.empty());
    }
    // "<P|C> <genome hex> <count> <hexfloat> ..."
    bool parse_row(const std::string& row) {
        const char* p = row.c_str();
        if ((p[0] != 'P' && p[0] != 'C') || p[1] != ' ') return false;
        const Budget b = p[0] == 'P' ? kProxy : kConfirm;
        char* end = nullptr;
        const unsigned long g = std::strtoul(p + 2, &end, 16);
        if (end == p + 2) return false;
        const char* q = end;
        const long count = std::strtol(q, &end, 10);
        if (end == q || count < 0) return false;
        std::vector<double> v;
        for (q = end; (long)v.size() < count; q = end) {
            const double x = std::strtod(q, &end);
            if (end == q) return false;
            v.push_back(x);
        }
        tab_[b][(uint32_t)g] = std::move(v);
        return true;
    }

    std::string header_;
    std::map<uint32_t, std::vector<double>> tab_[2];
    std::FILE* file_ = nullptr;
};

// Thirteen genomes as a ternary heap of depth two: parent slot i (i = 0..3)
// has the supporters 3i+1 .. 3i+3, so the root leads slots 1-3 and each of
// those leads three leaves.  settle() restores the heap's order by passes
// over the parents from the bottom (3, 2, 1, then the root): a parent swaps
// places with its best supporter when that one scores strictly higher (of
// equal bests, the first), and passes repeat until one moves nothing, at most
// 13 times.
struct RankedHierarchy {
    static constexpr int kSlots = 13;
    static constexpr int kParents = 4;
    std::array<uint32_t, kSlots> g{};

    static int supporter(int parent, int k) { return 3 * parent + 1 + k; }

    template <class Score>
    void settle(Score&& score) {
        for (int pass = 0; pass < kSlots; pass++) {
            bool moved = false;
            for (int parent = kParents - 1; parent >= 0; parent--) {
                int top = -1;
                for (int k = 0; k < 3; k++) {
                    const int s = supporter(parent, k);
                    if (score(g[s]) > score(g[parent]) && (top < 0 || score(g[s]) > score(g[top]))) top = s;
                }
                if (top >= 0) {
                    std::swap(g[parent], g[top]);
                    moved = true;
                }
            }
            if (!moved) return;
        }
    }
    size_t distinct() const { return std::set<uint32_t>(g.begin(), g.end()).size(); }
};

// Scores lists of genomes at n seeds x ng inner generations, in chunks of at
// most `bmax` genomes: through the caller's callback, or on the evaluator
// (batch_score, Scorer::chunk).  Each chunk's size and time go to the log.
struct ChunkedScoring {
    sidr_ctx* ctx;
    const sidr_instance_desc* inst;
    const sidr_gp_config* cfg;
    const Universe& uni;
    int bmax;
    sidr_vocab_fitness_fn callback;
    void* user;
    Log& log;
    long evaluated = 0;
    double seconds = 0.0;

    sidr_status operator()(const std::vector<uint32_t>& gs, int n, int ng,
                           std::vector<std::vector<double>>& res) {
        res.assign(gs.size(), std::vector<double>(n));
        for (size_t at = 0; at < gs.size(); at += bmax) {
            const int kb = (int)std::min<size_t>(bmax, gs.size() - at);
            std::vector<double> flat((size_t)kb * n);
            const double t0 = now_s();
            if (callback) {
                if (callback(user, gs.data() + at, kb, n, ng, flat.data()) != 0)
                    return gp_fail(SIDR_ERR_INVALID, "fitness callback failed");
            } else {
                Scorer sc{ctx, inst, *cfg, uni, SIDR_TRAIN_SEED, SIDR_TRAIN_N};
                const sidr_status s = sc.chunk(gs.data() + at, kb, n, ng, flat.data());
                if (s != SIDR_OK) return s;
            }
            const double dt = now_s() - t0;
            for (int k = 0; k < kb; k++)
                std::copy(flat.begin() + (size_t)k * n, flat.begin() + (size_t)(k + 1) * n, res[at + k].begin());
            evaluated += kb;
            seconds += dt;
            log("  batch %d genomes @%d seeds | %.1fs | %.2fs/eval\n", kb, n, dt, dt / kb);
        }
        return SIDR_OK;
    }
};

class VocabSearch {
public:
    VocabSearch(const sidr_vocab_ga_config& s, int cgens, const Universe& u, ScoreStore& store,
                ChunkedScoring& scoring, Log& log)
        : set_(s), cgens_(cgens), uni_(u), store_(store), scoring_(scoring), log_(log),
          rng_((uint64_t)s.ga_seed) {}

    struct Outcome {
        uint32_t champion = 0;
        double confirmed_mean = 0.0;
    };

    sidr_status run(const std::string& instance, Outcome& res) {
        sidr_status st = seed_hierarchy(instance);
        if (st != SIDR_OK) return st;
        double record = proxy(h_.g[0]);
        int flat_gens = 0;
        for (int gen = 0; gen < set_.gens; gen++) {
            report(("gen " + std::to_string(gen)).c_str(), true);
            if ((st = breed_generation()) != SIDR_OK) return st;
            if (proxy(h_.g[0]) > record) {
                record = proxy(h_.g[0]);
                flat_gens = 0;
            } else if (++flat_gens >= set_.stag) {
                log_("stop: stagnant %d gens\n", flat_gens);
                break;
            }
        }
        report("gen end", false);
        return confirm_finalists(res);
    }

private:
    double proxy(uint32_t g) const { return store_.mean(ScoreStore::kProxy, g); }
    // ranking of the pool and the finalists: higher proxy mean, then fewer terminals
    bool ranks_above(uint32_t a, uint32_t b) const {
        const double fa = proxy(a), fb = proxy(b);
        return fa != fb ? fa > fb : __builtin_popcount(a) < __builtin_popcount(b);
    }

    // Each universe bit on with probability 0.35.
    uint32_t draw_genome() {
        uint32_t g = 0;
        for (int b = 0; b < uni_.nb; b++)
            if (rng_.random() < 0.35) g |= 1u << b;
        return g;
    }
    // Uniform crossover (bit b from x when the draw is < 0.5), then every bit
    // flipped with probability pm / nb.
    uint32_t offspring(uint32_t x, uint32_t y) {
        uint32_t c = 0;
        for (int b = 0; b < uni_.nb; b++) c |= (rng_.random() < 0.5 ? x : y) & (1u << b);
        for (int b = 0; b < uni_.nb; b++)
            if (rng_.random() < set_.pm / uni_.nb) c ^= 1u << b;
        return c;
    }

    // Proxy scores for every genome of `gs` not scored yet (distinct, in
    // ascending order).
    sidr_status score_proxy(std::vector<uint32_t> gs) {
        std::sort(gs.begin(), gs.end());
        gs.erase(std::unique(gs.begin(), gs.end()), gs.end());
        gs.erase(std::remove_if(gs.begin(), gs.end(), [&](uint32_t g) { return store_.has(ScoreStore::kProxy, g); }),
                 gs.end());
        if (gs.empty()) return SIDR_OK;
        std::vector<std::vector<double>> res;
        const sidr_status st = scoring_(gs, set_.proxy, set_.pgens, res);
        if (st != SIDR_OK) return st;
        for (size_t i = 0; i < gs.size(); i++) store_.put(ScoreStore::kProxy, gs[i], std::move(res[i]));
        store_.sync();
        return SIDR_OK;
    }

    // The starting pool: the neutral seeds when asked for (the empty set, the
    // whole universe unless left out, every singleton), padded with random
    // genomes to 13; scored, ranked, the best 13 placed in the hierarchy.
    sidr_status seed_hierarchy(const std::string& instance) {
        std::vector<uint32_t> pool;
        if (set_.seeds_neutral) {
            pool.push_back(0);
            if (!set_.nofull) pool.push_back(uni_.nb >= 32 ? 0xffffffffu : (1u << uni_.nb) - 1u);
            for (int b = 0; b < uni_.nb; b++) pool.push_back(1u << b);
        }
        std::sort(pool.begin(), pool.end());
        pool.erase(std::unique(pool.begin(), pool.end()), pool.end());
        const size_t n_seeded = pool.size();
        while (pool.size() < (size_t)RankedHierarchy::kSlots) pool.push_back(draw_genome());
        log_("# ga %s | universe %d | seeds %s (%zu)%s | tree-13 uniform-x pm %.2f | gens %d stag %d\n",
             instance.c_str(), uni_.nb, set_.seeds_neutral ? "neutral" : "random", n_seeded,
             set_.nofull ? " nofull" : "", set_.pm, set_.gens, set_.stag);
        const sidr_status st = score_proxy(pool);
        if (st != SIDR_OK) return st;
        std::stable_sort(pool.begin(), pool.end(), [&](uint32_t a, uint32_t b) { return ranks_above(a, b); });
        std::copy(pool.begin(), pool.begin() + RankedHierarchy::kSlots, h_.g.begin());
        settle();
        return SIDR_OK;
    }

    void settle() {
        h_.settle([&](uint32_t g) { return proxy(g); });
    }

    void report(const char* label, bool with_distinct) {
        double avg = 0.0;
        for (uint32_t g : h_.g) avg += proxy(g);
        avg /= RankedHierarchy::kSlots;
        if (with_distinct)
            log_("%s | best %.2f [%s] | mean %.2f | unique %zu | evals %ld\n", label, proxy(h_.g[0]),
                 uni_.name_of(h_.g[0]).c_str(), avg, h_.distinct(), scoring_.evaluated);
        else
            log_("%s | best %.2f [%s] | mean %.2f | evals %ld\n", label, proxy(h_.g[0]),
                 uni_.name_of(h_.g[0]).c_str(), avg, scoring_.evaluated);
    }

    // One generation: fresh genomes in the two last leaves when at most six
    // of the 13 are distinct; one offspring per parent/supporter link (links
    // in slot order), which takes the place of the link's weaker end (the
    // supporter when they tie) if it scores strictly higher; then settle.
    sidr_status breed_generation() {
        sidr_status st;
        if (h_.distinct() <= 6) {
            const uint32_t a = draw_genome(), b = draw_genome();
            h_.g[RankedHierarchy::kSlots - 1] = a;
            h_.g[RankedHierarchy::kSlots - 2] = b;
            if ((st = score_proxy({a, b})) != SIDR_OK) return st;
            log_("  reinject 2\n");
        }
        struct Link {
            int parent, sup;
            uint32_t child;
        };
        std::vector<Link> links;
        for (int parent = 0; parent < RankedHierarchy::kParents; parent++)
            for (int k = 0; k < 3; k++) {
                const int s = RankedHierarchy::supporter(parent, k);
                links.push_back({parent, s, offspring(h_.g[parent], h_.g[s])});
            }
        std::vector<uint32_t> kids;
        for (const Link& l : links) kids.push_back(l.child);
        if ((st = score_proxy(kids)) != SIDR_OK) return st;
        for (const Link& l : links) {
            const int weaker = proxy(h_.g[l.sup]) <= proxy(h_.g[l.parent]) ? l.sup : l.parent;
            if (proxy(l.child) > proxy(h_.g[weaker])) h_.g[weaker] = l.child;
        }
        settle();
        return SIDR_OK;
    }

    // The hierarchy's distinct genomes, best-ranked first (ascending genome
    // order among equals), the first `top` confirmed at `confirm` seeds with
    // cgens inner generations; the champion has the highest confirmed mean
    // (ties: fewer terminals, then rank).
    sidr_status confirm_finalists(Outcome& res) {
        const std::set<uint32_t> distinct(h_.g.begin(), h_.g.end());
        std::vector<uint32_t> fin(distinct.begin(), distinct.end());
        std::stable_sort(fin.begin(), fin.end(), [&](uint32_t a, uint32_t b) { return ranks_above(a, b); });
        if ((int)fin.size() > set_.top) fin.resize(set_.top);
        log_("\nconfirming top-%zu at %d seeds:\n", fin.size(), set_.confirm);
        std::vector<uint32_t> todo;
        for (uint32_t g : fin)
            if (!store_.has(ScoreStore::kConfirm, g)) todo.push_back(g);
        if (!todo.empty()) {
            std::vector<std::vector<double>> scores;
            const sidr_status st = scoring_(todo, set_.confirm, cgens_, scores);
            if (st != SIDR_OK) return st;
            for (size_t i = 0; i < todo.size(); i++) store_.put(ScoreStore::kConfirm, todo[i], std::move(scores[i]));
            store_.sync();
        }
        size_t win = 0;
        for (size_t i = 1; i < fin.size(); i++) {
            const double m = store_.mean(ScoreStore::kConfirm, fin[i]);
            const double mw = store_.mean(ScoreStore::kConfirm, fin[win]);
            if (m > mw || (m == mw && __builtin_popcount(fin[i]) < __builtin_popcount(fin[win]))) win = i;
        }
        for (uint32_t g : fin)
            log_("  %.2f (proxy %.2f) [%s]\n", store_.mean(ScoreStore::kConfirm, g), proxy(g),
                 uni_.name_of(g).c_str());
        res.champion = fin[win];
        res.confirmed_mean = store_.mean(ScoreStore::kConfirm, fin[win]);
        return SIDR_OK;
    }

    const sidr_vocab_ga_config& set_;
    const int cgens_;
    const Universe& uni_;
    ScoreStore& store_;
    ChunkedScoring& scoring_;
    Log& log_;
    Mt19937 rng_;
    RankedHierarchy h_;
};

}  // namespace

extern "C" {

sidr_status sidr_vocab_batch_score(sidr_ctx* ctx, const sidr_instance_desc* inst,
                                   const sidr_gp_config* cfg, const char* base_csv,
                                   const char* universe_csv, const uint32_t* genomes, int32_t K,
                                   int32_t n_seeds, int32_t n_gens, int32_t bmax,
                                   int64_t block_seed, int32_t block_n, double* out,
                                   sidr_gp_result* result) {
    sidr_status st = check_common(ctx, inst, cfg, n_seeds, n_gens, block_n);
    if (st != SIDR_OK) return st;
    if (K < 0 || (K > 0 && (!genomes || !out)) || bmax < 1)
        return gp_fail(SIDR_ERR_INVALID, "genomes/out missing or bmax < 1");
    Universe u;
    if ((st = load_universe(base_csv, universe_csv, u)) != SIDR_OK) return st;
    const double t0 = now_s();
    Scorer sc{ctx, inst, *cfg, u, block_seed, block_n};
    for (int k0 = 0; k0 < K; k0 += bmax) {
        const int kb = std::min(bmax, K - k0);
        if ((st = sc.chunk(genomes + k0, kb, n_seeds, n_gens, out + (size_t)k0 * n_seeds)) != SIDR_OK)
            return st;
    }
    if (result) {
        result->eval_seconds = sc.t_eval;
        result->host_seconds = now_s() - t0 - sc.t_eval;
        result->evaluations = sc.n_evals;
    }
    return SIDR_OK;
}

sidr_status sidr_vocab_seq_score(sidr_ctx* ctx, const sidr_instance_desc* inst,
                                 const sidr_gp_config* cfg, const char* base_csv,
                                 const char* universe_csv, uint32_t genome, int32_t n_seeds,
                                 int32_t n_gens, int64_t block_seed, int32_t block_n, double* out) {
    sidr_status st = check_common(ctx, inst, cfg, n_seeds, n_gens, block_n);
    if (st != SIDR_OK) return st;
    if (!out) return gp_fail(SIDR_ERR_INVALID, "out is null");
    Universe u;
    if ((st = load_universe(base_csv, universe_csv, u)) != SIDR_OK) return st;
    Scorer sc{ctx, inst, *cfg, u, block_seed, block_n};
    return sc.sequential(genome, n_seeds, n_gens, out);
}

sidr_status sidr_vocab_gate(sidr_ctx* ctx, const sidr_instance_desc* inst,
                            const sidr_gp_config* cfg, const char* base_csv,
                            const char* universe_csv, int32_t n_seeds, int32_t n_gens,
                            int32_t bmax, int64_t block_seed, int32_t block_n, int64_t* compared,
                            int64_t* mismatches, double* max_diff) {
    sidr_status st = check_common(ctx, inst, cfg, n_seeds, n_gens, block_n);
    if (st != SIDR_OK) return st;
    Universe u;
    if ((st = load_universe(base_csv, universe_csv, u)) != SIDR_OK) return st;
    const int nb = u.nb;
    const uint32_t full = nb >= 32 ? 0xffffffffu : ((1u << nb) - 1u);
    const std::vector<uint32_t> gset = {0u, full, 1u << 0, 1u << (nb > 7 ? 7 : nb - 1),
                                        (1u << 1) | (1u << (nb > 4 ? 4 : 0)) | (1u << (nb > 9 ? 9 : 0))};
    std::vector<double> bat(gset.size() * n_seeds), ref(n_seeds);
    if ((st = sidr_vocab_batch_score(ctx, inst, cfg, base_csv, universe_csv, gset.data(),
                                     (int32_t)gset.size(), n_seeds, n_gens, bmax, block_seed, block_n,
                                     bat.data(), nullptr)) != SIDR_OK)
        return st;
    int64_t cmp = 0, bad = 0;
    double mx = 0.0;
    for (size_t i = 0; i < gset.size(); i++) {
        if ((st = sidr_vocab_seq_score(ctx, inst, cfg, base_csv, universe_csv, gset[i], n_seeds, n_gens,
                                       block_seed, block_n, ref.data())) != SIDR_OK)
            return st;
        for (int s = 0; s < n_seeds; s++) {
            const double a = bat[i * n_seeds + s];
            mx = std::max(mx, std::fabs(a - ref[s]));
            cmp++;
            if (a != ref[s]) bad++;
        }
    }
    if (compared) *compared = cmp;
    if (mismatches) *mismatches = bad;
    if (max_diff) *max_diff = mx;
    return SIDR_OK;
}

void sidr_vocab_ga_default_config(sidr_vocab_ga_config* c) {
    if (!c) return;
    c->pgens = 51;
    c->proxy = 16;
    c->confirm = 30;
    c->gens = 50;
    c->stag = 5;
    c->bmax = 10;
    c->top = 4;
    c->pm = 0.5;
    c->seeds_neutral = 0;
    c->nofull = 0;
    c->ga_seed = 20260714;
}

sidr_status sidr_vocab_ga(sidr_ctx* ctx, const sidr_instance_desc* inst,
                          const sidr_gp_config* cfg, const sidr_vocab_ga_config* ga,
                          const char* instance_name, const char* base_csv,
                          const char* universe_csv, const char* cache_path,
                          sidr_vocab_fitness_fn fitness, void* user, uint32_t* champion,
                          double* champion_mean, int64_t* evals_out, char* log, int64_t log_cap,
                          int64_t* log_len) {
    std::string err;
    if (!ga || !instance_name) return gp_fail(SIDR_ERR_INVALID, "null argument");
    if (!valid_config(cfg, err)) return gp_fail(SIDR_ERR_INVALID, err);
    if (!fitness && (!ctx || !inst)) return gp_fail(SIDR_ERR_INVALID, "no fitness source");
    if (ga->pgens < 1 || ga->proxy < 1 || ga->confirm < 1 || ga->gens < 0 || ga->stag < 1 ||
        ga->bmax < 1 || ga->top < 1)
        return gp_fail(SIDR_ERR_INVALID, "GA settings out of range");
    Universe u;
    sidr_status st = load_universe(base_csv, universe_csv, u);
    if (st != SIDR_OK) return st;
    Log text;

    // the cache file's header names everything its scores depend on (s4_selection/ga.cu:315-377)
    std::string names;
    for (int b = 0; b < u.nb; b++) names += (b ? "," : "") + u.uni[b];
    char header[512];
    std::snprintf(header, sizeof header, "# gacache v1 %s uni=%s proxy=%d pgens=%d confirm=%d cgens=%d",
                  instance_name, names.c_str(), ga->proxy, ga->pgens, ga->confirm, cfg->generations);
    ScoreStore store(header);
    if (cache_path && *cache_path) {
        const long loaded = store.attach(cache_path);
        if (loaded > 0) text("# cache %s | %ld entries loaded\n", cache_path, loaded);
    }
    ChunkedScoring scoring{ctx, inst, cfg, u, ga->bmax, fitness, user, text};
    VocabSearch search(*ga, cfg->generations, u, store, scoring, text);
    const double t0 = now_s();
    VocabSearch::Outcome res;
    if ((st = search.run(instance_name, res)) != SIDR_OK) return st;
    const double wall = now_s() - t0;
    text("\nCHAMPION train-%d %.2f | evals %ld | terms: %s\n", ga->confirm, res.confirmed_mean,
         scoring.evaluated, u.name_of(res.champion).c_str());
    text("PERF evals %ld | wall %.0fs | %.1fs/eval | batch-gpu %.0fs\n", scoring.evaluated, wall,
         wall / std::max(1L, scoring.evaluated), scoring.seconds);
    if (champion) *champion = res.champion;
    if (champion_mean) *champion_mean = res.confirmed_mean;
    if (evals_out) *evals_out = scoring.evaluated;
    return copy_text(text.text, log, log_cap, log_len);
}

sidr_status sidr_gen_trace(sidr_ctx* ctx, const sidr_instance_desc* inst,
                           const sidr_gp_config* cfg, const char* instance_name,
                           const char* base_csv, const char* extra_csv, int32_t n_seeds,
                           double km, int64_t test_seed, int32_t n_test, char* json,
                           int64_t json_cap, int64_t* json_len, double* mean_gain) {
    sidr_status st = check_common(ctx, inst, cfg, n_seeds, cfg ? cfg->generations : 1, n_test);
    if (st != SIDR_OK) return st;
    if (!instance_name) return gp_fail(SIDR_ERR_INVALID, "instance name is null");
    std::string err;
    std::vector<std::string> base, extra;
    if (!parse_terminals(base_csv, base, err)) return gp_fail(SIDR_ERR_INVALID, "base set: " + err);
    if (extra_csv && *extra_csv && !parse_terminals(extra_csv, extra, err))
        return gp_fail(SIDR_ERR_INVALID, "extra terminals: " + err);
    std::vector<std::string> vocab = base;
    vocab.insert(vocab.end(), extra.begin(), extra.end());
    const std::vector<int64_t> tmask = mask_of(vocab);
    const std::set<std::string> base_set(base.begin(), base.end());
    const int ps = cfg->population, T = cfg->train_samples, nn = inst->n, G = cfg->generations;

    std::vector<std::unique_ptr<Gp>> pops;
    for (int s = 0; s < n_seeds; s++) pops.push_back(new_population(*cfg, (uint64_t)s, vocab));
    parallel_for(n_seeds, [&](int i) { pops[i]->init(); });
    std::vector<std::vector<std::string>> trace(n_seeds);
    std::vector<std::vector<double>> f;
    auto gfit = [&](int gen_id) -> sidr_status {
        Packed pk;
        pack_all(pops, pk);
        std::vector<double> grouped((size_t)n_seeds * T * nn);
        for (int s = 0; s < n_seeds; s++) {
            const std::vector<double> one = durations_block(inst, T, (long long)s * 10000 + gen_id);
            std::copy(one.begin(), one.end(), grouped.begin() + (size_t)s * T * nn);
        }
        sidr_rules_desc r = pk.desc();
        std::vector<double> out((size_t)r.P * T);
        const sidr_status s2 =
            sidr_evaluate_grouped(ctx, &r, grouped.data(), n_seeds, T, ps, tmask.data(), out.data());
        if (s2 != SIDR_OK) return gp_fail(s2, std::string("evaluation: ") + sidr_last_error());
        population_means(out, n_seeds, ps, T, f);
        return SIDR_OK;
    };
    for (int gen = 0; gen < G; gen++) {
        if ((st = gfit(gen)) != SIDR_OK) return st;
        for (int s = 0; s < n_seeds; s++) {
            const size_t b = best_index(f[s]);
            const Rule& rule = pops[s]->pop[b];
            trace[s].push_back("{" + jstr("g") + ": " + std::to_string(gen) + ", " + jstr("fit") + ": " +
                               jnum(round_half_even(f[s][b], 1)) + ", " + jstr("sz") + ": " +
                               std::to_string(rule.size()) + ", " + jstr("ex") + ": " +
                               jstrlist(extras_of(rule, pops[s]->vocab, base_set)) + "}");
        }
        if (gen < G - 1) parallel_for(n_seeds, [&](int i) { pops[i]->step(f[i]); });
    }
    if ((st = gfit(G)) != SIDR_OK) return st;
    // every seed's final on the held-out block in one call (the pairs are
    // independent, so this equals the reference's one call per seed)
    Packed fin;
    std::vector<size_t> bsel(n_seeds);
    for (int s = 0; s < n_seeds; s++) {
        bsel[s] = best_index(f[s]);
        pack_rule(*pops[s], bsel[s], fin);
    }
    const std::vector<double> test = durations_block(inst, n_test, test_seed);
    sidr_rules_desc r = fin.desc();
    std::vector<double> ts((size_t)n_seeds * n_test);
    if ((st = sidr_evaluate(ctx, &r, test.data(), n_test, tmask.data(), ts.data())) != SIDR_OK)
        return gp_fail(st, std::string("held-out evaluation: ") + sidr_last_error());
    std::vector<double> gains;
    std::vector<std::string> finals;
    for (int s = 0; s < n_seeds; s++) {
        double got = 0.0;
        for (int t = 0; t < n_test; t++) got += ts[(size_t)s * n_test + t];
        got /= n_test;
        const double g = 100.0 * (got - km) / km;
        gains.push_back(g);
        const Rule& rule = pops[s]->pop[bsel[s]];
        std::string pre;
        size_t k = 0;
        prefix_at(rule, k, pops[s]->vocab, pre);
        finals.push_back("{" + jstr("seed") + ": " + std::to_string(s) + ", " + jstr("gain") + ": " +
                         jnum(round_half_even(g, 2)) + ", " + jstr("sz") + ": " + std::to_string(rule.size()) +
                         ", " + jstr("ex") + ": " + jstrlist(extras_of(rule, pops[s]->vocab, base_set)) + ", " +
                         jstr("rule") + ": " + jstr(pre) + "}");
    }
    double mean_g = 0.0, best_g = gains[0];
    int pos = 0;
    for (double g : gains) {
        mean_g += g;
        if (g > 0) pos++;
        if (g > best_g) best_g = g;
    }
    mean_g /= gains.size();
    double var = 0.0;
    for (double g : gains) var += (g - mean_g) * (g - mean_g);
    const double std_g = gains.size() > 1 ? std::sqrt(var / (gains.size() - 1)) : 0.0;
    std::vector<std::string> tr_parts;
    for (auto& tl : trace) tr_parts.push_back(jlist(tl));
    const std::string o =
        "{" + jstr("instance") + ": " + jstr(instance_name) + ", " + jstr("vocab_extra") + ": " +
        jstrlist(extra) + ", " + jstr("mean_gain") + ": " + jnum(round_half_even(mean_g, 2)) + ", " +
        jstr("std") + ": " + jnum(round_half_even(std_g, 2)) + ", " + jstr("seeds_positive") + ": " +
        jstr(std::to_string(pos) + "/" + std::to_string(gains.size())) + ", " + jstr("best_seed_gain") +
        ": " + jnum(round_half_even(best_g, 2)) + ", " + jstr("finals") + ": " + jlist(finals) + ", " +
        jstr("trace") + ": " + jlist(tr_parts) + "}";
    if (mean_gain) *mean_gain = mean_g;
    return copy_text(o, json, json_cap, json_len);
}

sidr_status sidr_redeploy(sidr_ctx* ctx, const sidr_instance_desc* inst, const char* instance_name,
                          const char* trace_json, const char* base_csv, double km,
                          int64_t test_seed, int32_t n_test, double* trace_gain, double* gain,
                          double* delta, int32_t* sealed) {
    if (!ctx || !inst || !instance_name || n_test < 1) return gp_fail(SIDR_ERR_INVALID, "bad argument");
    JVal tr;
    sidr_status st = parse_json(trace_json, tr);
    if (st != SIDR_OK) return st;
    const JVal* in = tr.get("instance");
    if (!in || in->kind != JVal::STR || in->str != instance_name)
        return gp_fail(SIDR_ERR_INVALID, "trace instance mismatch");
    const JVal* finals = tr.get("finals");
    if (!finals || finals->kind != JVal::ARR || finals->arr.empty())
        return gp_fail(SIDR_ERR_INVALID, "trace has no finals");
    const JVal* best = nullptr;
    for (const JVal& f : finals->arr) {
        const JVal* g = f.get("gain");
        const JVal* r = f.get("rule");
        if (!g || g->kind != JVal::NUM || !r || r->kind != JVal::STR)
            return gp_fail(SIDR_ERR_INVALID, "a final lacks gain or rule");
        if (!best || g->num > best->get("gain")->num) best = &f;
    }
    std::string err;
    std::vector<std::string> base, vocab;
    if (!parse_terminals(base_csv, base, err)) return gp_fail(SIDR_ERR_INVALID, "base set: " + err);
    if ((st = vocab_of_trace(tr, base, vocab)) != SIDR_OK) return st;
    const std::vector<int64_t> tmask = mask_of(vocab);
    Packed pk;
    if ((st = compile_prefix(best->get("rule")->str, pk)) != SIDR_OK) return st;
    const std::vector<double> test = durations_block(inst, n_test, test_seed);
    sidr_rules_desc r = pk.desc();
    std::vector<double> ts(n_test);
    if ((st = sidr_evaluate(ctx, &r, test.data(), n_test, tmask.data(), ts.data())) != SIDR_OK)
        return gp_fail(st, std::string("held-out evaluation: ") + sidr_last_error());
    double got = 0.0;
    for (int s = 0; s < n_test; s++) got += ts[s];
    got /= n_test;
    const double g = 100.0 * (got - km) / km;
    const double tg = best->get("gain")->num;
    const double d = std::fabs(g - tg);
    if (trace_gain) *trace_gain = tg;
    if (gain) *gain = g;
    if (delta) *delta = d;
    if (sealed) *sealed = d <= 0.005 ? 1 : 0;
    return SIDR_OK;
}

sidr_status sidr_trace_mean_train(sidr_ctx* ctx, const sidr_instance_desc* inst,
                                  const char* trace_json, const char* base_csv,
                                  int64_t train_seed, int32_t n_train, double* mean_train,
                                  double* heldout) {
    if (!ctx || !inst || n_train < 1) return gp_fail(SIDR_ERR_INVALID, "bad argument");
    JVal tr;
    sidr_status st = parse_json(trace_json, tr);
    if (st != SIDR_OK) return st;
    const JVal* finals = tr.get("finals");
    const JVal* mg = tr.get("mean_gain");
    if (!finals || finals->kind != JVal::ARR || finals->arr.empty() || !mg || mg->kind != JVal::NUM)
        return gp_fail(SIDR_ERR_INVALID, "trace lacks finals or mean_gain");
    std::vector<std::pair<long long, std::string>> by_seed;
    for (const JVal& f : finals->arr) {
        const JVal* s = f.get("seed");
        const JVal* r = f.get("rule");
        if (!s || s->kind != JVal::NUM || !r || r->kind != JVal::STR)
            return gp_fail(SIDR_ERR_INVALID, "a final lacks seed or rule");
        by_seed.push_back({(long long)s->num, r->str});
    }
    std::stable_sort(by_seed.begin(), by_seed.end(),
                     [](const auto& a, const auto& b) { return a.first < b.first; });
    std::string err;
    std::vector<std::string> base, vocab;
    if (!parse_terminals(base_csv, base, err)) return gp_fail(SIDR_ERR_INVALID, "base set: " + err);
    if ((st = vocab_of_trace(tr, base, vocab)) != SIDR_OK) return st;
    const std::vector<int64_t> tmask = mask_of(vocab);
    Packed pk;
    for (const auto& bs : by_seed)
        if ((st = compile_prefix(bs.second, pk)) != SIDR_OK) return st;
    const std::vector<double> train = durations_block(inst, n_train, train_seed);
    sidr_rules_desc r = pk.desc();
    std::vector<double> fits((size_t)r.P * n_train);
    if ((st = sidr_evaluate(ctx, &r, train.data(), n_train, tmask.data(), fits.data())) != SIDR_OK)
        return gp_fail(st, std::string("train evaluation: ") + sidr_last_error());
    double acc = 0.0;
    for (int p = 0; p < r.P; p++) {
        double m = 0.0;
        for (int s = 0; s < n_train; s++) m += fits[(size_t)p * n_train + s];
        acc += m / n_train;
    }
    if (mean_train) *mean_train = acc / r.P;
    if (heldout) *heldout = mg->num;
    return SIDR_OK;
}

sidr_status sidr_rule_compile_prefix(const char* prefix, int32_t* ops, int32_t* args, int32_t* len) {
    if (!prefix || !len) return gp_fail(SIDR_ERR_INVALID, "null argument");
    Packed pk;
    const sidr_status st = compile_prefix(prefix, pk);
    if (st != SIDR_OK) return st;
    *len = (int32_t)pk.ops.size();
    if (ops && args) {
        std::memcpy(ops, pk.ops.data(), pk.ops.size() * 4);
        std::memcpy(args, pk.args.data(), pk.args.size() * 4);
    }
    return SIDR_OK;
}

}  // extern "C"
