// ref_shim.cpp -- extern "C" entry points over the reference's own engine
// headers (augustompm/solver-informed-dispatching-rules, engine/*.hpp),
// compiled in place from the reference tree into oracle/_ref/libsidr_ref.so by
// oracle/Makefile.  TEST INFRASTRUCTURE ONLY: the tests use it to pin the C
// oracle and the workload generators, and bench.py's reference arm times its
// sim_batch on the host cores.  No reference source is copied into this repo.
#include <cstdint>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "gp.hpp"
#include "sim_host.hpp"
#include "tree.hpp"
#include "vocab.hpp"

namespace {

SimData make_sd(int n, int m, double tmax, const double* scores, const double* durations,
                const double* open_t, const double* close_t, const double* dist,
                const double* d2d) {
    SimData sd;
    sd.n = n;
    sd.m = m;
    sd.ld = n + 1;
    sd.tmax = tmax;
    sd.scores.assign(scores, scores + n);
    sd.durations.assign(durations, durations + n);
    sd.open_t.assign(open_t, open_t + n);
    sd.close_t.assign(close_t, close_t + n);
    sd.dist.assign(dist, dist + (size_t)(n + 1) * (n + 1));
    sd.dist_to_depot.assign(d2d, d2d + n);
    return sd;
}

std::vector<std::string> split_csv(const char* s) {
    std::vector<std::string> out;
    std::string cur;
    for (const char* p = s; *p; ++p) {
        if (*p == ',') {
            if (!cur.empty()) out.push_back(cur);
            cur.clear();
        } else {
            cur += *p;
        }
    }
    if (!cur.empty()) out.push_back(cur);
    return out;
}

}  // namespace

extern "C" {

// load_instance-equivalent: parse a Solomon (cordeau=0) or Cordeau (1) file
// with the reference parser; fills up to cap POIs (id order) and returns the
// POI count (depot included), or -1.
int ref_parse_instance(const char* path, int cordeau, int cap, double* x, double* y,
                       double* score, double* open_t, double* close_t, double* duration,
                       double* tmax) {
    try {
        Instance inst = cordeau ? parse_cordeau(path) : parse_solomon(path);
        int np = (int)inst.pois.size();
        for (int i = 0; i < np && i < cap; i++) {
            const POI& p = inst.pois[i];
            x[i] = p.x;
            y[i] = p.y;
            score[i] = p.score;
            open_t[i] = p.open_time;
            close_t[i] = p.close_time;
            duration[i] = p.duration;
        }
        *tmax = inst.tmax;
        return np;
    } catch (...) {
        return -1;
    }
}

// SimData(inst, m).dist from POI coordinates (engine/sim_host.hpp:18-39).
void ref_build_dist(int n, const double* x, const double* y, double* dist, double* d2d) {
    Instance inst;
    for (int i = 0; i <= n; i++) {
        POI p{};
        p.id = i;
        p.x = x[i];
        p.y = y[i];
        inst.pois.push_back(p);
    }
    inst.tmax = 0.0;
    SimData sd(inst, 3, 0.2);
    std::memcpy(dist, sd.dist.data(), sd.dist.size() * sizeof(double));
    std::memcpy(d2d, sd.dist_to_depot.data(), sd.dist_to_depot.size() * sizeof(double));
}

void ref_zp_of(int n, double tmax, const double* scores, const double* durations,
               const double* open_t, const double* close_t, const double* dist, const double* d2d,
               double* zp) {
    SimData sd = make_sd(n, 3, tmax, scores, durations, open_t, close_t, dist, d2d);
    std::vector<double> z = zp_of(sd);
    std::memcpy(zp, z.data(), 10 * sizeof(double));
}

void ref_gen_durations(int n, const double* durations, double sigma, int S, long long base_seed,
                       double* out) {
    SimData sd;
    sd.n = n;
    sd.sigma = sigma;
    sd.durations.assign(durations, durations + n);
    std::vector<double> v = gen_durations(sd, S, base_seed);
    std::memcpy(out, v.data(), v.size() * sizeof(double));
}

// compile_rmod(parse_prefix(prefix)); returns the node count or -1 when it
// does not fit cap.
int ref_compile(const char* prefix, int cap, int32_t* ops, int32_t* args) {
    try {
        Compiled c = compile_rmod(parse_prefix(prefix));
        int L = (int)c.ops.size();
        if (L > cap) return -1;
        for (int k = 0; k < L; k++) {
            ops[k] = c.ops[k];
            args[2 * k] = c.args[k][0];
            args[2 * k + 1] = c.args[k][1];
        }
        return L;
    } catch (...) {
        return -1;
    }
}

// ramped_half_and_half(tc, Mt19937(seed), pop) (engine/gp.hpp:67-77); the
// prefix strings are written '\n'-separated into buf; returns bytes used or -1.
long ref_rhh(const char* terminals_csv, int with_rmod, int min_depth, int max_depth,
             unsigned long long seed, int pop, char* buf, long cap) {
    TreeConfig tc;
    tc.terminals = split_csv(terminals_csv);
    tc.functions = with_rmod ? FUNCS_RMOD : FUNCTIONS;
    tc.min_depth = min_depth;
    tc.max_depth = max_depth;
    Mt19937 rng((uint64_t)seed);
    std::vector<NodeP> popv = ramped_half_and_half(tc, rng, pop);
    std::string all;
    for (auto& t : popv) {
        all += to_prefix(t);
        all += '\n';
    }
    if ((long)all.size() + 1 > cap) return -1;
    std::memcpy(buf, all.c_str(), all.size() + 1);
    return (long)all.size();
}

// The reference's CPU evaluator over a grouped, multi-mask batch: sim_batch
// (engine/sim_host.hpp:67-83) per rule, rules split over nthreads std::threads.
// out[p*T + s].
void ref_eval_pairs(int n, int m, double tmax, const double* scores, const double* durations,
                    const double* open_t, const double* close_t, const double* dist,
                    const double* d2d, const double* zp_in, const int32_t* ops,
                    const int32_t* args, const int32_t* offsets, const int32_t* lengths, int P,
                    const double* grouped_sampled, int T, int group_size, const int64_t* masks,
                    int mask_group, double* out, int nthreads) {
    SimData sd = make_sd(n, m, tmax, scores, durations, open_t, close_t, dist, d2d);
    std::vector<double> zp(zp_in, zp_in + 10);
    if (nthreads < 1) nthreads = 1;
    if (nthreads > P) nthreads = P > 0 ? P : 1;
    auto work = [&](int p0, int p1) {
        for (int p = p0; p < p1; p++) {
            Compiled c;
            for (int k = 0; k < lengths[p]; k++) {
                c.ops.push_back(ops[offsets[p] + k]);
                c.args.push_back({args[2 * (offsets[p] + k)], args[2 * (offsets[p] + k) + 1]});
            }
            std::vector<int64_t> mask(masks + (size_t)(p / mask_group) * N_TERMS,
                                      masks + (size_t)(p / mask_group + 1) * N_TERMS);
            int g = p / group_size;
            std::vector<double> smp(grouped_sampled + (size_t)g * T * n,
                                    grouped_sampled + (size_t)(g + 1) * T * n);
            std::vector<double> r = sim_batch(sd, c, smp, T, mask, zp);
            std::memcpy(out + (size_t)p * T, r.data(), (size_t)T * sizeof(double));
        }
    };
    std::vector<std::thread> th;
    for (int t = 1; t < nthreads; t++)
        th.emplace_back(work, (int)((long long)P * t / nthreads),
                        (int)((long long)P * (t + 1) / nthreads));
    work(0, (int)((long long)P / nthreads));
    for (auto& x : th) x.join();
}

// Mt19937 draws for the RNG gate: kind 0 = random(), 1 = gauss(0,1),
// 2 = randbelow(arg).
void ref_mt_draws(unsigned long long seed, int kind, long long arg, int count, double* out) {
    Mt19937 r((uint64_t)seed);
    for (int i = 0; i < count; i++) {
        if (kind == 0) out[i] = r.random();
        else if (kind == 1) out[i] = r.gauss(0.0, 1.0);
        else out[i] = (double)r.randbelow((uint64_t)arg);
    }
}

}  // extern "C"

extern "C" {

// The reference's GP over `gens` steps with given fitness arrays
// (fits[g*pop + p]): ramped_half_and_half with Mt19937(seed), then gp_step
// (engine/gp.hpp:67-194) after each generation's fitness.  Writes the gens+1
// populations as prefix text, one rule per line, generations separated by a
// line "#".  Returns bytes used or -1.
long ref_gp_replay(const char* terminals_csv, int with_rmod, unsigned long long seed, int pop,
                   int gens, const double* fits, char* buf, long cap) {
    TreeConfig tc;
    tc.terminals = split_csv(terminals_csv);
    tc.functions = with_rmod ? FUNCS_RMOD : FUNCTIONS;
    EvolutionConfig cfg;
    cfg.population_size = pop;
    Mt19937 rng((uint64_t)seed);
    std::vector<NodeP> p = ramped_half_and_half(tc, rng, pop);
    std::string all;
    for (int g = 0; g <= gens; g++) {
        for (auto& t : p) {
            all += to_prefix(t);
            all += '\n';
        }
        all += "#\n";
        if (g == gens) break;
        std::vector<double> f(fits + (size_t)g * pop, fits + (size_t)(g + 1) * pop);
        p = gp_step(p, f, rng, tc, cfg);
    }
    if ((long)all.size() + 1 > cap) return -1;
    std::memcpy(buf, all.c_str(), all.size() + 1);
    return (long)all.size();
}

}  // extern "C"
