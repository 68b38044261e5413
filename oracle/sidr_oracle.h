/*
 * sidr_oracle.h -- CPU oracle for the rule x scenario evaluator.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * simulator (augustompm/solver-informed-dispatching-rules, engine/sim_core.hpp,
 * engine/sim_terms.hpp, engine/sim_host.hpp, engine/rng.hpp).  It exists to
 * check the CUDA evaluator; no product code path links it.  Only the tests,
 * __graft_entry__.smoke() and the cpu_baseline leg of bench.py load it.
 *
 * Parity of this restatement is pinned against the reference's own golden
 * vectors (verify/golden/sim.txt, gp.txt, durations.txt, rng.txt, through the
 * fixtures under tests/golden/) and against the reference's sim_batch compiled
 * from its own headers into oracle/_ref/.
 *
 * Every arithmetic expression keeps the reference's operand order and
 * association; build with -ffp-contract=off so no multiply-add is fused.
 */
#ifndef SIDR_ORACLE_H
#define SIDR_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SO_N_TERMS 61
#define SO_MAX_N 512
#define SO_MAX_STACK 32

/* Instance arrays in the reference's SimData layout (engine/sim_host.hpp:12-40):
 * customers 0..n-1, dist is (n+1)x(n+1) row-major with the depot at index 0. */
typedef struct so_simdata {
    int n, m, ld;
    double tmax;
    const double *scores, *durations, *open_t, *close_t, *dist, *dist_to_depot;
} so_simdata;

/* dist[(n+1)^2] and dist_to_depot[n] from coordinates (x[0], y[0]) = depot,
 * following SimData's constructor (engine/sim_host.hpp:29-38). */
void so_build_dist(int n, const double* x, const double* y, double* dist, double* dist_to_depot);

/* zp[10] = 5 means then 5 stds of the z-features (engine/sim_core.hpp:277-312,
 * engine/sim_host.hpp:96-105). */
void so_zstats(const so_simdata* sd, double* zp);

/* MT19937 with Python-compatible seeding and draws (engine/rng.hpp). */
typedef struct so_mt {
    uint32_t mt[624];
    int mti;
    int has_gauss;
    double gauss_next;
} so_mt;
void so_mt_seed(so_mt* r, uint64_t seed);
uint32_t so_mt_genrand(so_mt* r);
double so_mt_random(so_mt* r);
double so_mt_gauss(so_mt* r, double mu, double sigma);

/* Scenario s uses a fresh generator seeded base_seed + s
 * (engine/sim_host.hpp:43-58).  out is [S][n]. */
void so_gen_durations(int n, const double* durations, double sigma, int S, long long base_seed,
                      double* out);

/* The postfix interpreter (engine/sim_core.hpp:11-41). */
double so_eval_tree(const int32_t* ops, const int32_t* args, int len, const double* terms,
                    double* stack);

/* One (rule, scenario) rollout (engine/sim_core.hpp:207-238). */
double so_sim_one(const so_simdata* sd, const int32_t* ops, const int32_t* args, int len,
                  const double* sampled, const int64_t* term_mask, const double* zp);

/* Work counters of one rollout, for the op model of the roofline. */
typedef struct so_counts {
    int64_t decisions;     /* pick_best calls */
    int64_t candidates;    /* feasible unvisited candidates scored */
    int64_t tokens;        /* interpreter tokens executed */
} so_counts;

/* Every (rule, scenario) pair of a grouped, multi-mask batch, the CPU twin of
 * FactoryContext::evaluate_grouped_masks (engine/factory.cuh:193-216):
 * rule p reads scenarios of group p/group_size and mask row p/mask_group.
 * out[p*T + s].  evaluate == G=1, group_size=mask_group=P.  Runs on nthreads
 * host threads (rules split across threads).  counts may be NULL. */
void so_eval_pairs(const so_simdata* sd, const double* zp,
                   const int32_t* ops, const int32_t* args, const int32_t* offsets,
                   const int32_t* lengths, int P,
                   const double* grouped_sampled, int T, int group_size,
                   const int64_t* masks, int mask_group, double* out, int nthreads,
                   so_counts* counts);

#ifdef __cplusplus
}
#endif
#endif
