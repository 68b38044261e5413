/*
 * sidr_gp.h -- C-ABI of the host GP loop that drives the evaluator.
 *
 * The reference's GP (augustompm/solver-informed-dispatching-rules,
 * engine/gp.hpp:13-194) and its seed-batched driver (engine/gp_engine.cu:
 * 131-203), rebuilt on flat prefix-order rule arrays: ramped half-and-half
 * initialisation, Koza 90/10 point selection, subtree crossover and mutation
 * under the depth limit, size-7 tournaments, elitism and gp_step's rates, all
 * driven by a Python-compatible MT19937 so that the same seed gives the same
 * populations as the reference.  Fitness comes from the B200 evaluator.
 */
#ifndef SIDR_GP_H
#define SIDR_GP_H

#include <stdint.h>

#include "sidr.h"

#ifdef __cplusplus
extern "C" {
#endif

/* EvolutionConfig and TreeConfig (engine/gp.hpp:13-34). */
typedef struct sidr_gp_config {
    int32_t population;        /* 1024 */
    int32_t generations;       /* 51   */
    int32_t max_depth;         /* 8    */
    int32_t min_depth;         /* 2    */
    int32_t tournament;        /* 7    */
    int32_t elitism;           /* 10   */
    double crossover_rate;     /* 0.80 */
    double mutation_rate;      /* 0.15 */
    double reproduction_rate;  /* 0.05 */
    int32_t train_samples;     /* 1    */
    int32_t test_samples;      /* 500  */
    int32_t with_rmod;         /* 0: FUNCTIONS, 1: FUNCS_RMOD (engine/tree.hpp:33-34) */
} sidr_gp_config;

/* The reference defaults (engine/gp.hpp:20-34). */
void sidr_gp_default_config(sidr_gp_config* cfg);

/* One GP population of one seed (engine/gp_engine.cu:69-84's state).
 * terminals_csv: the terminal set, comma separated ("ERC" = random constant,
 * label "%.3f"); the generator is Mt19937(seed). */
typedef struct sidr_gp_session sidr_gp_session;
sidr_status sidr_gp_create(const sidr_gp_config* cfg, const char* terminals_csv, uint64_t seed,
                           sidr_gp_session** out);
void sidr_gp_destroy(sidr_gp_session* s);

/* The population as prefix text (engine/tree.hpp:62-69), '\n' separated;
 * returns the bytes needed (call with cap 0 to size the buffer). */
int64_t sidr_gp_population_text(const sidr_gp_session* s, char* buf, int64_t cap);

/* The population compiled to the evaluator's PackedTrees layout
 * (engine/factory.cuh:26-40): sizes first (pass NULL arrays), then fill. */
sidr_status sidr_gp_population_packed(const sidr_gp_session* s, int32_t* ops, int32_t* args,
                                      int32_t* offsets, int32_t* lengths, int64_t* n_nodes);

/* gp_step (engine/gp.hpp:170-194) with the given per-rule fitness. */
sidr_status sidr_gp_step(sidr_gp_session* s, const double* fitness);

/* Number of sidr_gp_step calls the session has made (-1 for NULL). */
int64_t sidr_gp_generation(const sidr_gp_session* s);

/* Checkpoint / resume (the reference resumes only its vocabulary GA, through
 * the evaluation cache of s4_selection/ga.cu:301-346; the GP itself restarts).
 * sidr_gp_checkpoint writes the session's whole state as text -- config,
 * step count, terminal set, leaf-label table (ERC constants included), the
 * MT19937 state and the population -- and returns the bytes needed (call
 * with cap 0 to size the buffer; -1 for NULL).  sidr_gp_restore makes a new
 * session from it that continues exactly as the checkpointed one would;
 * malformed or inconsistent text is refused with SIDR_ERR_INVALID. */
int64_t sidr_gp_checkpoint(const sidr_gp_session* s, char* buf, int64_t cap);
sidr_status sidr_gp_restore(const char* checkpoint, sidr_gp_session** out);

/* The seed-batched GP run of engine/gp_engine.cu:131-203 (exhaust_batched):
 * n_seeds populations (seeds first_seed .. first_seed+n_seeds-1) evolve
 * together, each generation evaluated in one grouped call on the evaluator with
 * train_samples scenarios of base seed seed*10000+gen per population; after the
 * last generation the best rule of each population (on one more train block) is
 * scored on test_samples scenarios from test_seed.
 *   best_test[n_seeds]      mean held-out score of each population's best rule
 *   best_train[gens*n_seeds] best train fitness per generation and population
 *   best_rules              the best rules' prefix text, '\n' separated
 *   eval_seconds / host_seconds  time in evaluator calls / in the host GP
 */
typedef struct sidr_gp_result {
    double eval_seconds;
    double host_seconds;
    int64_t evaluations;
} sidr_gp_result;
sidr_status sidr_gp_run_batched(sidr_ctx* ctx, const sidr_instance_desc* inst,
                                const sidr_gp_config* cfg, const char* terminals_csv,
                                const int64_t* term_mask, int32_t n_seeds, int64_t first_seed,
                                int64_t test_seed, double* best_test, double* best_train,
                                char* best_rules, int64_t rules_cap, sidr_gp_result* result);

/* The seed-batched run one generation at a time, with checkpoint and resume
 * (the reference's exhaust_batched, engine/gp_engine.cu:131-203, runs to the
 * end in one call and cannot resume).  sidr_gp_run_batched is create, step
 * through every generation, finish.
 *   sidr_gp_batched_create    the populations of seeds first_seed ..
 *                             first_seed + n_seeds - 1 (ctx must hold inst;
 *                             the driver keeps a copy of what it needs)
 *   sidr_gp_batched_step      evaluates (and breeds from) up to `generations`
 *                             more generations, no further than cfg->generations
 *   sidr_gp_batched_generation  generations evaluated so far
 *   sidr_gp_batched_checkpoint  the run's whole state as text: seeds, the
 *                             instance's hash, the mask, the generation reached,
 *                             best train fitness so far, time and evaluation
 *                             counters, and every seed's session as
 *                             sidr_gp_checkpoint writes it; returns the bytes
 *                             needed (cap 0 sizes the buffer; -1 for NULL)
 *   sidr_gp_batched_restore   a run that continues exactly as the checkpointed
 *                             one would; refused (SIDR_ERR_INVALID) when the
 *                             text is malformed or was written for another
 *                             instance; ctx must hold inst
 *   sidr_gp_batched_finish    after the last generation: the final train block,
 *                             each seed's best rule on the held-out block, and
 *                             the outputs of sidr_gp_run_batched (its times and
 *                             evaluations count the resumed parts too) */
typedef struct sidr_gp_batched sidr_gp_batched;
sidr_status sidr_gp_batched_create(sidr_ctx* ctx, const sidr_instance_desc* inst, const sidr_gp_config* cfg,
                                   const char* terminals_csv, const int64_t* term_mask, int32_t n_seeds,
                                   int64_t first_seed, int64_t test_seed, sidr_gp_batched** out);
sidr_status sidr_gp_batched_step(sidr_gp_batched* b, int32_t generations);
int64_t sidr_gp_batched_generation(const sidr_gp_batched* b);
int64_t sidr_gp_batched_checkpoint(const sidr_gp_batched* b, char* buf, int64_t cap);
sidr_status sidr_gp_batched_restore(sidr_ctx* ctx, const sidr_instance_desc* inst, const char* checkpoint,
                                    sidr_gp_batched** out);
sidr_status sidr_gp_batched_finish(sidr_gp_batched* b, double* best_test, double* best_train, char* best_rules,
                                   int64_t rules_cap, sidr_gp_result* result);
void sidr_gp_batched_destroy(sidr_gp_batched* b);

/* Many instances x many seeds (no single reference call: the reference runs
 * exhaust_batched, engine/gp_engine.cu:131-203, once per instance).  For each
 * of the K instances (zps [K][10], masks [K][61]) the seed-batched run of
 * sidr_gp_run_batched with seeds first_seed .. first_seed + n_seeds - 1; all
 * K * n_seeds populations are evaluated together in ONE multi-instance launch
 * per generation (sidr_multi_*), each on its own instance and train block.
 * Per instance the results equal sidr_gp_run_batched's on that instance
 * alone.  shape: the launch's block shape (0 .. SIDR_MULTI_SHAPES-1), or -1 to
 * choose it on the first launch (sidr_multi_autotune_sampled on every 16th
 * rule) and keep the choice.  Each generation builds
 * its batch anew (instance tables included, on the host).
 *   best_test[K*n_seeds]           held-out mean of each population's best rule
 *   best_train[gens*K*n_seeds]     index (gen*K + k)*n_seeds + s
 *   best_rules                     K*n_seeds prefix lines in (k, s) order */
sidr_status sidr_gp_run_multi(const sidr_instance_desc* insts, const double* zps, int32_t K,
                              const sidr_gp_config* cfg, const char* terminals_csv, const int64_t* masks,
                              int32_t n_seeds, int64_t first_seed, int64_t test_seed, int32_t shape,
                              int32_t device, double* best_test, double* best_train, char* best_rules,
                              int64_t rules_cap, sidr_gp_result* result);

/* gen_durations (engine/sim_host.hpp:43-58) on the host: [S][n]. */
sidr_status sidr_gen_durations(int32_t n, const double* durations, double sigma, int32_t S,
                               int64_t base_seed, double* out);

/* gen_durations on the GPU (the reference samples on the host:
 * engine/sim_host.hpp:50-58 with engine/rng.hpp:27-147), bit-identical to
 * sidr_gen_durations.  One warp per scenario runs the MT19937 seeding and
 * refresh in shared memory; the Box-Muller log, cos and sin are computed in
 * double-double arithmetic, and a pair whose C-library result those values
 * do not settle (a few percent) is recomputed on the host with the C library
 * after the kernel (a block with more of them than an eighth of its pairs
 * is sampled on the host as a whole).  out: [S][n] doubles in host memory
 * (out_on_device = 0) or in the device memory of `device` (1).  stats (may
 * be NULL): Box-Muller pairs drawn and pairs computed on the host.  The call
 * allocates its device scratch and waits for its work. */
typedef struct sidr_sample_stats {
    int64_t pairs;
    int64_t host_pairs;
} sidr_sample_stats;
sidr_status sidr_gen_durations_device(int32_t device, int32_t n, const double* durations, double sigma,
                                      int32_t S, int64_t base_seed, double* out, int32_t out_on_device,
                                      sidr_sample_stats* stats);
/* Diagnostic of the sampler (no reference counterpart): the double-double
 * log(1 - u2[i]), sin(2 pi u1[i]) and cos(2 pi u1[i]) it settles pairs with
 * and the second C-library candidate each names (the value itself when it
 * names one), out[9 i ..] = {log hi, lo, second, sin hi, lo, second, cos hi,
 * lo, second}, computed by the device build (on_device = 1, on `device`) or
 * the host build (0) of the same code; the two must agree bit for bit. */
sidr_status sidr_sample_dd_eval(int32_t device, const double* u1, const double* u2, int32_t k,
                                int32_t on_device, double* out);

#ifdef __cplusplus
}
#endif
#endif
