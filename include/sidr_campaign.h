/*
 * sidr_campaign.h -- C-ABI of the campaign drivers around the evaluator.
 *
 * The reference's stage-3/4 programs, rebuilt on the host GP of sidr_gp.h and
 * the B200 evaluator of sidr.h:
 *   - the vocabulary GA over terminal subsets (s4_selection/ga.cu): lockstep
 *     retraining of many genomes in one grouped-masks launch per generation
 *     (batch_score, :111-205), its one-genome sequential twin (seq_score,
 *     :208-258), the --gate check between the two (:260-286), and the
 *     tree-13 GA itself with its evaluation cache (:288-523);
 *   - the per-generation trace of a GP campaign written as the reference's
 *     trace JSON (s3_generation/gen_trace.cu);
 *   - redeploy sealing of a trace's best rule on the held-out block
 *     (s4_selection/redeploy.cu);
 *   - the train-side score of the cross-validatory choice between traces
 *     (s4_selection/choice.cu).
 *
 * Genomes are bitmasks over a universe of terminal names: bit b adds
 * universe[b] to the base terminal set (s4_selection/ga.cu:90-95).  Term sets
 * are comma-separated names.  Failures return a status and set
 * sidr_last_error().
 */
#ifndef SIDR_CAMPAIGN_H
#define SIDR_CAMPAIGN_H

#include <stdint.h>

#include "sidr.h"
#include "sidr_gp.h"

#ifdef __cplusplus
extern "C" {
#endif

/* The fixed blocks of the campaign programs: the TRAIN block 2M x 64
 * (s4_selection/ga.cu:31-32, choice.cu:14-15) and the held-out block 1M x 500
 * (s3_generation/gen_trace.cu:20-21, redeploy.cu:14-15). */
#define SIDR_TRAIN_SEED 2000000
#define SIDR_TRAIN_N 64
#define SIDR_TEST_SEED 1000000
#define SIDR_TEST_N 500

/* batch_score (s4_selection/ga.cu:111-205).  For each genome k and seed
 * s < n_seeds a GP population (Mt19937(s), the genome's terminal set, cfg's
 * population) is trained for n_gens generations on train blocks of
 * cfg->train_samples scenarios from base seed s*10000+gen; genomes go through
 * in chunks of bmax, and each generation of a chunk is ONE
 * sidr_evaluate_grouped_masks call over chunk x seeds x population with one
 * mask row per genome.  After generation n_gens the best rule of each
 * population (strict >, first index) is scored on block_n scenarios from
 * block_seed.  out[K * n_seeds]: those means, genome-major.  result (may be
 * NULL): evaluator and host seconds and evaluations. */
sidr_status sidr_vocab_batch_score(sidr_ctx* ctx, const sidr_instance_desc* inst,
                                   const sidr_gp_config* cfg, const char* base_csv,
                                   const char* universe_csv, const uint32_t* genomes, int32_t K,
                                   int32_t n_seeds, int32_t n_gens, int32_t bmax,
                                   int64_t block_seed, int32_t block_n, double* out,
                                   sidr_gp_result* result);

/* seq_score (s4_selection/ga.cu:208-258): one genome, one
 * sidr_evaluate_grouped call per generation under the genome's mask, the
 * finals scored with sidr_evaluate.  out[n_seeds]. */
sidr_status sidr_vocab_seq_score(sidr_ctx* ctx, const sidr_instance_desc* inst,
                                 const sidr_gp_config* cfg, const char* base_csv,
                                 const char* universe_csv, uint32_t genome, int32_t n_seeds,
                                 int32_t n_gens, int64_t block_seed, int32_t block_n, double* out);

/* --gate (s4_selection/ga.cu:260-286): the five gate genomes {0, all,
 * bit 0, bit min(7, nb-1), bits 1|4|9 (clipped)} scored by batch_score and by
 * seq_score at n_seeds seeds x n_gens generations; counts the compared values
 * and the mismatches (bitwise), and the largest |difference|.  SIDR_OK means
 * the gate ran; *mismatches == 0 means it passed. */
sidr_status sidr_vocab_gate(sidr_ctx* ctx, const sidr_instance_desc* inst,
                            const sidr_gp_config* cfg, const char* base_csv,
                            const char* universe_csv, int32_t n_seeds, int32_t n_gens,
                            int32_t bmax, int64_t block_seed, int32_t block_n, int64_t* compared,
                            int64_t* mismatches, double* max_diff);

/* The GA's settings (s4_selection/ga.cu:10-13 command line, defaults in
 * brackets). */
typedef struct sidr_vocab_ga_config {
    int32_t pgens;         /* [51] inner generations of a proxy evaluation */
    int32_t proxy;         /* [16] seeds of a proxy evaluation */
    int32_t confirm;       /* [30] seeds of the champion confirmation */
    int32_t gens;          /* [50] GA generation cap */
    int32_t stag;          /* [5]  stagnation cutoff */
    int32_t bmax;          /* [10] genomes per batch */
    int32_t top;           /* [4]  finalists confirmed */
    double pm;             /* [0.5] mutation multiplier: per-gene rate pm / nb */
    int32_t seeds_neutral; /* [0]  1: seed the pool with {}, {all}, singletons */
    int32_t nofull;        /* [0]  1: leave {all} out of the neutral seeds */
    int64_t ga_seed;       /* [20260714] the GA's own Mt19937 */
} sidr_vocab_ga_config;

void sidr_vocab_ga_default_config(sidr_vocab_ga_config* cfg);

/* A fitness source for the GA in place of batch_score: fills
 * out[K * n_seeds] (genome-major) with per-seed scores of genomes[K] at
 * n_seeds seeds and n_gens inner generations; returns 0 on success. */
typedef int (*sidr_vocab_fitness_fn)(void* user, const uint32_t* genomes, int32_t K,
                                     int32_t n_seeds, int32_t n_gens, double* out);

/* The GA (s4_selection/ga.cu:288-523): pool of 13 (seeded, then random genomes
 * with bit rate 0.35), tree of leader/supporter clusters restored by swaps,
 * 12 uniform-crossover children per generation replacing the worse parent,
 * re-injection when at most 6 genomes are distinct, stagnation stop, top
 * finalists confirmed at `confirm` seeds with cfg->generations inner
 * generations, champion by confirmed mean (ties: fewer terminals).
 * fitness == NULL: batch_score on ctx/inst with the TRAIN block; otherwise
 * the callback is the only fitness source (ctx and inst may be NULL).
 * cache_path (may be NULL): the evaluation cache file of ga.cu:315-377
 * (header line, "P"/"C" lines with hexfloat scores), read at start and
 * appended as batches finish.  log (may be NULL): the program's stdout lines
 * (timings included), needed bytes in *log_len.  instance_name labels the
 * log and the cache header. */
sidr_status sidr_vocab_ga(sidr_ctx* ctx, const sidr_instance_desc* inst,
                          const sidr_gp_config* cfg, const sidr_vocab_ga_config* ga,
                          const char* instance_name, const char* base_csv,
                          const char* universe_csv, const char* cache_path,
                          sidr_vocab_fitness_fn fitness, void* user, uint32_t* champion,
                          double* champion_mean, int64_t* evals, char* log, int64_t log_cap,
                          int64_t* log_len);

/* gen_trace (s3_generation/gen_trace.cu:55-185): n_seeds GP runs (Mt19937(s),
 * base + extra terminals, cfg) evaluated together per generation; per seed and
 * generation the best rule's train fitness (rounded half-even to 0.1), size and
 * extra terminals; at the end each seed's best rule is scored on n_test
 * scenarios from test_seed and its gain over km (100*(got-km)/km) recorded.
 * json receives the trace file's text as the reference writes it (needed
 * bytes in *json_len); mean_gain (may be NULL) the mean gain. */
sidr_status sidr_gen_trace(sidr_ctx* ctx, const sidr_instance_desc* inst,
                           const sidr_gp_config* cfg, const char* instance_name,
                           const char* base_csv, const char* extra_csv, int32_t n_seeds,
                           double km, int64_t test_seed, int32_t n_test, char* json,
                           int64_t json_cap, int64_t* json_len, double* mean_gain);

/* redeploy (s4_selection/redeploy.cu:17-50): the trace's best final (largest
 * "gain", first on ties) is parsed from its prefix text and scored on n_test
 * scenarios from test_seed under base + the trace's "vocab_extra"; *gain is
 * its gain over km, *delta = |gain - trace gain|, *sealed = delta <= 0.005.
 * The trace's "instance" must equal instance_name. */
sidr_status sidr_redeploy(sidr_ctx* ctx, const sidr_instance_desc* inst, const char* instance_name,
                          const char* trace_json, const char* base_csv, double km,
                          int64_t test_seed, int32_t n_test, double* trace_gain, double* gain,
                          double* delta, int32_t* sealed);

/* Mean TRAIN score of a trace (s4_selection/choice.cu:41-52, 70-89): the
 * trace's finals sorted by seed, each scored on n_train scenarios from
 * train_seed under base + "vocab_extra"; the mean over rules of each rule's
 * mean.  *heldout receives the trace's "mean_gain". */
sidr_status sidr_trace_mean_train(sidr_ctx* ctx, const sidr_instance_desc* inst,
                                  const char* trace_json, const char* base_csv,
                                  int64_t train_seed, int32_t n_train, double* mean_train,
                                  double* heldout);

/* Prefix text of one rule (engine/tree.hpp:62-95) compiled to the
 * evaluator's post-order encoding (engine/vocab.hpp:99-126).  Sizes first
 * (NULL arrays), then fill; *len = node count. */
sidr_status sidr_rule_compile_prefix(const char* prefix, int32_t* ops, int32_t* args, int32_t* len);

#ifdef __cplusplus
}
#endif
#endif
