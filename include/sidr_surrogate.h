/*
 * sidr_surrogate.h -- C-ABI of the surrogate-assisted GP (no counterpart in
 * the reference, which evaluates every offspring in full).
 *
 * A rule's phenotype -- its priority ranking on fixed decision situations
 * recorded from simulator rollouts, plus token-count features -- feeds a
 * 40 -> 256 -> 256 -> 1 ReLU MLP with BF16 weights and activations and FP32
 * accumulation whose GEMMs run on hand-written sm_100a tensor-core kernels
 * (tcgen05.mma with TMEM accumulators).  The model is trained online on the
 * fitness the simulator has just produced and pre-screens GP offspring; the
 * simulator decides every reported fitness, and the GP falls back
 * to plain breeding when the model's rank correlation on an audit sample is
 * too low.
 */
#ifndef SIDR_SURROGATE_H
#define SIDR_SURROGATE_H

#include <stdint.h>

#include "sidr.h"
#include "sidr_gp.h"

#ifdef __cplusplus
extern "C" {
#endif

#define SIDR_MLP_INPUTS 40
#define SIDR_MLP_HIDDEN 256

/* Decision situations: `rule` (one rule, P = 1) rolled out on S scenarios
 * (sampled [S][n]) under `mask` by the evaluator, recording its first
 * max_decisions decisions of every rollout: for decision d of scenario s and
 * candidate c < max_cand (candidates in ascending customer order),
 * terms[((s*max_decisions + d)*max_cand + c)*61 + slot] holds the candidate's
 * 61-slot terminal table as pick_best fills it (engine/sim_core.hpp:84-197:
 * every slot active under the mask; inactive slots 0), cust[...] (may be
 * NULL) its customer index, and info[(s*max_decisions + d)*2] = {candidate
 * count, chosen customer or -1}; a rollout's unused decision entries have
 * candidate count 0. */
sidr_status sidr_capture_situations(sidr_ctx* ctx, const sidr_rules_desc* rule, const double* sampled,
                                    int32_t S, const int64_t* mask, int32_t max_decisions,
                                    int32_t max_cand, double* terms, int32_t* cust, int32_t* info);

/* Phenotype features of P rules over n_sit situations (terms
 * [n_sit][max_cand][61], ncand[n_sit] candidates each, ref[n_sit] = the
 * position of a reference choice among them): for situation j the rule's
 * priorities (eval_tree, engine/sim_core.hpp:11-41, NaN -> -1e300) rank the
 * candidates as pick_best does (strict >, lower position first on ties), and
 * feature j is the reference choice's place in that ranking / (ncand - 1).
 * Then 8 token-count features: length/255, depth/16, leaves/128, distinct
 * slots/32, constants/32, and the shares of +/-, * and /, and min/max/rmod
 * among the operators.  features[P][n_sit + 8]; n_sit = 32 gives the model's
 * 40 inputs. */
sidr_status sidr_phenotype(const sidr_rules_desc* rules, const double* terms, const int32_t* ncand,
                           const int32_t* ref, int32_t n_sit, int32_t max_cand, int device,
                           float* features);

/* C[M x N] (FP32) = A[M x K] * B[N x K]^T with BF16 operands given as raw
 * 16-bit patterns, on the tensor-core kernel the model uses (diagnostic).
 * splits > 1 splits K over CTAs that accumulate atomically.  N <= 256. */
sidr_status sidr_gemm_bf16(const uint16_t* A, const uint16_t* B, int32_t M, int32_t N, int32_t K,
                           int32_t splits, int device, float* C);

/* Failure-detection check of the GEMM kernel's bounded waits (diagnostic; no
 * reference counterpart).  One launch of the kernel on a 128 x 48 x 32 zero
 * problem in which the elected thread issues no MMA and no commit, so the
 * mbarrier phase every thread waits on never completes: each wait gives up
 * after wait_limit polls (1 .. 2^20), the kernel frees its tensor memory and
 * raises its error flag, and the host reads the flag.  Returns
 * SIDR_ERR_KERNEL when the flag was raised (the expected outcome); the device
 * context stays usable. */
sidr_status sidr_gemm_wait_check(int device, uint32_t wait_limit);

/* The model: parameters 0 W1 [256 x 48] (input columns 40..47 are zero
 * padding), 1 b1 [256], 2 W2 [256 x 256], 3 b2 [256], 4 w3 [256], 5 b3 [1],
 * FP32 masters with BF16 copies for the GEMMs; He-uniform initialisation
 * from seed. */
typedef struct sidr_mlp sidr_mlp;
sidr_status sidr_mlp_create(int device, uint64_t seed, sidr_mlp** out);
void sidr_mlp_destroy(sidr_mlp* m);

/* Reads (write = 0) or replaces (write = 1) parameter `which`'s FP32 values;
 * grads (may be NULL) receives its gradient from the last sidr_mlp_gradients
 * or training step; *count its size. */
sidr_status sidr_mlp_param(sidr_mlp* m, int32_t which, int32_t write, float* values, float* grads,
                           int64_t* count);

/* The model's whole training state, for checkpoints: every parameter's FP32
 * values, Adam first and second moments (parameters in order 0..5, each as
 * values, m, v), *count floats in all, and the Adam step count.  write = 0
 * reads into state (and *step), write = 1 replaces them from state (and
 * *step; the BF16 copies are refreshed).  state NULL: only *count (and
 * *step) are set. */
sidr_status sidr_mlp_state(sidr_mlp* m, int32_t write, float* state, int64_t* count, int64_t* step);

/* y[rows] = model(x[rows][40]). */
sidr_status sidr_mlp_predict(sidr_mlp* m, const float* x, int32_t rows, float* y);

/* Mean squared error of the model on (x, t) and the gradients of every
 * parameter (read them with sidr_mlp_param); no update. */
sidr_status sidr_mlp_gradients(sidr_mlp* m, const float* x, const float* t, int32_t rows, float* loss);

/* `steps` Adam steps (beta 0.9 / 0.999, eps 1e-8) of `batch` rows drawn
 * without replacement from (x[n][40], t[n]), reshuffled every pass. */
sidr_status sidr_mlp_train(sidr_mlp* m, const float* x, const float* t, int32_t n, int32_t steps,
                           int32_t batch, float lr, uint64_t seed, float* final_loss);

/* The surrogate-assisted GP's settings (defaults in brackets). */
typedef struct sidr_sgp_config {
    int32_t screen;            /* [8192] offspring bred and screened per generation */
    int32_t train_steps;       /* [200] Adam steps per generation */
    int32_t batch;             /* [1024] rows per step */
    float lr;                  /* [1e-3] */
    int32_t audit;             /* [128] screened offspring also simulated for the audit */
    double rho_min;            /* [0.8] audit Spearman rho below which the generation breeds plainly */
    int32_t history;           /* [3] generations of simulated fitness the model trains on */
    int32_t n_situations;      /* [32] decision situations of the phenotype (n_situations + 8 = 40) */
    int32_t capture_scenarios; /* [16] rollouts of the first generation's best rule they are sampled from */
    int32_t max_cand;          /* [64] candidates kept per situation */
    uint64_t model_seed;       /* [1] */
    int32_t use_surrogate;     /* [1] 0: the same driver with plain breeding (the comparison run) */
    int32_t device;            /* [0] device of the model and of the phenotype kernel */
    int32_t selection;         /* [0] 0: the best-predicted distinct offspring overall;
                                  1: pre-selection, the best-predicted of each group of
                                  screen / (slots screened) consecutive offspring */
    int32_t target;            /* [1] what the model is trained on: 0 the simulated fitness
                                  standardised over the history; 1 its ranks over the
                                  history as uniform scores (mean 0, variance 1), which
                                  keeps the order and drops the skew of broken rules */
    double screen_fraction;    /* [1.0] share of the non-elite slots filled by screened
                                  offspring in a screened generation; the rest are bred
                                  plainly (gp_step's loop), which keeps diversity */
    int32_t distinct;          /* [1] selection 0 keeps one child per 0: rule; 1: ranking of
                                  the decision situations (phenotype), so near-clones of one
                                  behaviour do not fill the population */
} sidr_sgp_config;

void sidr_sgp_default_config(sidr_sgp_config* cfg);

typedef struct sidr_sgp_result {
    double eval_seconds;   /* in the evaluator (population, audit, held-out, capture) */
    double model_seconds;  /* phenotypes, training, prediction */
    double host_seconds;   /* the rest: breeding, compiling, bookkeeping */
    int64_t evaluations;
    int32_t generations_screened, generations_fallback;
} sidr_sgp_result;

/* A GP run (engine/gp.hpp semantics, Mt19937(seed), train blocks of
 * cfg->train_samples scenarios from base seed seed*10000+gen) whose
 * offspring are pre-screened: each generation the model is trained on the
 * last `history` generations' simulated fitness (`target`), `screen`
 * offspring are bred by gp_step's loop, their phenotypes predicted, `audit`
 * of them simulated for Spearman's rho; at rho >= rho_min the next
 * population is the elites plus the screened offspring (`selection`) in
 * `screen_fraction` of the remaining slots and plainly bred offspring in the
 * rest, otherwise plain gp_step.  The decision situations come from the first generation's
 * best rule.  Every fitness reported is simulated.  Per generation g:
 * best_train[g], held_out[g] (the generation's best rule on test_samples
 * scenarios from test_seed), rho[g] (NaN when not audited), gen_seconds[g]
 * (wall clock since the start); best_rule: the last generation's best rule
 * as prefix text. */
sidr_status sidr_sgp_run(sidr_ctx* ctx, const sidr_instance_desc* inst, const sidr_gp_config* cfg,
                         const sidr_sgp_config* sc, const char* terminals_csv, const int64_t* mask,
                         uint64_t seed, int64_t test_seed, double* best_train, double* held_out,
                         double* rho, double* gen_seconds, char* best_rule, int64_t rule_cap,
                         sidr_sgp_result* result);

/* sidr_sgp_run with checkpoints (the reference's GP runs to the end in one
 * call and cannot resume).  After every `every` generations (0: never) the
 * driver's whole state -- the GP session, the decision situations, the
 * model's weights, Adam moments and step count, the fitness history the
 * model trains on, the counters and the per-generation outputs so far -- is
 * written to checkpoint_path, through a temporary file renamed over it.  If
 * checkpoint_path holds a checkpoint when the call starts, the run resumes
 * from it and gives exactly the outputs of an uninterrupted run (times
 * excepted); one written for another seed, test seed, instance, mask or
 * setting is refused (SIDR_ERR_INVALID).  stop_after >= 0: the call writes a
 * checkpoint and returns after that many generations of its own (the outputs
 * of the generations run so far are filled, best_rule is not); *finished
 * (may be NULL) is 1 when the run reached its last generation.  A NULL
 * checkpoint_path is sidr_sgp_run. */
sidr_status sidr_sgp_run_resumable(sidr_ctx* ctx, const sidr_instance_desc* inst, const sidr_gp_config* cfg,
                                   const sidr_sgp_config* sc, const char* terminals_csv, const int64_t* mask,
                                   uint64_t seed, int64_t test_seed, const char* checkpoint_path, int32_t every,
                                   int32_t stop_after, int32_t* finished, double* best_train, double* held_out,
                                   double* rho, double* gen_seconds, char* best_rule, int64_t rule_cap,
                                   sidr_sgp_result* result);

/* The large combined run (no single reference call: the reference runs
 * exhaust_batched, engine/gp_engine.cu:131-203, once per instance and seed
 * set, without a surrogate): K instances (zps [K][10], masks [K][61]) x
 * n_seeds GP runs each (GP seeds first_seed .. first_seed + n_seeds - 1),
 * population e = k * n_seeds + s, evolved together with the pre-screening of
 * sidr_sgp_run.  Per generation every population is simulated in ONE
 * multi-instance launch (sidr_multi_*; shape as in sidr_gp_run_multi), each
 * on its own train block (base seed seed*10000 + gen) of its instance; each
 * instance has its own decision situations (from the first generation's best
 * rule of its first seed) and its own model, trained on the window of all its
 * seeds' simulated fitness; every population breeds and screens its own
 * offspring, and all audits run in one more multi-instance launch.  Per
 * generation g and population e: best_train[g*E + e], held_out[g*E + e] (the
 * best rule on test_samples scenarios from test_seed of its instance),
 * rho[g*E + e] (NaN when not audited); any of them may be NULL.  best_rules
 * (may be NULL): the last generation's best rule of every population as prefix
 * text, one line each in population order.  With K = 1 and n_seeds = 1 the
 * run is sidr_sgp_run's, value for value.
 * result->generations_screened / _fallback count population-generations. */
sidr_status sidr_sgp_run_multi(const sidr_instance_desc* insts, const double* zps, int32_t K,
                               const sidr_gp_config* cfg, const sidr_sgp_config* sc,
                               const char* terminals_csv, const int64_t* masks, int32_t n_seeds,
                               int64_t first_seed, int64_t test_seed, int32_t shape,
                               double* best_train, double* held_out, double* rho,
                               char* best_rules, int64_t rules_cap, sidr_sgp_result* result);

/* sidr_sgp_run_multi with checkpoints, as sidr_sgp_run_resumable: every
 * `every` generations the whole state -- every population's GP session,
 * each instance's situations, model (weights, Adam moments, step count) and
 * fitness window, the launch shape, the counters and the per-generation
 * outputs so far -- goes to checkpoint_path (temporary file, then rename);
 * a call that finds a checkpoint there resumes from it and gives exactly the
 * uninterrupted run's outputs (times excepted); one written for other
 * instances, seeds, masks or settings is refused (SIDR_ERR_INVALID);
 * stop_after >= 0 ends the call after that many generations with a
 * checkpoint written (best_rules is filled only by the call that reaches
 * the last generation); *finished (may be NULL) is 1 when the run is
 * complete.  A NULL checkpoint_path is sidr_sgp_run_multi. */
sidr_status sidr_sgp_run_multi_resumable(const sidr_instance_desc* insts, const double* zps, int32_t K,
                                         const sidr_gp_config* cfg, const sidr_sgp_config* sc,
                                         const char* terminals_csv, const int64_t* masks, int32_t n_seeds,
                                         int64_t first_seed, int64_t test_seed, int32_t shape,
                                         const char* checkpoint_path, int32_t every, int32_t stop_after,
                                         int32_t* finished, double* best_train, double* held_out, double* rho,
                                         char* best_rules, int64_t rules_cap, sidr_sgp_result* result);

#ifdef __cplusplus
}
#endif
#endif
