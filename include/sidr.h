/*
 * sidr.h -- C-ABI of the B200 rule x scenario evaluator.
 *
 * Scores postfix-encoded dispatching rules against stochastic route-simulation
 * scenarios of the stochastic team orienteering problem with time windows,
 * bit-exact against the reference CPU simulator
 * (augustompm/solver-informed-dispatching-rules, engine/sim_host.hpp:67-83
 * sim_batch -> engine/sim_core.hpp sim_one/pick_best).
 *
 * Plain pointers and sizes only.  Every function returns a status and never
 * exits the process (the reference's CUDA_CHECK calls exit(2),
 * engine/factory.cuh:16-18); sidr_last_error() describes the last failure on
 * the calling thread.  One context per host thread, or external locking.
 *
 * Data formats are the reference's own:
 *   instance  -- SimData SoA (engine/sim_host.hpp:12-40): customers 0..n-1,
 *                dist (n+1)x(n+1) row-major with the depot at index 0;
 *   rules     -- PackedTrees (engine/factory.cuh:20-24): post-order int32
 *                ops[] (-1 terminal slot, -2 constant in thousandths, 0..5
 *                + - * / min max, 6 rmod) with two int32 args per node, and
 *                per-rule offsets[] / lengths[];
 *   scenarios -- sampled service durations, [G groups][T scenarios][n];
 *   masks     -- int64 rows of 61 terminal flags (engine/sim_host.hpp:85-94);
 *   output    -- out[p*T + s], the collected score of rule p on scenario s.
 */
#ifndef SIDR_H
#define SIDR_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SIDR_N_TERMS 61   /* engine/vocab.hpp:16 N_TERMS   */
#define SIDR_MAX_N 512    /* engine/vocab.hpp:17 MAX_N     */
#define SIDR_MAX_TREE 1024 /* engine/vocab.hpp:18 MAX_TREE */
#define SIDR_MAX_STACK 32 /* engine/vocab.hpp:19 MAX_STACK */

typedef enum sidr_status {
    SIDR_OK = 0,
    SIDR_ERR_INVALID = 1,   /* bad argument, size or pointer            */
    SIDR_ERR_RULE = 2,      /* malformed rule (opcode, slot, stack)      */
    SIDR_ERR_TOO_LARGE = 3, /* n > SIDR_MAX_N, rule > SIDR_MAX_TREE ...  */
    SIDR_ERR_CUDA = 4,      /* a CUDA runtime call failed                */
    SIDR_ERR_NO_DEVICE = 5, /* no usable CUDA device                     */
    SIDR_ERR_KERNEL = 6,    /* the kernel reported an internal fault     */
    SIDR_ERR_NONFINITE = 7  /* NaN or infinity in instance or scenarios  */
} sidr_status;

typedef struct sidr_ctx sidr_ctx;
typedef struct sidr_batch sidr_batch;

/* One instance, the reference's SimData (engine/sim_host.hpp:12-40). */
typedef struct sidr_instance_desc {
    int32_t n;                    /* customers (depot excluded), 1..SIDR_MAX_N */
    int32_t m;                    /* vehicles                                  */
    double tmax;                  /* route deadline (depot due time)           */
    const double* scores;         /* [n]                                       */
    const double* durations;      /* [n] expected service times                */
    const double* open_t;         /* [n]                                       */
    const double* close_t;        /* [n]                                       */
    const double* dist;           /* [(n+1)*(n+1)], depot at 0                 */
    const double* dist_to_depot;  /* [n]                                       */
} sidr_instance_desc;

/* Rules in the reference's PackedTrees layout (engine/factory.cuh:20-40). */
typedef struct sidr_rules_desc {
    const int32_t* ops;      /* [n_nodes]                       */
    const int32_t* args;     /* [2*n_nodes]                     */
    const int32_t* offsets;  /* [P] first node of rule p        */
    const int32_t* lengths;  /* [P] node count of rule p        */
    int32_t P;               /* rules                           */
    int64_t n_nodes;         /* length of ops                   */
} sidr_rules_desc;

const char* sidr_last_error(void);
const char* sidr_status_string(sidr_status s);
int sidr_version(void);

/* zp_of (engine/sim_host.hpp:96-105 -> zstats, engine/sim_core.hpp:277-312):
 * the 5 z-feature means then 5 stds at the initial state, computed on the host
 * with the same libm as the reference. */
sidr_status sidr_zstats(const sidr_instance_desc* inst, double zp[10]);

/* Diagnostic, host only (no reference counterpart): builds the instance's
 * tables and checks ATRISK's per-pair step functions -- the outcome of
 * engine/sim_terms.hpp:225-257's term (+0, s_j, or erf needed) as a function
 * of the candidate's finish time, which the kernel looks up -- against the
 * classification itself at every switch point, its neighbours and random
 * times.  *checked: points checked; *mismatches: must be 0. */
sidr_status sidr_atrisk_table_check(const sidr_instance_desc* inst, int32_t seed, int64_t* checked,
                                    int64_t* mismatches);

/* FactoryContext(sd, zp) (engine/factory.cuh:129-137): copies the instance to
 * device `device` once, with the per-instance lookup tables the kernels use. */
sidr_status sidr_ctx_create(const sidr_instance_desc* inst, const double zp[10], int device,
                            sidr_ctx** out);
void sidr_ctx_destroy(sidr_ctx* ctx);

/* FactoryContext::evaluate (engine/factory.cuh:144-164): all P rules on the
 * same N scenarios (sampled [N][n]) under one mask; out[P*N] host. */
sidr_status sidr_evaluate(sidr_ctx* ctx, const sidr_rules_desc* rules, const double* sampled,
                          int32_t N, const int64_t* term_mask, double* out);

/* FactoryContext::evaluate_grouped (engine/factory.cuh:167-189): rule p uses
 * scenario group p/group_size of grouped_sampled [G][T][n]; out[P*T] host. */
sidr_status sidr_evaluate_grouped(sidr_ctx* ctx, const sidr_rules_desc* rules,
                                  const double* grouped_sampled, int32_t G, int32_t T,
                                  int32_t group_size, const int64_t* term_mask, double* out);

/* FactoryContext::evaluate_grouped_masks (engine/factory.cuh:193-216): as
 * grouped, with mask row p/mask_group of masks [ceil(P/mask_group)][61].
 * G (the group count, which the reference infers from the vector size) is
 * passed explicitly so the scenario buffer can be bounds-checked. */
sidr_status sidr_evaluate_grouped_masks(sidr_ctx* ctx, const sidr_rules_desc* rules,
                                        const double* grouped_sampled, int32_t G, int32_t T,
                                        int32_t group_size, int32_t mask_group,
                                        const int64_t* masks, double* out);

/* Device-resident batches (no reference counterpart; the reference copies
 * every input on every call, engine/factory.cuh:144-164).  sidr_batch_create
 * validates and repacks the rules, uploads rules, scenarios and masks once and
 * keeps them in HBM; sidr_batch_run launches the evaluator on `stream`
 * (a cudaStream_t, 0 = legacy default) and returns without waiting;
 * sidr_batch_read waits for the stream and copies out[P*T] to the host;
 * sidr_batch_fitness writes the per-rule mean over the T scenarios, summed in
 * scenario order then divided by T, as the reference drivers do
 * (engine/gp_engine.cu:76-81). */
sidr_status sidr_batch_create(sidr_ctx* ctx, const sidr_rules_desc* rules,
                              const double* grouped_sampled, int32_t G, int32_t T,
                              int32_t group_size, int32_t mask_group, const int64_t* masks,
                              sidr_batch** out);
sidr_status sidr_batch_run(sidr_batch* b, void* stream);
sidr_status sidr_batch_read(sidr_batch* b, double* out);
sidr_status sidr_batch_fitness(sidr_batch* b, double* fitness);
/* Device pointer of the [P*T] result buffer (valid until destroy). */
const double* sidr_batch_device_out(const sidr_batch* b);
void sidr_batch_destroy(sidr_batch* b);

/* Work counters of the last run of a batch (filled when the batch was run with
 * counting enabled by sidr_batch_set_counting; no reference counterpart).
 * fp64_ops is the op model of the roofline: the floating-point operations the
 * reference's loops perform for the same decisions -- per neighbour visited
 * by an enabled terminal family, its feasibility test (6 ops) plus the
 * family's payload; ATRISK neighbours 40 (two erf counted as 15 each);
 * candidate setup and the rule's binary operators 1 each. */
typedef struct sidr_counts {
    int64_t decisions;   /* pick_best calls                               */
    int64_t candidates;  /* feasible candidates scored                     */
    int64_t scan_iters;  /* (candidate, neighbour) pairs of the fused scan */
    int64_t heavy_iters; /* ATRISK neighbour iterations (two erf each)     */
    int64_t hop_iters;   /* second-hop and REACH-k step neighbour pairs    */
    int64_t fp64_ops;    /* op-model total, see above                      */
} sidr_counts;
sidr_status sidr_batch_set_counting(sidr_batch* b, int enable);
sidr_status sidr_batch_counts(sidr_batch* b, sidr_counts* out);

/* Block shape of a batch's launches (no reference counterpart).  Shape 0 (the
 * default) budgets 128 registers per thread for 4 resident blocks of 4 warps
 * per SM; shape 1 budgets 96 for 5, which hides more latency at the price of
 * spills and pays on rules that spend their time in ATRISK.  Shapes 0 and 1
 * run one (rule, scenario) pair per warp, shapes 2 and 3 (the same register
 * budgets) two pairs per warp, 16 lanes each, which keeps more lanes busy
 * when decisions have few candidates.  All give the same scores
 * (the reference runs one thread per pair, engine/factory.cuh:42-61; these
 * are the other end of the range).  sidr_batch_autotune_sampled times each shape on every
 * stride-th rule of the batch (all its scenarios; the first of reps + 1 runs
 * warms up), keeps the faster for sidr_batch_run and reports it in *chosen and
 * the times in ms[SIDR_BATCH_SHAPES] (either may be null).  The sampled rules'
 * scores are overwritten; run the batch afterwards.  The counting launch
 * always uses shape 0. */
#define SIDR_BATCH_SHAPES 4
sidr_status sidr_batch_set_shape(sidr_batch* b, int32_t shape);
/* The block shape of a context's sidr_evaluate* calls (default 0). */
sidr_status sidr_ctx_set_shape(sidr_ctx* ctx, int32_t shape);
sidr_status sidr_batch_autotune_sampled(sidr_batch* b, int32_t reps, int32_t stride,
                                        int32_t* chosen, float* ms);

/* Multi-instance batches (no reference counterpart; the reference evaluates
 * one instance per FactoryContext).  K instances of uneven size, each with its
 * own rules, scenarios and mask, evaluated together in ONE persistent launch:
 * rule p belongs to instance rule_instance[p], reads the [T][n_k] scenario
 * block at sampled + sampled_offsets[k] (in doubles; the flat host buffer
 * holds n_sampled doubles) and mask row k of masks [K][61]; out[p*T + s].
 * Rules are grouped by the size class of their instance (SIDR_SIZE_CLASSES:
 * n <= 32, n <= 64, n <= 128, larger); each non-empty class is one launch,
 * with a block shape of its own, and within a class work is handed out
 * longest-estimated-rule first.  Block shapes compiled in (warps per block x
 * minimum resident blocks per SM x lanes per pair): 0: 4x3x32, 1: 8x2x32,
 * 2: 2x6x32, 3: 4x3x16, 4: 4x3x8; 16 and 8 lanes per pair run 2 and 4 pairs
 * per warp, for small instances whose decisions have few candidates.
 * sidr_multi_autotune times each shape on this batch (every class at that
 * shape; reps runs, best time), keeps the fastest and remembers the choice
 * for batches of the same layout (instances' sizes, rule and scenario
 * counts, program sizes, SM count) in this process; ms[] (may be NULL)
 * receives each shape's time, *chosen its index.  sidr_multi_capture records
 * the launches (counter reset + kernel per class) as a CUDA graph that
 * sidr_multi_run then replays. */
typedef struct sidr_multi sidr_multi;
#define SIDR_MULTI_SHAPES 5
#define SIDR_SIZE_CLASSES 4
sidr_status sidr_multi_create(const sidr_instance_desc* insts, const double* zps, int32_t K,
                              const sidr_rules_desc* rules, const int32_t* rule_instance,
                              const double* sampled, int64_t n_sampled,
                              const int64_t* sampled_offsets, int32_t T, const int64_t* masks,
                              int32_t device, sidr_multi** out);
sidr_status sidr_multi_autotune(sidr_multi* m, int32_t reps, int32_t* chosen, float* ms);
/* The same choice made on a sample of the batch: each shape is timed on every
 * stride-th rule of the longest-first work order (all T scenarios), so that
 * the sample keeps the batch's mix of instance sizes and rule costs and the
 * tuning of a full-size batch takes about 1/stride of a launch per shape. */
sidr_status sidr_multi_autotune_sampled(sidr_multi* m, int32_t reps, int32_t stride, int32_t* chosen,
                                        float* ms);
/* A shape per size class, chosen on a sample of the class: each shape runs
 * every stride-th rule of the class's part of the work order (all T
 * scenarios) in one launch; the fastest is kept for that class.
 * chosen[SIDR_SIZE_CLASSES] (may be NULL) receives each class's shape (-1 for
 * a class without rules), ms[SIDR_SIZE_CLASSES * SIDR_MULTI_SHAPES] (may be
 * NULL) the times, ms[c * SIDR_MULTI_SHAPES + shape] (-1 where not timed). */
sidr_status sidr_multi_autotune_classes(sidr_multi* m, int32_t reps, int32_t stride, int32_t* chosen,
                                        float* ms);
/* The same shape for every class (sidr_multi_set_shape) or for one. */
sidr_status sidr_multi_set_shape(sidr_multi* m, int32_t shape);
sidr_status sidr_multi_set_class_shape(sidr_multi* m, int32_t size_class, int32_t shape);
/* Each class's shape and number of rules (either pointer may be NULL). */
sidr_status sidr_multi_shapes(sidr_multi* m, int32_t* shapes, int32_t* class_rules);
sidr_status sidr_multi_capture(sidr_multi* m);
sidr_status sidr_multi_run(sidr_multi* m, void* stream);
sidr_status sidr_multi_read(sidr_multi* m, double* out);
void sidr_multi_destroy(sidr_multi* m);

/* Host-only validation of rules under their masks (no device needed): the
 * checks every evaluate call makes -- opcodes, terminal slots < 61, no stack
 * underflow, stack depth <= SIDR_MAX_STACK, one value left, length <=
 * SIDR_MAX_TREE -- plus compilation into the kernel's programs.  *max_rows
 * (may be NULL) receives the per-lane value rows the largest program needs.
 * No reference counterpart: the reference interpreter does not validate
 * (engine/sim_core.hpp:11-41). */
sidr_status sidr_rules_check(const sidr_rules_desc* rules, const int64_t* masks,
                             int32_t mask_group, int32_t* max_rows);

/* Evaluation that allocates no device memory (no counterpart in the
 * reference).  For callers that cannot call cudaMalloc: code whose device
 * memory belongs to another allocator (a framework's caching pool that must
 * not be bypassed), or that must not pay cudaMalloc/cudaFree's implicit
 * device synchronisation on every call.  Same meaning as
 * sidr_evaluate_grouped_masks, but without a context: the instance, zp,
 * rules, scenarios, masks and out are all HOST buffers, and everything the
 * evaluator keeps on the device -- the instance's lookup tables, the compiled
 * rules, the scenarios, the work-queue counter and the scores before they are
 * copied back -- is placed in one file-scope static device array of
 * SIDR_STATIC_SCRATCH_BYTES, which every GPU that loads the library holds
 * until the process exits.  Limits: n <= SIDR_STATIC_MAX_N, and all of the
 * above must fit the array; larger calls return SIDR_ERR_TOO_LARGE with the
 * sizes in sidr_last_error().  The first call on a device looks up the
 * array's device address there.  All calls in a process share the one array,
 * which keeps the last call's contents; each call clears what must start at
 * zero.  Calls that overlapped on the GPU would race on the array, so each
 * call holds a process-wide lock from its first copy to its last and returns
 * only after the scores are in `out`.  The work runs on a non-blocking
 * stream the library creates once per device (no implicit synchronisation
 * with the caller's legacy-stream work), the caller's current device is
 * restored on return, and the array's device address is kept for the life of
 * the process: a cudaDeviceReset between calls is not supported.  A kernel
 * error word raised during the call returns SIDR_ERR_KERNEL. */
#define SIDR_STATIC_SCRATCH_BYTES (16u << 20)
#define SIDR_STATIC_MAX_N 128
sidr_status sidr_evaluate_static(const sidr_instance_desc* inst, const double zp[10],
                                 const sidr_rules_desc* rules, const double* grouped_sampled,
                                 int32_t G, int32_t T, int32_t group_size, int32_t mask_group,
                                 const int64_t* masks, int32_t device, double* out);

/* Device-side guard check (diagnostic; no reference counterpart).  The
 * evaluator kernel checks each rule record against the shared-memory slice
 * its launch was sized for before staging it; a record that does not fit is
 * refused (its scores become NaN) and the launch raises the kernel error
 * word, which every host path reads back as SIDR_ERR_KERNEL.  Host
 * validation makes that unreachable in normal calls; this entry launches the
 * batch with its slice capacities set to zero, so every rule with at least
 * one instruction is refused.  Expected result: SIDR_ERR_KERNEL, with the
 * batch still usable by sidr_batch_run afterwards. */
sidr_status sidr_batch_guard_check(sidr_batch* b);

/* Number of kernel launches issued by this library since load (evaluator
 * and per-rule fitness kernels). */
int64_t sidr_kernel_launches(void);

/* Host<->device bytes moved by the calling thread's last sidr_evaluate*
 * call (rules, scenarios and masks up; scores down). */
sidr_status sidr_last_transfer_bytes(int64_t* h2d, int64_t* d2h);

/* Measured FP64 pipe throughput of `device`, in operations per second: a
 * kernel of independent double-precision add/multiply chains over every SM
 * (each instruction one operation), best of `reps` timed runs.  The
 * denominator of the evaluator's roofline; no reference counterpart. */
sidr_status sidr_fp64_peak(int device, int reps, double* ops_per_s);

/* The device erf (fn 0), erfc (1) and exp (2) that the evaluator uses for
 * ATRISK's normal CDF and PBUST (engine/sim_terms.hpp:221-223, :571) in place
 * of CUDA's, on host arrays x[n] -> out[n] (diagnostic; no reference
 * counterpart).  They reproduce glibc 2.39's results bit for bit. */
sidr_status sidr_libm_eval(int32_t fn, const double* x, int64_t n, int device, double* out);

/* The device pow that the evaluator uses for rmod (engine/sim_core.hpp:30-35)
 * in place of CUDA's: out[i] = x[i]^y[i] on host arrays (diagnostic; no
 * reference counterpart).  It reproduces glibc 2.39's pow bit for bit. */
sidr_status sidr_libm_pow(const double* x, const double* y, int64_t n, int device, double* out);

#ifdef __cplusplus
}
#endif
#endif
