// sidr_internal.hpp -- shared host/device definitions of the evaluator.
//
// Device-side layout of one instance (built once per context) and of one
// batch of rules x scenarios (built per evaluate call or per sidr_batch).
#pragma once
#include <cstdint>

namespace sidr {

constexpr int kTerms = 61;     // engine/vocab.hpp:16
constexpr int kMaxN = 512;     // engine/vocab.hpp:17
constexpr int kMaxTree = 1024; // engine/vocab.hpp:18
constexpr int kMaxStack = 32;  // engine/vocab.hpp:19
constexpr int kMaxWords = kMaxN / 32;
constexpr double kSigma = 0.2;                // SIM_SIGMA, engine/sim_terms.hpp:15
constexpr double kSqrt2 = 1.4142135623730951; // SQRT2_C, engine/sim_terms.hpp:16
constexpr int kOrdCoincident = 1 << 14;       // flag bit of the sorted neighbour lists

// ----------------------------------------------------------------- instance
//
// Besides the SimData arrays the context keeps lookup tables that turn the
// reference's per-neighbour feasibility arithmetic into one comparison.  For
// origin node o (0 = depot, i+1 = customer i) and customer j, with
// t = dist[o][j+1]:
//
//   F[o*n + j] = the largest double f such that the reference's standard test
//                (arrive = f + t; arrive <= close_j; start = max(arrive, open_j);
//                 start + dur_j + d2d_j <= tmax) passes, or -inf if none does.
//                Every operation in that chain is IEEE round-to-nearest and
//                monotone in f, so the test passes exactly when f <= F.
//   G[o*n + j] = the same for the robust test (service time * (1 + SIM_SIGMA)).
//   R[o*n + j] = scores[j] / (t > 1e-10 ? t : 1e-10): the score-per-time ratio
//                every neighbour scan divides out (same operands, same IEEE
//                division as the reference).
//   zlt / zle  = per origin row, bit j set when t < 1e-10 / !(t > 1e-10):
//                the coincident-location skips of the NS family and of the
//                structural best-neighbour search.
//   P1[c*n + j], P0[j] = pow(var, 0.5) of ATRISK's two variance cases
//                (var = (0.2 d_c)^2 + (0.2 d_j)^2, or 0 + (0.2 d_j)^2),
//                precomputed on the host with the reference's libm; -1 when
//                var <= 1e-18 (the reference's deterministic branch).
//
//   TK[2*(j*n + c)], TC[j*n + c] = ATRISK's classification of the pair
//                (candidate c, customer j) as a step function of the
//                candidate's finish time f: switch points {k0, k1}, interval
//                i = (k_{i-1}, k_i] (unused points +inf) has outcome
//                (TC >> 2i) & 3 -- 0: the term is +0, 1: it is s_j, 2: the
//                kernel classifies the pair itself (a factor needs erf).  Every test of the
//                classification is monotone in f, so the outcome changes only
//                at their switch points, found by bisection on the host.
//
// Two further layouts of the same values serve the two access patterns:
//   * neighbour-major pair tables FR = {F, R} and GD = {G, dist[o][j+1]} at
//     pair index j*ld + o, and DP = {dist[c+1][j+1], P1[c*n + j]} at pair
//     index j*n + c: in the fused candidate scan and in ATRISK all lanes
//     visit the same neighbour j from different origins, so one warp's
//     16-byte loads stay in one row (ATRISK reads both of its per-pair values
//     with one load), and CU = {close, open, P0, dur, d2d, score} per customer
//     (three 16-byte loads for the per-customer values ATRISK's pairs read);
//   * per-origin neighbour lists ord[o*ns + k] sorted by (R desc, index asc),
//     rows padded to ns = a multiple of 4, with sF/sG (F and G in that order),
//     bit 14 of ord marking coincident locations, and cnt_pos[o] / cnt_gm1[o]
//     = the number of leading entries whose ratio exceeds 0 / -1: a greedy
//     "best feasible neighbour by ratio" search -- strict > over ascending
//     index from an initial best of 0 or -1, as in REACH2's second hop and
//     REACH-k -- returns the first feasible entry among those, so it stops
//     early.  bF / bG hold, per row and chunk of 4 entries, {the largest sF
//     / sG of the chunk, the largest of the chunk and every later one}: a
//     search at time tm skips a chunk whose largest threshold is below tm
//     (no entry of it passes tm <= threshold) and stops at a chunk whose
//     suffix maximum is.
struct DevInst {
    int n, m, ld, nw;
    double tmax;
    const double *scores, *durations, *open_t, *close_t, *d2d, *dist;
    const double *F, *G, *R, *P1, *P0;
    const uint32_t *zlt, *zle;
    const double *FR, *GD, *DP;   // interleaved pairs
    const double* CU;              // [n][6] per-customer pack
    const double* TK;              // [n][n][2] ATRISK's step functions at j*n + c: switch points
    const uint8_t* TC;             // [n][n] and outcome codes
    int ns;                        // sorted-list row stride
    const int16_t* ord;
    const double *sF, *sG;
    const double *bF, *bG;         // [ld][ns/4] {chunk max, suffix max}
    const int32_t *cnt_pos, *cnt_gm1;
    const double* zp;  // [10]
};

// ------------------------------------------------------------ rule programs
//
// Each postfix rule is compiled on the host into three-address instructions
// over per-lane value rows held in shared memory: rows [0, K) hold the rule's
// terminals (only the slots it reads), rows [K, K+D) its stack temporaries.
// An operand is 10 bits: bit 9 set = constant-pool index, else a row.
//   word = op | a << 3 | b << 13 | dst << 23
constexpr uint32_t kOpConst = 512u;

enum NeedBits : uint32_t {
    kNeedNS = 1u << 0,       // NS value (slots 10, 28, 29)
    kNeedRegret = 1u << 1,   // 11 (33, 43)
    kNeedNSRob = 1u << 2,    // 12 (45, 46)
    kNeedMaxN = 1u << 3,     // 13
    kNeedReach2 = 1u << 4,   // 14 (32)
    kNeedNSTW = 1u << 5,     // 15
    kNeedStruct = 1u << 6,   // 17-19, 28, 29 (FRAGCNT, FRAGSCORE, DOWNSLACK)
    kNeedPBust = 1u << 7,    // 20
    kNeedReachK = 1u << 8,   // 21-23 (steps in reach_k)
    kNeedAtRisk = 1u << 9,   // 30 (34)
    kNeedReach2Rob = 1u << 10, // 41 (43)
    kNeedAgg = 1u << 11,     // VFRAC, NFEAS (25, 26)
    kNeedFScore = 1u << 12,  // FEASCORE (51)
    kNeedNFeasRob = 1u << 13, // NFEASROB (52)
    kNeedExplore = 1u << 14, // slots computed by the direct per-lane path
    kNeedRmod = 1u << 15,    // the program has rmod instructions (opcode 6)
    kNeedNSFused = kNeedNS | kNeedMaxN | kNeedReach2 | kNeedNSTW,
    kNeedRob = kNeedNSRob | kNeedReach2Rob,
    kNeedAfterC = kNeedStruct | kNeedPBust | kNeedReachK,
};

// Counters of the counting instantiation: decisions, candidates, fused-scan
// neighbours, ATRISK neighbours, second-hop/REACH-step neighbours, op model.
constexpr int kStats = 6;
// Op-model constants (see sidr_counts in include/sidr.h).
constexpr int kOpsTest = 7;       // one neighbour feasibility test incl. the skip
constexpr int kOpsAtRisk = 40;    // ATRISK neighbour: 2 div, 2 erf (15 each), 8 more
constexpr int kOpsHop = 8;        // second-hop / REACH-k step neighbour
constexpr int kOpsCandidate = 12; // candidate setup (ta .. sd_c)

struct RuleMeta {
    int32_t prog_off;   // first instruction word
    int32_t const_off;  // first constant
    int32_t slot_off;   // first compact-slot byte
    int16_t n_ins;      // instructions
    int16_t n_const;    // constants
    int16_t K;          // terminal rows
    int16_t D;          // temporary rows
    int16_t res;        // result operand
    int8_t reach_k;     // deepest REACH-k step needed (0, 1, 3, 5)
    uint16_t scan_ops;  // op-model cost of one fused-scan neighbour (counting only)
    int16_t inst;       // instance of a multi-instance batch (0 otherwise)
    uint32_t need;      // NeedBits
    uint64_t explore;   // bit s set: exploration slot s is read
};

struct DevBatch {
    int P, T, group_size, n;
    const uint32_t* prog;
    const double* consts;
    const uint8_t* slots;
    const RuleMeta* meta;
    const double* sampled;  // [G][T][n]
    double* out;            // [P][T]
    unsigned long long* counter;  // work-queue head
    unsigned long long* stats;    // [kStats] counters (may be null)
    int* error;                   // kernel error word
    int rows, prog_cap, const_cap;  // per-warp shared-memory sizing
    // Multi-instance batches: per-instance descriptors, scenario block offsets
    // (doubles; instance k's [T][n_k] block starts at sampled + smp_off[k]), and
    // the order in which rules are handed out (null = index order).
    const DevInst* insts;
    const int64_t* smp_off;
    const int32_t* order;
    int n_inst;   // descriptors at insts
    int P_items;  // rules in the work queue (0: all P); with `order`, a sample of the batch
};

// Codes of the kernel error word (DevBatch::error); the host turns a nonzero
// word into SIDR_ERR_KERNEL.  The first code raised in a launch is kept.
constexpr int kErrRuleRecord = 1;  // a rule record exceeds the launch's shared-memory slice
constexpr int kErrRuleIndex = 2;   // a work item names a rule outside the batch
constexpr int kErrInstance = 3;    // a rule names an instance outside the batch

// Decision-situation capture (capture_kernel only): for scenario s and its
// d-th decision (d < dec), candidate c (< cand) -> its k terminal rows at
// rows[((s*dec + d)*cand + c)*k] and its customer at cust[(s*dec + d)*cand + c];
// info[(s*dec + d)*2] = {candidates, chosen customer (-1: none)}.
struct CaptureBuf {
    double* rows;
    int32_t* cust;
    int32_t* info;
    int dec, cand, k;
};

}  // namespace sidr
