// sidr_kernel.cuh -- the B200 rule x scenario evaluator kernel.
//
// Mapping (one persistent launch):
//   * one warp simulates one (rule, scenario) pair at a time and pulls the
//     next pair from a global work queue (pairs ordered rule-major, so a warp
//     usually keeps its rule's program staged in shared memory);
//   * at each decision point (engine/sim_core.hpp:43-204, pick_best) the warp
//     builds the feasible-candidate bitmask with one ballot per 32 customers,
//     compacts it, and spreads the candidates over its lanes, 32 per round;
//   * each lane computes its candidate's terminals with fused neighbour scans
//     (every terminal's sum still runs over j in ascending order, so each
//     accumulator sees the reference's operation sequence), evaluates the rule
//     program from shared memory, and the warp picks the best candidate with
//     shuffles (strict >, lowest index on ties, NaN -> -1e300: :199-201);
//   * the route state (visited bitmask, position, clock, collected score) is
//     warp-uniform; the rollout order is sim_one's (:207-238).
//
// Bit-exactness: compiled with -fmad=false; every floating-point expression
// keeps the reference's operand order.  The lookup tables of DevInst replace
// only comparisons whose outcome they reproduce exactly (see sidr_internal.hpp)
// and divisions with identical operands.
#pragma once
#include <cuda_runtime.h>

#include "sidr_internal.hpp"
#include "sidr_libm.cuh"

namespace sidr {

constexpr unsigned kFull = 0xffffffffu;

// The lanes that simulate one (rule, scenario) pair: the whole warp
// (LPP = 32) or a group of 16 or 8 lanes, so that a warp runs 2 or 4 pairs
// side by side.  Small instances have few candidates per decision, and a
// group that matches them keeps more lanes busy.  Every collective of the
// pair's simulation (ballots, shuffles, syncs) names only its group's lanes;
// with LPP = 32 they are the plain full-warp forms.
template <int LPP>
struct Group {
    static_assert(LPP == 32 || LPP == 16 || LPP == 8, "lanes per pair: 32, 16 or 8");
    static constexpr int kPerWarp = 32 / LPP;
    // lane within the group
    __device__ __forceinline__ static int lane() { return (int)(threadIdx.x & (LPP - 1)); }
    // the group's place in its warp
    __device__ __forceinline__ static int index() { return (int)((threadIdx.x & 31) / LPP); }
    __device__ __forceinline__ static int first() { return (int)((threadIdx.x & 31) & ~(LPP - 1)); }
    __device__ __forceinline__ static unsigned mask() {
        if constexpr (LPP == 32) return kFull;
        else return ((1u << LPP) - 1u) << first();
    }
    __device__ __forceinline__ static void sync() {
        if constexpr (LPP == 32) __syncwarp();
        else __syncwarp(mask());
    }
    // the group's predicate bits, bit k = group lane k
    __device__ __forceinline__ static uint32_t ballot(bool p) {
        if constexpr (LPP == 32) return __ballot_sync(kFull, p);
        else return __ballot_sync(mask(), p) >> first();
    }
    template <class T>
    __device__ __forceinline__ static T shfl_xor(T v, int off) {
        return __shfl_xor_sync(mask(), v, off);
    }
    // v of group lane src
    template <class T>
    __device__ __forceinline__ static T shfl(T v, int src) {
        return __shfl_sync(mask(), v, first() + src);
    }
};

// Block shape of the evaluator: warps per block and the minimum resident
// blocks per SM that bound its registers (__launch_bounds__).  The kernel is
// latency-bound (dependent FP64 chains and L1-missing table loads), so 16
// warps per SM at 128 registers, with a few spills, beat 12 at 168 and 20 at
// 96 (measured on gp-generation and evolved populations).
#ifndef SIDR_WARPS_PER_BLOCK
#define SIDR_WARPS_PER_BLOCK 4
#endif
#ifndef SIDR_MIN_BLOCKS
#define SIDR_MIN_BLOCKS 4
#endif

// Section-cycle hooks for profiling builds only (-DSIDR_SECTION_CLOCKS): the
// first active lane of each warp adds the cycles spent in a section to
// sidr_section_cycles[].  In normal builds they compile to nothing.
#ifdef SIDR_SECTION_CLOCKS
__device__ unsigned long long sidr_section_cycles[16];
#define SIDR_SEC_MARK(var)      \
    __syncwarp(__activemask()); \
    const long long var = clock64();
#define SIDR_SEC_ADD(idx, var)                                                             \
    do {                                                                                   \
        const unsigned am_ = __activemask();                                               \
        __syncwarp(am_);                                                                   \
        if ((threadIdx.x & 31) == __ffs(am_) - 1)                                          \
            atomicAdd(&sidr_section_cycles[idx], (unsigned long long)(clock64() - (var))); \
    } while (0)
#else
#define SIDR_SEC_MARK(var)
#define SIDR_SEC_ADD(idx, var)
#endif

// Shared-memory slice of one pair group (a warp when LPP = 32).
struct WarpSmem {
    DevInst* inst;     // the rule's instance (multi-instance batches)
    double* rows;      // [rows][LPP]; between rounds also ATRISK's erf queue
    double* cst;       // [const_cap]
    uint32_t* prog;    // [prog_cap]
    int16_t* cand;     // [kMaxN]
    uint32_t* unv;     // [kMaxWords] unvisited customers
    uint32_t* feas;    // [kMaxWords] feasible-now & unvisited
    uint32_t* atr;     // [kMaxWords] ATRISK's arrive-by-close filter
    uint8_t* slots;    // [64] compact row -> terminal slot
    int qcap;          // doubles in the ATRISK queue (carved rows * LPP)
};

__host__ __device__ inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// A copy of the current rule's instance descriptor (multi-instance batches)
// closes every warp's slice.
constexpr size_t kInstBytes = (sizeof(DevInst) + 15) / 16 * 16;

// The value rows double as ATRISK's queue of erf arguments, which runs
// before a round's terminals are written: at least kQueueRows rows
// (kQueueRows * 16 queue entries of two doubles) are carved.
constexpr int kQueueRows = 16;

__host__ __device__ inline int carved_rows(int rows) { return rows < kQueueRows ? kQueueRows : rows; }

// Bytes of one group's slice; a block of W warps takes W * (32 / lpp) of them.
__host__ __device__ inline size_t warp_slice_bytes(int rows, int const_cap, int prog_cap, int lpp = 32) {
    size_t b = kInstBytes;
    b += (size_t)carved_rows(rows) * lpp * sizeof(double);
    b += (size_t)const_cap * sizeof(double);
    b += align_up((size_t)prog_cap * sizeof(uint32_t), 8);
    b += (size_t)kMaxN * sizeof(int16_t);
    b += 3 * kMaxWords * sizeof(uint32_t);
    b += 64;
    return align_up(b, 16);
}

__device__ __forceinline__ WarpSmem carve(unsigned char* base, int rows, int const_cap,
                                          int prog_cap, int lpp = 32) {
    WarpSmem s;
    s.inst = reinterpret_cast<DevInst*>(base);
    base += kInstBytes;
    s.rows = reinterpret_cast<double*>(base);
    s.cst = s.rows + (size_t)carved_rows(rows) * lpp;
    s.prog = reinterpret_cast<uint32_t*>(s.cst + const_cap);
    s.cand = reinterpret_cast<int16_t*>(
        reinterpret_cast<unsigned char*>(s.prog) + align_up((size_t)prog_cap * 4, 8));
    s.unv = reinterpret_cast<uint32_t*>(s.cand + kMaxN);
    s.feas = s.unv + kMaxWords;
    s.atr = s.feas + kMaxWords;
    s.slots = reinterpret_cast<uint8_t*>(s.atr + kMaxWords);
    s.qcap = carved_rows(rows) * lpp;
    return s;
}

// ------------------------------------------------------------ small helpers

__device__ __forceinline__ double sel_max(double a, double b) { return a > b ? a : b; }

// The reference's standard neighbour test, evaluated directly
// (engine/sim_terms.hpp loop bodies); used by the exploration terminals.
__device__ __forceinline__ bool fits_std(const DevInst& I, int j, double arrive) {
    if (arrive > I.close_t[j]) return false;
    const double st = arrive > I.open_t[j] ? arrive : I.open_t[j];
    return !(st + I.durations[j] + I.d2d[j] > I.tmax);
}

__device__ __forceinline__ bool fits_scaled(const DevInst& I, int j, double arrive, double mul) {
    if (arrive > I.close_t[j]) return false;
    const double st = arrive > I.open_t[j] ? arrive : I.open_t[j];
    return !(st + I.durations[j] * mul + I.d2d[j] > I.tmax);
}

__device__ __forceinline__ bool is_unvisited(const WarpSmem& S, int j) {
    return (S.unv[j >> 5] >> (j & 31)) & 1u;
}

__device__ __forceinline__ uint32_t bit_in_word(int node, int w) {
    return (node >= 0 && (node >> 5) == w) ? (1u << (node & 31)) : 0u;
}

// The sorted neighbour lists are read four entries at a time: a 32-byte
// chunk of thresholds and an 8-byte chunk of four indices.
struct Chunk4 {
    double t[4];
    int q[4];
};

__device__ __forceinline__ Chunk4 load_chunk(const double* sT, const int16_t* ord, int k) {
    Chunk4 c;
    const double2 t01 = *reinterpret_cast<const double2*>(sT + k);
    const double2 t23 = *reinterpret_cast<const double2*>(sT + k + 2);
    const uint2 qq = *reinterpret_cast<const uint2*>(ord + k);
    c.t[0] = t01.x; c.t[1] = t01.y; c.t[2] = t23.x; c.t[3] = t23.y;
    c.q[0] = (int)(qq.x & 0xffffu);
    c.q[1] = (int)(qq.x >> 16);
    c.q[2] = (int)(qq.y & 0xffffu);
    c.q[3] = (int)(qq.y >> 16);
    return c;
}

// REACH2's second loop (engine/sim_terms.hpp:112-126, robust :175-189): the
// best unvisited customer outside {x0, x1} by score/time from origin node o at
// time tm, skipping coincident locations, init 0.0.  `table` is sF (standard)
// or sG (robust), `bmax` its chunk maxima bF / bG.  The argmax with strict >
// over ascending index is the first feasible entry among the cnt_pos[o]
// leading entries of o's sorted list (those whose ratio exceeds 0.0); chunks
// whose thresholds are all below tm hold none.  Returns the chosen customer's
// score, or 0.0.
template <bool COUNT>
__device__ double second_hop_score(const DevInst& I, const WarpSmem& S, const double* table,
                                   const double* bmax, int o, double tm, int x0, int x1,
                                   unsigned long long& hops) {
    const size_t row = (size_t)o * I.ns;
    const int16_t* ord = I.ord + row;
    const double* sT = table + row;
    const double2* bm = reinterpret_cast<const double2*>(bmax) + row / 4;
    const int cnt = I.cnt_pos[o];
    double res = 0.0;
    // The scan leaves both loops by flags rather than returning from inside
    // the unrolled body, which keeps the warp's exit point single.
    for (int k = 0; k < cnt; k += 4) {
        const double2 mx = bm[k >> 2];
        if (tm > mx.y) break;
        if (tm > mx.x) continue;
        const Chunk4 c = load_chunk(sT, ord, k);
        bool hit = false;
#pragma unroll
        for (int e = 0; e < 4; e++) {
            if (k + e >= cnt) break;
            if (COUNT) hops++;
            const int q = c.q[e];  // coincident entries keep bit 14 and never match
            if (q < kOrdCoincident && q != x0 && q != x1 && is_unvisited(S, q) && tm <= c.t[e]) {
                res = I.scores[q];
                hit = true;
                break;
            }
        }
        if (hit) break;
    }
    return res;
}

// One REACH-k greedy step (engine/sim_terms.hpp:415-431): the best unvisited
// customer outside the walk by score/max(t,1e-10) under the standard test, no
// coincident skip, init -1.0 -- the first feasible entry among the cnt_gm1[o]
// leading entries of o's sorted list (chunks skipped as in second_hop_score).
// p0..p4: the walk so far (-1 = unused).
template <bool COUNT>
__device__ int reach_step(const DevInst& I, const WarpSmem& S, int o, double tm, int p0, int p1,
                          int p2, int p3, int p4, unsigned long long& hops) {
    const size_t row = (size_t)o * I.ns;
    const int16_t* ord = I.ord + row;
    const double* sF = I.sF + row;
    const double2* bm = reinterpret_cast<const double2*>(I.bF) + row / 4;
    const int cnt = I.cnt_gm1[o];
    int res = -1;
    for (int k = 0; k < cnt; k += 4) {
        const double2 mx = bm[k >> 2];
        if (tm > mx.y) break;
        if (tm > mx.x) continue;
        const Chunk4 c = load_chunk(sF, ord, k);
#pragma unroll
        for (int e = 0; e < 4; e++) {
            if (k + e >= cnt) break;
            if (COUNT) hops++;
            const int q = c.q[e] & (kOrdCoincident - 1);
            if (q != p0 && q != p1 && q != p2 && q != p3 && q != p4 && is_unvisited(S, q) &&
                tm <= c.t[e]) {
                res = q;
                break;
            }
        }
        if (res >= 0) break;
    }
    return res;
}

// ------------------------------------------------- exploration terminals
// Direct restatements for the slots outside the 29-terminal menu
// (engine/sim_terms.hpp:129-154, 259-401, 443-519).  They read the instance
// arrays straight, like the reference, and are used only when a mask enables
// them.

__device__ __noinline__ double x_skiploss(const DevInst& I, const WarpSmem& S, int i, int cur, double ct) {
    const int ld = I.ld;
    double bv = 0.0, fq = 0.0;
    int bq = -1;
    for (int q = 0; q < I.n; q++) {
        if (q == i || !is_unvisited(S, q)) continue;
        const double t = I.dist[(size_t)cur * ld + q + 1];
        if (t < 1e-10) continue;
        const double arrive = ct + t;
        if (arrive > I.close_t[q]) continue;
        const double st = arrive > I.open_t[q] ? arrive : I.open_t[q];
        if (st + I.durations[q] + I.d2d[q] > I.tmax) continue;
        const double v = I.scores[q] / t;
        if (v > bv) {
            bv = v;
            bq = q;
            fq = st + I.durations[q];
        }
    }
    if (bq < 0) return 0.0;
    const double ai = fq + I.dist[(size_t)(bq + 1) * ld + i + 1];
    if (ai > I.close_t[i]) return I.scores[i];
    const double si = ai > I.open_t[i] ? ai : I.open_t[i];
    if (si + I.durations[i] + I.d2d[i] > I.tmax) return I.scores[i];
    return 0.0;
}

__device__ __noinline__ double x_reach_k_rob(const DevInst& I, const WarpSmem& S, int c, double fin_rob_c,
                                int K) {
    const int ld = I.ld;
    int path[6] = {c, -1, -1, -1, -1, -1};
    int at = c + 1;
    double tm = fin_rob_c, tot = 0.0;
    for (int step = 0; step < K; step++) {
        int best = -1;
        double bv = -1.0;
        for (int q = 0; q < I.n; q++) {
            if (!is_unvisited(S, q)) continue;
            bool on = false;
#pragma unroll
            for (int k = 0; k < 6; k++) on |= (path[k] == q);
            if (on) continue;
            const double ta = I.dist[(size_t)at * ld + q + 1];
            if (!fits_scaled(I, q, tm + ta, 1.0 + kSigma)) continue;
            const double tt = ta > 1e-10 ? ta : 1e-10;
            const double v = I.scores[q] / tt;
            if (v > bv) {
                bv = v;
                best = q;
            }
        }
        if (best < 0) break;
        const double arrive = tm + I.dist[(size_t)at * ld + best + 1];
        const double st = arrive > I.open_t[best] ? arrive : I.open_t[best];
        tm = st + I.durations[best] * (1.0 + kSigma);
        at = best + 1;
        tot += I.scores[best];
        path[step + 1] = best;
    }
    return tot;
}

__device__ __noinline__ double x_ns_family(const DevInst& I, const WarpSmem& S, int i, double fin, int kind) {
    // kind 0: NSA2 score/t^2, 1: NSA05 score/sqrt(t), 2: NNFWD, 3: NNK3, 4: SCORERANK
    const int ld = I.ld;
    double acc = 0.0, d1 = -1.0, d2 = -1.0, d3 = -1.0, below = 0.0, tot = 0.0;
    for (int j = 0; j < I.n; j++) {
        if (j == i || !is_unvisited(S, j)) continue;
        const double t = I.dist[(size_t)(i + 1) * ld + j + 1];
        if (t < 1e-10) continue;
        if (!fits_std(I, j, fin + t)) continue;
        if (kind == 0) acc += I.scores[j] / (t * t);
        else if (kind == 1) acc += I.scores[j] / sqrt(t);
        else if (kind == 2) {
            if (d1 < 0.0 || t < d1) d1 = t;
        } else if (kind == 3) {
            if (d1 < 0.0 || t < d1) {
                d3 = d2;
                d2 = d1;
                d1 = t;
            } else if (d2 < 0.0 || t < d2) {
                d3 = d2;
                d2 = t;
            } else if (d3 < 0.0 || t < d3) {
                d3 = t;
            }
        } else {
            tot += 1.0;
            if (I.scores[j] < I.scores[i]) below += 1.0;
        }
    }
    if (kind <= 1) return acc;
    if (kind == 2) return d1 < 0.0 ? 0.0 : 1.0 / (1.0 + d1);
    if (kind == 3) {
        if (d1 < 0.0) return 0.0;
        double s = d1, k = 1.0;
        if (d2 >= 0.0) {
            s += d2;
            k += 1.0;
        }
        if (d3 >= 0.0) {
            s += d3;
            k += 1.0;
        }
        return 1.0 / (1.0 + s / k);
    }
    if (tot == 0.0) return 1.0;
    return below / tot;
}

__device__ __noinline__ double x_ns_rob_m(const DevInst& I, const WarpSmem& S, int i, double fin, double m) {
    const int ld = I.ld;
    const double ms = m * kSigma;
    const double frob = fin + I.durations[i] * ms;
    double acc = 0.0;
    for (int j = 0; j < I.n; j++) {
        if (j == i || !is_unvisited(S, j)) continue;
        const double t = I.dist[(size_t)(i + 1) * ld + j + 1];
        if (t < 1e-10) continue;
        if (!fits_scaled(I, j, frob + t, 1.0 + ms)) continue;
        acc += I.scores[j] / t;
    }
    return acc;
}

__device__ __noinline__ double x_nnchain(const DevInst& I, const WarpSmem& S, int c, double fin_c, int K) {
    const int ld = I.ld;
    int path[4] = {c, -1, -1, -1};
    int at = c + 1, done = 0;
    double tm = fin_c, tot = 0.0;
    for (int step = 0; step < K; step++) {
        int best = -1;
        double bd = -1.0;
        for (int q = 0; q < I.n; q++) {
            if (!is_unvisited(S, q)) continue;
            bool on = false;
#pragma unroll
            for (int k = 0; k < 4; k++) on |= (path[k] == q);
            if (on) continue;
            const double ta = I.dist[(size_t)at * ld + q + 1];
            if (ta < 1e-10) continue;
            if (!fits_std(I, q, tm + ta)) continue;
            if (bd < 0.0 || ta < bd) {
                bd = ta;
                best = q;
            }
        }
        if (best < 0) break;
        const double arrive = tm + bd;
        const double st = arrive > I.open_t[best] ? arrive : I.open_t[best];
        tm = st + I.durations[best];
        at = best + 1;
        tot += bd;
        done++;
        if (step + 1 < 4) path[step + 1] = best;
    }
    if (done == 0) return 0.0;
    return 1.0 / (1.0 + tot / done);
}

__device__ __noinline__ double x_detour(const DevInst& I, const WarpSmem& S, int i, int cur, double fin,
                           double ta_i) {
    const int ld = I.ld;
    double tot = 0.0, cnt = 0.0;
    for (int j = 0; j < I.n; j++) {
        if (j == i || !is_unvisited(S, j)) continue;
        const double t = I.dist[(size_t)(i + 1) * ld + j + 1];
        if (t < 1e-10) continue;
        if (!fits_std(I, j, fin + t)) continue;
        tot += ta_i + t - I.dist[(size_t)cur * ld + j + 1];
        cnt += 1.0;
    }
    if (cnt == 0.0) return 0.0;
    return tot / cnt;
}

__device__ __forceinline__ double t_rand_dev(int i) {
    long long x = (((long long)i + 1) * 1103515245LL + 12345LL) & 0x7FFFFFFFLL;
    x = (x * 1103515245LL + 12345LL) & 0x7FFFFFFFLL;
    return (double)(x % 100000LL) / 1000.0;
}

// -------------------------------------------------------- decision context

struct Decision {
    int cur, remaining;
    double ct, sat, vfrac, nfeas, fscore, nfeasrob;
};

// Counters of one warp (COUNT instantiation only).
struct WarpCounts {
    unsigned long long dec, cand, scan, heavy, hop, ops;
};

// What the ATRISK pass of one lane reads, as plain values (held in registers
// across the out-of-line call): the per-customer pack CU, the scores, the
// candidate's column of DP, the decision's customer set and the erf queue in
// shared memory, and the candidate's mean finish and deviation.
struct AtRiskView {
    const double2* CU;      // per customer {close, open}, {P0, dur}, {d2d, score}
    const double* scores;
    const double2* DP;      // {dist(c, j), P1(c, j)} at j * n + c
    const double2* DPc;     // DP + ci
    const double2* TKc;     // TK + ci: the step functions' switch points {k0, k1} at j * n
    const uint8_t* TCc;     // TC + ci: their outcome codes at j * n
    const uint32_t* atr;
    double* Q;
    int n, nw, cap, ci;
    double tmax, fin_c, sd_c;
};

// One (candidate, customer) pair of ATRISK, classified without branches.  The
// term is sj * (1 - p_win * p_bud).  A normal-CDF factor whose argument lies
// at least 8.5 standard deviations from the mean is exactly 0 or 1 -- the
// reference's erf (glibc) returns +-1 for |x| >= 6, and |d| >= 8.5 s gives
// x >= 6.01 after both roundings -- and so is one whose deviation is
// degenerate.  When both factors are exact the term is sj (a product of 0)
// or +0 (a product of 1, which leaves the sum unchanged); p_bud is not
// needed when p_win is exactly 0.  Only the rest (about 5% of pairs on the
// benchmark workloads) need erf of (num / den) * 1/sqrt(2): ew / eb.
struct AtRiskClass {
    bool add;        // both factors exact and the term is sj
    bool ew, eb;     // p_win / p_bud need erf (p_win is otherwise exactly 1 when eb)
    bool pb1;        // p_bud exactly 1 (when ew and not eb)
    double wnum;     // p_win's numerator (denominator sd_c)
    double bnum, bden;
};

// The four 16-byte loads of pair (candidate, j): {dist(c, j), P1(c, j)} and
// the customer's {close, open}, {P0, dur}, {d2d, score}.
struct AtRiskLoad {
    double2 dp, co, pd, es;
};

__device__ __forceinline__ AtRiskLoad at_risk_load(const AtRiskView& v, int j, bool live) {
    const int js = live ? j : 0;
    const double2* cu = v.CU + 3 * (size_t)js;
    AtRiskLoad L;
    L.dp = v.DPc[(size_t)js * v.n];
    L.co = cu[0];
    L.pd = cu[1];
    L.es = cu[2];
    return L;
}

__device__ __forceinline__ AtRiskClass at_risk_compute(const AtRiskView& v, const AtRiskLoad& L,
                                                       bool live, double hw, double lw) {
    const double2 dp = L.dp, co = L.co, pd = L.pd, es = L.es;
    const double cj = co.x, oj = co.y, p0 = pd.x, dj = pd.y, ej = es.x;
    const double marr = v.fin_c + dp.x;
    const double dw = cj - marr;
    const bool sdv = v.sd_c > 1e-9;
    const bool ew = sdv && !(dw >= hw) && !(dw <= lw);
    const bool pw1 = sdv ? dw >= hw : marr <= cj;  // p_win exactly 1, when not ew
    const bool late = marr > oj;
    const double mst = late ? marr : oj;
    const double pv = late ? dp.y : p0;
    const double mb = mst + dj + ej;
    const double db = v.tmax - mb;
    const bool pvv = pv >= 0.0;
    const double hb = 8.5 * pv, lb = -8.5 * pv;
    const bool eb = (ew || pw1) && pvv && !(db >= hb) && !(db <= lb);
    AtRiskClass c;
    c.pb1 = pvv ? db >= hb : mb <= v.tmax;
    c.ew = live && ew;
    c.eb = live && eb;
    c.add = live && !ew && !eb && !(pw1 && c.pb1);
    c.wnum = dw;
    c.bnum = db;
    c.bden = pv;
    return c;
}

__device__ __forceinline__ AtRiskClass at_risk_class(const AtRiskView& v, int j, bool live,
                                                     double hw, double lw) {
    return at_risk_compute(v, at_risk_load(v, j, live), live, hw, lw);
}

__device__ __forceinline__ double norm_cdf_ratio(double num, double den) {
    return 0.5 * (1.0 + libm::erf_((num / den) * 0.7071067811865476));
}

// ATRISK (t_eloss_chance, engine/sim_terms.hpp:225-257) of each lane's
// candidate v.ci (-1: the lane has none), called by the whole warp at the
// start of a scoring round.  The reference adds the terms of the unvisited
// customers j != ci that can still be reached before their close in
// ascending j; that set (S.atr) is the decision's, so every lane walks the
// same list, the per-customer loads are broadcasts and the lanes' pair loads
// fall in one row of DP.  The list is taken 32 customers (one word) at a
// time.  Pass 1 classifies the word's pairs, one per step with the next
// pair's loads already issued, into per-lane bit masks, and queues the (numerator,
// denominator) of every erf argument warp-wide in the value rows; the warp
// evaluates the queue 32 entries at a time; pass 2 adds the terms in order
// from the masks, the word's scores (one per lane, shuffled) and the queue
// (positions from the same ballots).  A word whose arguments overflow the
// queue is added by at_risk_word_direct.  The "warp" above is the pair's
// group of LPP lanes.
template <bool COUNT, int LPP = 32>
__device__ __noinline__ double at_risk(const AtRiskView v, WarpCounts& wc);

// The pairs of word w of the customer set in ascending order, one at a
// time with erf inline: the path of a word whose erf arguments overflow the
// queue.  Returns eloss with the word's terms added.
__device__ __noinline__ double at_risk_word_direct(const AtRiskView v, int w, uint32_t word,
                                                   double eloss) {
    const double hw = 8.5 * v.sd_c, lw = -8.5 * v.sd_c;
    for (uint32_t bits = word; bits;) {
        const int j = (w << 5) + __ffs(bits) - 1;
        bits &= bits - 1;
        if (v.ci < 0 || j == v.ci) continue;
        const AtRiskClass c = at_risk_class(v, j, true, hw, lw);
        const double sj = v.scores[j];
        if (c.add) {
            eloss += sj;
        } else if (c.ew || c.eb) {
            const double fw = c.ew ? norm_cdf_ratio(c.wnum, v.sd_c) : 1.0;
            const double fb = c.eb ? norm_cdf_ratio(c.bnum, c.bden) : (c.pb1 ? 1.0 : 0.0);
            eloss += sj * (1.0 - fw * fb);
        }
    }
    return eloss;
}

template <bool COUNT, int LPP>
__device__ __noinline__ double at_risk(const AtRiskView v, WarpCounts& wc) {
    using G = Group<LPP>;
    const int lane = G::lane();
    const uint32_t lt = (1u << lane) - 1u;
    const bool has = v.ci >= 0;
    // the value rows: terms of the pairs classified in full, then their entries
    double* const T = v.Q;
    int* const QE = reinterpret_cast<int*>(v.Q + v.cap);
    double eloss = 0.0;
    unsigned long long heavy = 0;

    for (int w = 0; w < v.nw; w++) {
        const uint32_t word = v.atr[w];
        if (word == 0) continue;
        const uint32_t own = has ? bit_in_word(v.ci, w) : 0u;
        if (COUNT && has) heavy += __popc(word & ~own);
        G::sync();  // the previous word's reads of T are done
        SIDR_SEC_MARK(t_p1)
        // pass 1: each pair's outcome from its step function at the candidate's
        // finish time, one pair per step with the next pair's loads issued
        // first; the pairs whose outcome needs the full classification are
        // queued (customer bit, lane) in (customer, lane) order
        uint32_t addm = 0, fullm = 0;
        int qn = 0;
        const double f = v.fin_c;
        int bc = __ffs(word) - 1;
        uint32_t bits = word & (word - 1);
        bool lc = has && !((own >> bc) & 1u);
        size_t rc = (size_t)(lc ? (w << 5) + bc : 0) * v.n;
        double2 ka = v.TKc[rc];
        int kc = v.TCc[rc];
        for (;;) {
            const bool more = bits != 0;  // group-uniform
            const int bn = more ? __ffs(bits) - 1 : bc;
            bits &= bits - 1;
            const bool ln = has && !((own >> bn) & 1u);
            const size_t rn = (size_t)(ln ? (w << 5) + bn : 0) * v.n;
            const double2 na = v.TKc[rn];
            const int nc = v.TCc[rn];
            const int iv = (f > ka.x) + (f > ka.y);
            const int code = lc ? (kc >> (2 * iv)) & 3 : 0;
            const uint32_t m = 1u << bc;
            addm |= code == 1 ? m : 0u;
            const bool full = code == 2;
            fullm |= full ? m : 0u;
            const uint32_t bf = G::ballot(full);
            const int pos = qn + __popc(bf & lt);
            qn += __popc(bf);
            if (full && pos < v.cap) QE[pos] = (bc << 8) | lane;
            if (!more) break;
            bc = bn;
            lc = ln;
            ka = na;
            kc = nc;
        }
        SIDR_SEC_ADD(11, t_p1);
        if (qn > v.cap) {  // group-uniform
            eloss = at_risk_word_direct(v, w, word, eloss);
            continue;
        }
        SIDR_SEC_MARK(t_q)
        // the queued pairs, LPP at a time with every lane busy: the owner's
        // finish time and deviation come by shuffle, the term (s_j, +0 or
        // s_j (1 - p_win p_bud) with erf) goes to T in queue order
        if (qn) {
            G::sync();
            for (int base = 0; base < qn; base += LPP) {
                const int k = base + lane;
                const bool valid = k < qn;
                const int e = valid ? QE[k] : 0;
                const int owner = e & 31;
                const double fin = G::shfl(v.fin_c, owner), sd = G::shfl(v.sd_c, owner);
                const int ci = G::shfl(v.ci, owner);
                if (valid) {
                    const int j = (w << 5) + (e >> 8);
                    const double2* cu = v.CU + 3 * (size_t)j;
                    AtRiskLoad L;
                    L.dp = v.DP[(size_t)j * v.n + ci];
                    L.co = cu[0];
                    L.pd = cu[1];
                    L.es = cu[2];
                    AtRiskView o = v;
                    o.fin_c = fin;
                    o.sd_c = sd;
                    const AtRiskClass c = at_risk_compute(o, L, true, 8.5 * sd, -8.5 * sd);
                    const double sj = L.es.y;
                    double term = 0.0;
                    if (c.add) {
                        term = sj;
                    } else if (c.ew || c.eb) {
                        const double fw = c.ew ? norm_cdf_ratio(c.wnum, sd) : 1.0;
                        const double fb = c.eb ? norm_cdf_ratio(c.bnum, c.bden) : (c.pb1 ? 1.0 : 0.0);
                        term = sj * (1.0 - fw * fb);
                    }
                    T[k] = term;
                }
            }
            G::sync();
        }
        SIDR_SEC_ADD(12, t_q);
        SIDR_SEC_MARK(t_p2)
        // pass 2: the terms in ascending customer order, each lane its own sum
        // (a +0 term leaves it unchanged)
        const int jl = (w << 5) + lane;
        const double sw = (LPP == 32 && jl < v.n) ? v.scores[jl] : 0.0;
        qn = 0;
        for (uint32_t bits2 = word; bits2;) {
            const int b = __ffs(bits2) - 1;
            bits2 &= bits2 - 1;
            const uint32_t m = 1u << b;
            double sj;
            if constexpr (LPP == 32) sj = __shfl_sync(kFull, sw, b);
            else sj = v.scores[(w << 5) + b];
            const bool full = (fullm & m) != 0;
            const uint32_t bf = G::ballot(full);
            const int pos = qn + __popc(bf & lt);
            qn += __popc(bf);
            if (addm & m) eloss += sj;
            else if (full) eloss += T[pos];
        }
        SIDR_SEC_ADD(13, t_p2);
    }
    G::sync();
    if (COUNT) {
        wc.heavy += heavy;
        wc.ops += heavy * kOpsAtRisk;
    }
    return eloss;
}

// The view of lane's candidate ci (-1: none) at decision d.
__device__ __forceinline__ AtRiskView at_risk_view(const DevInst& I, const WarpSmem& S,
                                                   const Decision& d, int ci) {
    AtRiskView v;
    v.CU = reinterpret_cast<const double2*>(I.CU);
    v.scores = I.scores;
    v.DP = reinterpret_cast<const double2*>(I.DP);
    v.DPc = v.DP;
    v.TKc = reinterpret_cast<const double2*>(I.TK);
    v.TCc = I.TC;
    v.atr = S.atr;
    v.Q = S.rows;
    v.n = I.n;
    v.nw = I.nw;
    v.cap = S.qcap / 2;
    v.ci = ci;
    v.tmax = I.tmax;
    v.fin_c = 0.0;
    v.sd_c = 0.0;
    if (ci >= 0) {
        const double ta = I.dist[(size_t)d.cur * I.ld + ci + 1];
        const double open_i = I.open_t[ci], dur_i = I.durations[ci];
        const double arr_c = d.ct + ta;
        const double st_c = arr_c > open_i ? arr_c : open_i;
        v.fin_c = st_c + dur_i;
        v.sd_c = kSigma * dur_i;
        v.DPc += ci;
        v.TKc += ci;
        v.TCc += ci;
    }
    return v;
}

// Terminals of candidate i into the lane's value rows, then the rule program.
// Returns the priority (NaN mapped to -1e300).  eloss: the candidate's ATRISK
// value (at_risk), when the rule reads it.
template <bool COUNT, bool RMOD, int LPP = 32>
__device__ double score_candidate(const DevInst& I, const WarpSmem& S, const RuleMeta& rm,
                                  const Decision& d, int i, double eloss, WarpCounts& wc) {
    const int lane = Group<LPP>::lane();
    const int n = I.n, ld = I.ld;
    const uint32_t need = rm.need;
    const double tmax = I.tmax;
    const double ct = d.ct;
    const int cur = d.cur;

    SIDR_SEC_MARK(t_setup)
    const double ta = I.dist[(size_t)cur * ld + i + 1];
    const double open_i = I.open_t[i], close_i = I.close_t[i];
    const double dur_i = I.durations[i], sc_i = I.scores[i], d2d_i = I.d2d[i];
    const double to = open_i - ct;
    const double tc = close_i - ct;
    const double tsv = to > ta ? to : ta;
    const double tfv = tsv + dur_i;
    const double fin = ct + tfv;                 // finish_i of the NS family
    const double arr_c = ct + ta;
    const double st_c = arr_c > open_i ? arr_c : open_i;
    const double fin_c = st_c + dur_i;           // finish_c of the cascade family
    const double frob = fin + dur_i * kSigma;    // robust finish
    if (COUNT) wc.ops += kOpsCandidate + rm.n_ins;

    double ns = 0.0, maxn = 0.0, r2v = 0.0, nstw = 0.0, regret = 0.0, nsrob = 0.0, r2rv = 0.0;
    double fcnt = 0.0, fsc = 0.0, smin = 1e18, sbv = -1.0, k1v = -1.0;
    int r2j = -1, r2rj = -1, sbq = -1, k1q = -1;

    SIDR_SEC_ADD(2, t_setup);
    SIDR_SEC_MARK(t_fused)
    const uint32_t fused = kNeedNSFused | kNeedRegret | kNeedRob | kNeedAfterC;
    if (need & fused) {
        // neighbour-major pairs of origin i+1: {F, R} and {G, dist} at j*ld + i+1
        const double2* FRi = reinterpret_cast<const double2*>(I.FR) + (i + 1);
        const double2* GDi = reinterpret_cast<const double2*>(I.GD) + (i + 1);
        const bool need_gd =
            (need & (kNeedRob | kNeedNSTW | kNeedStruct | kNeedPBust)) != 0;
        const uint32_t* zlti = I.zlt + (size_t)(i + 1) * I.nw;
        const uint32_t* zlei = I.zle + (size_t)(i + 1) * I.nw;
        unsigned long long scan = 0;

        // One neighbour j (bit b of its word): every accumulator is updated in
        // ascending j, as each reference loop runs.
        auto visit = [&](int j, int b, double2 fr, double2 gd, uint32_t zl, uint32_t ze,
                         uint32_t nowb) {
            if (COUNT) scan++;
            const double Fj = fr.x, Rj = fr.y;
            const double sj = I.scores[j];
            const bool nz = !((zl >> b) & 1u);
            const bool fa = fin <= Fj;
            if (need & kNeedNSFused) {
                if (fa && nz) {
                    ns += Rj;
                    if (Rj > maxn) maxn = Rj;
                    if (Rj > r2v) {
                        r2v = Rj;
                        r2j = j;
                    }
                    if (need & kNeedNSTW) {
                        const double arrive = fin + gd.y;
                        const double oj = I.open_t[j];
                        if (arrive >= oj) {
                            nstw += Rj;  // wait 0: weight 1 - 0/win = 1 (or 1 when win <= 1e-10)
                        } else {
                            const double wait = oj - arrive;
                            const double win = I.close_t[j] - oj;
                            double wt = win > 1e-10 ? 1.0 - wait / win : 1.0;
                            if (wt < 0.0) wt = 0.0;
                            nstw += Rj * wt;
                        }
                    }
                }
            }
            if (need & kNeedRegret) {
                if (((nowb >> b) & 1u) && !fa) regret += sj;
            }
            if (need & kNeedRob) {
                if (nz && frob <= gd.x) {
                    nsrob += Rj;
                    if (Rj > r2rv) {
                        r2rv = Rj;
                        r2rj = j;
                    }
                }
            }
            if (need & kNeedAfterC) {
                const bool fc = fin_c <= Fj;
                if ((need & kNeedStruct) && ((nowb >> b) & 1u) && !fc) {
                    fcnt += 1.0;
                    fsc += sj;
                }
                if (fc) {
                    if (need & (kNeedStruct | kNeedPBust)) {
                        const double aq = fin_c + gd.y;
                        const double slack = I.close_t[j] - aq;
                        if (slack < smin) smin = slack;
                        if (!((ze >> b) & 1u) && Rj > sbv) {
                            sbv = Rj;
                            sbq = j;
                        }
                    }
                    if ((need & kNeedReachK) && Rj > k1v) {
                        k1v = Rj;
                        k1q = j;
                    }
                }
            }
        };

        for (int w = 0; w < I.nw; w++) {
            uint32_t bits = S.unv[w] & ~bit_in_word(i, w);
            if (!bits) continue;
            const uint32_t zl = zlti[w], ze = zlei[w];
            const uint32_t nowb = S.feas[w];
            // one neighbour per iteration, the next one's loads issued before the visit
            int bc = __ffs(bits) - 1;
            bits &= bits - 1;
            double2 frc = FRi[(size_t)((w << 5) + bc) * ld];
            double2 gdc = make_double2(0.0, 0.0);
            if (need_gd) gdc = GDi[(size_t)((w << 5) + bc) * ld];
            for (;;) {
                const bool more = bits != 0;
                const int bn = more ? __ffs(bits) - 1 : bc;
                bits &= bits - 1;
                const double2 frn = FRi[(size_t)((w << 5) + bn) * ld];
                double2 gdn = make_double2(0.0, 0.0);
                if (need_gd) gdn = GDi[(size_t)((w << 5) + bn) * ld];
                visit((w << 5) + bc, bc, frc, gdc, zl, ze, nowb);
                if (!more) break;
                bc = bn;
                frc = frn;
                gdc = gdn;
            }
        }
        if (COUNT) {
            wc.scan += scan;
            wc.ops += scan * rm.scan_ops;
        }
    }

    SIDR_SEC_ADD(3, t_fused);
    SIDR_SEC_MARK(t_hops)
    // REACH2 / REACH2ROB second hops.
    double reach2 = 0.0, reach2rob = 0.0;
    if ((need & kNeedReach2) && r2j >= 0) {
        const double arrive = fin + I.dist[(size_t)(i + 1) * ld + r2j + 1];
        const double st = arrive > I.open_t[r2j] ? arrive : I.open_t[r2j];
        const double fj = st + I.durations[r2j];
        reach2 = I.scores[r2j] + second_hop_score<COUNT>(I, S, I.sF, I.bF, r2j + 1, fj, i, r2j, wc.hop);
    }
    if ((need & kNeedReach2Rob) && r2rj >= 0) {
        const double arrive = frob + I.dist[(size_t)(i + 1) * ld + r2rj + 1];
        const double st = arrive > I.open_t[r2rj] ? arrive : I.open_t[r2rj];
        const double fj = st + I.durations[r2rj] * (1.0 + kSigma);
        reach2rob = I.scores[r2rj] + second_hop_score<COUNT>(I, S, I.sG, I.bG, r2rj + 1, fj, i, r2rj, wc.hop);
    }

    // REACH-1/3/5 share one greedy path (each is the running total after
    // 1, 3 or 5 steps of the same walk, engine/sim_terms.hpp:405-441).
    double rk1 = 0.0, rk3 = 0.0, rk5 = 0.0;
    if (need & kNeedReachK) {
        int p1 = -1, p2 = -1, p3 = -1, p4 = -1;  // the walk's customers after the candidate
        double tot = 0.0, tm = 0.0;
        int at = 0;
        bool alive = k1q >= 0;
        if (alive) {
            const double arrive = fin_c + I.dist[(size_t)(i + 1) * ld + k1q + 1];
            const double st = arrive > I.open_t[k1q] ? arrive : I.open_t[k1q];
            tm = st + I.durations[k1q];
            at = k1q + 1;
            tot += I.scores[k1q];
            p1 = k1q;
        }
        rk1 = tot;
        for (int step = 2; step <= rm.reach_k; step++) {
            if (alive) {
                const int bq = reach_step<COUNT>(I, S, at, tm, i, p1, p2, p3, p4, wc.hop);
                if (bq < 0) {
                    alive = false;
                } else {
                    const double arrive = tm + I.dist[(size_t)at * ld + bq + 1];
                    const double st = arrive > I.open_t[bq] ? arrive : I.open_t[bq];
                    tm = st + I.durations[bq];
                    at = bq + 1;
                    tot += I.scores[bq];
                    if (step == 2) p2 = bq;
                    else if (step == 3) p3 = bq;
                    else if (step == 4) p4 = bq;
                }
            }
            if (step == 3) rk3 = tot;
            if (step == 5) rk5 = tot;
        }
    }

    SIDR_SEC_ADD(4, t_hops);
    SIDR_SEC_MARK(t_pbust)
    double pbust = 0.0;
    if ((need & kNeedPBust) && sbq >= 0) {
        const double ab = fin_c + I.dist[(size_t)(i + 1) * ld + sbq + 1];
        const double sd = kSigma * dur_i;
        if (sd > 1e-12) {
            const double z = (I.close_t[sbq] - ab) / (sd * kSqrt2);
            pbust = 0.5 * libm::erfc_(z);
        } else {
            pbust = ab > I.close_t[sbq] ? 1.0 : 0.0;
        }
    }
    const double downslack = smin > 1e17 ? 0.0 : smin;

    SIDR_SEC_ADD(5, t_pbust);
    SIDR_SEC_MARK(t_rows)
    // Terminal rows.
    for (int k = 0; k < rm.K; k++) {
        const int slot = S.slots[k];
        double v;
        switch (slot) {
        case 0: v = sc_i; break;
        case 1: v = dur_i; break;
        case 2: v = to; break;
        case 3: v = tc; break;
        case 4: v = ta; break;
        case 5: v = d2d_i; break;
        case 6: v = tsv; break;
        case 7: v = tfv; break;
        case 8: v = tc - ta; break;
        case 9: v = d.remaining * tmax + (tmax - ct); break;
        case 10: v = ns; break;
        case 11: v = regret; break;
        case 12: v = nsrob; break;
        case 13: v = maxn; break;
        case 14: v = reach2; break;
        case 15: v = nstw; break;
        case 16: v = t_rand_dev(i); break;
        case 17: v = fcnt; break;
        case 18: v = fsc; break;
        case 19: v = downslack; break;
        case 20: v = pbust; break;
        case 21: v = rk1; break;
        case 22: v = rk3; break;
        case 23: v = rk5; break;
        case 24: v = d.sat; break;
        case 25: v = d.vfrac; break;
        case 26: v = d.nfeas; break;
        case 27: v = (double)d.remaining; break;
        case 28: v = fsc / (ns + 1.0); break;
        case 29: v = fsc - ns; break;
        case 30: v = eloss; break;
        case 31: v = (tc - I.zp[0]) / I.zp[5]; break;
        case 32: v = (reach2 - I.zp[1]) / I.zp[6]; break;
        case 33: v = (regret - I.zp[2]) / I.zp[7]; break;
        case 34: v = (eloss - I.zp[3]) / I.zp[8]; break;
        case 35: v = (d2d_i - I.zp[4]) / I.zp[9]; break;
        case 36: v = 0.1; break;
        case 37: v = 0.2; break;
        case 38: v = 0.3; break;
        case 39: v = 0.4; break;
        case 40: v = 0.5; break;
        case 41: v = reach2rob; break;
        case 42: {
            double den = tmax - ct;
            if (den < 1.0) den = 1.0;
            v = (ta + dur_i) / den;
            break;
        }
        case 43: v = reach2rob - regret; break;
        case 44: v = x_skiploss(I, S, i, cur, ct); break;
        case 45: v = ns - nsrob; break;
        case 46: {
            double den = ta + d2d_i;
            if (den < 1.0) den = 1.0;
            v = (sc_i + nsrob) / den;
            break;
        }
        case 47: v = x_reach_k_rob(I, S, i, st_c + dur_i * (1.0 + kSigma), 3); break;
        case 48: v = x_reach_k_rob(I, S, i, st_c + dur_i * (1.0 + kSigma), 5); break;
        case 49: v = x_ns_family(I, S, i, fin, 0); break;
        case 50: v = x_ns_family(I, S, i, fin, 1); break;
        case 51: v = d.fscore; break;
        case 52: v = d.nfeasrob; break;
        case 53: v = x_ns_rob_m(I, S, i, fin, 0.5); break;
        case 54: v = x_ns_rob_m(I, S, i, fin, 2.0); break;
        case 55: v = x_ns_family(I, S, i, fin, 2); break;
        case 56: v = x_ns_family(I, S, i, fin, 3); break;
        case 57: v = x_nnchain(I, S, i, fin_c, 3); break;
        case 58: v = I.dist[(size_t)cur * ld + 0] + d2d_i - ta; break;
        case 59: v = x_detour(I, S, i, cur, fin, ta); break;
        case 60: v = x_ns_family(I, S, i, fin, 4); break;
        default: v = 0.0; break;
        }
        S.rows[k * LPP + lane] = v;
    }

    SIDR_SEC_ADD(6, t_rows);
    SIDR_SEC_MARK(t_prog)
    // Rule program (engine/sim_core.hpp:11-41 as three-address code).
    for (int q = 0; q < rm.n_ins; q++) {
        const uint32_t wd = S.prog[q];
        const uint32_t op = wd & 7u;
        const uint32_t oa = (wd >> 3) & 1023u, ob = (wd >> 13) & 1023u, od = wd >> 23;
        const double a = (oa & kOpConst) ? S.cst[oa & 511u] : S.rows[oa * LPP + lane];
        const double b = (ob & kOpConst) ? S.cst[ob & 511u] : S.rows[ob * LPP + lane];
        double r;
        switch (op) {
        case 0: r = a + b; break;
        case 1: r = a - b; break;
        case 2: r = a * b; break;
        case 3: r = fabs(b) < 1e-10 ? 1.0 : a / b; break;
        case 4: r = a < b ? a : b; break;
        case 5: r = a > b ? a : b; break;
        default:
            // rmod: glibc's pow restated, so the result is the CPU's.  Only the
            // RMOD instantiation has it; the others never see opcode 6 (the
            // host picks the kernel, the staging guard refuses such rules), and
            // their unreachable branch keeps the shape of a call to CUDA's pow
            // on rmod's clamped arguments: with it the kernel measured 5 % faster
            // than with a constant there (instruction placement; the
            // instructions executed are the same), and its value is never used.
            if constexpr (RMOD) r = libm::rmod_(a, b);
            else r = pow(a > 0.0 ? a : 0.0, 1.0 + (b < 0.0 ? 0.0 : (b > 1.0 ? 1.0 : b)));
        }
        S.rows[od * LPP + lane] = r;
    }
    SIDR_SEC_ADD(7, t_prog);
    const uint32_t res = (uint32_t)rm.res;
    double pri = (res & kOpConst) ? S.cst[res & 511u] : S.rows[res * LPP + lane];
    if (pri != pri) pri = -1e300;
    return pri;
}

// Where a capture launch records one decision (slot < 0: not recorded).
struct CaptureAt {
    const CaptureBuf* C;
    int slot;
};

// One decision: returns the chosen customer or -1 (pick_best).  CAPTURE:
// every candidate's terminal rows (the first B.cap_k rows: the rule was
// compiled with all active slots as rows) and the choice are recorded.
// LPP: lanes of the pair's group; candidates are spread LPP per round.
template <bool COUNT, bool RMOD, bool CAPTURE = false, int LPP = 32>
__device__ int decide(const DevInst& I, const WarpSmem& S, const RuleMeta& rm, Decision& d,
                      WarpCounts& wc, CaptureAt cap = CaptureAt{nullptr, -1}) {
    static_assert(LPP == 32 || !CAPTURE, "capture runs whole warps");
    using G = Group<LPP>;
    const int lane = G::lane();
    const int n = I.n, ld = I.ld, nw = I.nw;
    const uint32_t need = rm.need;
    const bool need_atr = (need & kNeedAtRisk) != 0;

    SIDR_SEC_MARK(t_prep)
    // Feasible-now bitmask (the reference's candidate filter, :75-82) and
    // ATRISK's arrive-by-close filter, one ballot per LPP customers.
    const double* Fc = I.F + (size_t)d.cur * n;
    const double* Dc = I.dist + (size_t)d.cur * ld + 1;
    for (int w = 0; w < nw; w++) {
        uint32_t bf = 0, ba = 0;
#pragma unroll
        for (int h = 0; h < 32; h += LPP) {
            const int t = h + lane;
            const int j = (w << 5) + t;
            const bool u = (S.unv[w] >> t) & 1u;
            const bool f = u && d.ct <= Fc[j];
            bf |= G::ballot(f) << h;
            if (need_atr) {
                const bool a = u && !(d.ct + Dc[j] > I.close_t[j]);
                ba |= G::ballot(a) << h;
            }
        }
        if (lane == 0) {
            S.feas[w] = bf;
            S.atr[w] = ba;
        }
    }
    G::sync();

    SIDR_SEC_ADD(0, t_prep);
    SIDR_SEC_MARK(t_compact)
    int ncand = 0;
    for (int w = 0; w < nw; w++) {
        const uint32_t bits = S.feas[w];
#pragma unroll
        for (int h = 0; h < 32; h += LPP) {
            const int t = h + lane;
            if ((bits >> t) & 1u) S.cand[ncand + __popc(bits & ((1u << t) - 1u))] = (int16_t)((w << 5) + t);
        }
        ncand += __popc(bits);
    }
    G::sync();

    // Per-decision aggregates (:55-71).
    d.sat = I.tmax > 0.0 ? d.ct / I.tmax : 0.0;
    if (need & (kNeedAgg | kNeedFScore | kNeedNFeasRob)) {
        int unv = 0;
        for (int w = 0; w < nw; w++) unv += __popc(S.unv[w]);
        d.vfrac = (double)(n - unv) / n;
        d.nfeas = (double)ncand;
        double fs = 0.0, nr = 0.0;
        if (need & (kNeedFScore | kNeedNFeasRob)) {
            for (int k = 0; k < ncand; k++) {
                const int j = S.cand[k];
                fs += I.scores[j];
                const double arr = d.ct + Dc[j];
                const double st = arr > I.open_t[j] ? arr : I.open_t[j];
                if (st + I.durations[j] * (1.0 + kSigma) + I.d2d[j] <= I.tmax) nr += 1.0;
            }
        }
        d.fscore = fs;
        d.nfeasrob = nr;
    } else {
        d.vfrac = d.nfeas = d.fscore = d.nfeasrob = 0.0;
    }
    if (COUNT && lane == 0) {
        wc.dec++;
        wc.cand += ncand;
        wc.ops += 2ull * n;
    }

    SIDR_SEC_ADD(1, t_compact);
    int best = -1;
    double best_pri = -1e300;
    for (int base = 0; base < ncand; base += LPP) {
        const int k = base + lane;
        double pri = -1e300;
        int idx = 0x7fffffff;
        SIDR_SEC_MARK(t_atr)
        const double eloss =
            need_atr ? at_risk<COUNT, LPP>(at_risk_view(I, S, d, k < ncand ? S.cand[k] : -1), wc) : 0.0;
        SIDR_SEC_ADD(10, t_atr);
        if (k < ncand) {
            idx = S.cand[k];
            pri = score_candidate<COUNT, RMOD, LPP>(I, S, rm, d, idx, eloss, wc);
            if (CAPTURE && cap.slot >= 0 && k < cap.C->cand) {
                const CaptureBuf& C = *cap.C;
                const size_t at = (size_t)cap.slot * C.cand + k;
                for (int r = 0; r < C.k; r++) C.rows[at * C.k + r] = S.rows[r * 32 + lane];
                C.cust[at] = idx;
            }
        }
        SIDR_SEC_MARK(t_argmax)
#pragma unroll
        for (int off = LPP / 2; off > 0; off >>= 1) {
            const double op = G::shfl_xor(pri, off);
            const int oi = G::shfl_xor(idx, off);
            if (op > pri || (op == pri && oi < idx)) {
                pri = op;
                idx = oi;
            }
        }
        if (pri > best_pri) {
            best_pri = pri;
            best = idx;
        }
        SIDR_SEC_ADD(8, t_argmax);
    }
    if (CAPTURE && cap.slot >= 0 && lane == 0) {
        cap.C->info[2 * cap.slot] = ncand;
        cap.C->info[2 * cap.slot + 1] = best;
    }
    return best;
}

// sim_one (engine/sim_core.hpp:207-238) for one pair; every lane of the
// pair's group returns the same total.
template <bool COUNT, bool RMOD, bool CAPTURE = false, int LPP = 32>
__device__ double rollout(const DevInst& I, const WarpSmem& S, const RuleMeta& rm,
                          const double* smp, WarpCounts& wc, const CaptureBuf* capC = nullptr,
                          int scenario = 0) {
    using G = Group<LPP>;
    const int lane = G::lane();
    const int n = I.n, ld = I.ld;
    for (int w = lane; w < I.nw; w += LPP) {
        const int lo = w << 5;
        const int cnt = n - lo >= 32 ? 32 : n - lo;
        S.unv[w] = cnt >= 32 ? kFull : ((1u << cnt) - 1u);
    }
    G::sync();
    double total = 0.0;
    int dec_no = 0;
    for (int v = 0; v < I.m; v++) {
        Decision d;
        d.remaining = I.m - v - 1;
        d.cur = 0;
        d.ct = 0.0;
        for (;;) {
            int b;
            if constexpr (CAPTURE) {
                CaptureAt cap{capC, dec_no < capC->dec ? scenario * capC->dec + dec_no : -1};
                dec_no++;
                b = decide<COUNT, RMOD, true>(I, S, rm, d, wc, cap);
            } else {
                b = decide<COUNT, RMOD, false, LPP>(I, S, rm, d, wc);
            }
            if (b < 0) break;
            SIDR_SEC_MARK(t_upd)
            const double arrive = d.ct + I.dist[(size_t)d.cur * ld + b + 1];
            const double st = arrive > I.open_t[b] ? arrive : I.open_t[b];
            d.ct = st + smp[b];
            d.cur = b + 1;
            total += I.scores[b];
            if (lane == 0) S.unv[b >> 5] &= ~(1u << (b & 31));
            G::sync();
            SIDR_SEC_ADD(9, t_upd);
        }
    }
    return total;
}

// Why a rule record cannot run in a warp slice carved for B (0 = it can):
// program, constants and rows beyond the slice's capacities, a result operand
// outside them, rmod instructions in a kernel built without them, or
// (multi-instance batches) an instance outside the batch.
__device__ __forceinline__ int rule_record_error(const RuleMeta& m, const DevBatch& B, bool multi,
                                                 bool rmod) {
    const bool fits = m.n_ins >= 0 && m.n_ins <= B.prog_cap && m.n_const >= 0 &&
                      m.n_const <= B.const_cap && m.K >= 0 && m.K <= 64 && m.D >= 0 &&
                      m.K + m.D <= B.rows && m.res >= 0 &&
                      ((m.res & kOpConst) ? (m.res & 511) < m.n_const : m.res < m.K + m.D);
    if (!fits || (!rmod && (m.need & kNeedRmod))) return kErrRuleRecord;
    if (multi && (m.inst < 0 || m.inst >= B.n_inst)) return kErrInstance;
    return 0;
}

// One work item (a rule and a scenario) on the pair's group: the rule's
// program, constants, slot list (and, MULTI, its instance descriptor) are
// staged into the group's slice when the rule changes, then the rollout runs
// and its total is stored.
template <bool COUNT, bool MULTI, bool RMOD, bool CAPTURE, int LPP>
__device__ __forceinline__ void run_item(const DevInst& I0, const DevBatch& B, const WarpSmem& S,
                                         unsigned long long item, int& staged, RuleMeta& rm,
                                         WarpCounts& wc, const CaptureBuf* capC) {
    using G = Group<LPP>;
    const int lane = G::lane();
    const int r = (int)(item / (unsigned long long)B.T);
    const int s = (int)(item % (unsigned long long)B.T);
    const int p = B.order ? B.order[r] : r;
    if (p != staged) {
        // Guard of the group's shared-memory slice: a rule record the launch
        // was not sized for is refused (error word set, score NaN) before
        // anything of it is staged.  Host validation makes this unreachable;
        // the host reads the word back after every launch.
        const int code = (p < 0 || p >= B.P) ? kErrRuleIndex : rule_record_error(B.meta[p], B, MULTI, RMOD);
        if (code) {
            if (lane == 0) {
                atomicCAS(B.error, 0, code);
                if (p >= 0 && p < B.P) B.out[(size_t)p * B.T + s] = __longlong_as_double(0x7ff8000000000000LL);
            }
            staged = -1;
            G::sync();
            return;
        }
        rm = B.meta[p];
        for (int q = lane; q < rm.n_ins; q += LPP) S.prog[q] = B.prog[rm.prog_off + q];
        for (int q = lane; q < rm.n_const; q += LPP) S.cst[q] = B.consts[rm.const_off + q];
        for (int q = lane; q < rm.K; q += LPP) S.slots[q] = B.slots[rm.slot_off + q];
        if (MULTI) {
            const unsigned long long* src =
                reinterpret_cast<const unsigned long long*>(B.insts + rm.inst);
            unsigned long long* dst = reinterpret_cast<unsigned long long*>(S.inst);
            for (int q = lane; q < (int)(sizeof(DevInst) / 8); q += LPP) dst[q] = src[q];
        }
        staged = p;
        G::sync();
    }
    const DevInst& I = MULTI ? *S.inst : I0;
    const double* smp =
        MULTI ? B.sampled + B.smp_off[rm.inst] + (size_t)s * I.n
              : B.sampled + ((size_t)(p / B.group_size) * B.T + s) * (size_t)B.n;
    double tot;
    if constexpr (CAPTURE) tot = rollout<COUNT, RMOD, true>(I, S, rm, smp, wc, capC, s);
    else tot = rollout<COUNT, RMOD, false, LPP>(I, S, rm, smp, wc);
    if (lane == 0) B.out[(size_t)p * B.T + s] = tot;
}

// The persistent work loop.  MULTI: every rule carries its instance; the
// group stages the instance descriptor with the rule's program.  LPP < 32:
// the warp's first lane takes 32 / LPP consecutive items from the queue at
// once (usually one rule on neighbouring scenarios), one per group; the groups
// run side by side and the warp takes its next items when all are done.
template <bool COUNT, bool MULTI, bool RMOD, bool CAPTURE = false, int LPP = 32>
__device__ __forceinline__ void eval_body(const DevInst& I0, const DevBatch& B,
                                          const CaptureBuf* capC = nullptr) {
    static_assert(LPP == 32 || (!COUNT && !CAPTURE), "counting and capture run whole warps");
    using G = Group<LPP>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31;
    const int gib = (threadIdx.x >> 5) * G::kPerWarp + G::index();  // group in block
    const size_t slice = warp_slice_bytes(B.rows, B.const_cap, B.prog_cap, LPP);
    const WarpSmem S = carve(smem_raw + (size_t)gib * slice, B.rows, B.const_cap, B.prog_cap, LPP);

    const unsigned long long total =
        (unsigned long long)(B.P_items > 0 ? B.P_items : B.P) * (unsigned long long)B.T;
    int staged = -1;
    RuleMeta rm;
    WarpCounts wc = {0, 0, 0, 0, 0, 0};
    for (;;) {
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(B.counter, (unsigned long long)G::kPerWarp);
        base = __shfl_sync(kFull, base, 0);
        if (base >= total) break;
        if constexpr (LPP == 32) {
            run_item<COUNT, MULTI, RMOD, CAPTURE, LPP>(I0, B, S, base, staged, rm, wc, capC);
        } else {
            const unsigned long long item = base + (unsigned long long)G::index();
            if (item < total) run_item<COUNT, MULTI, RMOD, CAPTURE, LPP>(I0, B, S, item, staged, rm, wc, capC);
        }
    }
    if (COUNT) {
        // dec/cand/per-decision ops live in lane 0; the rest are per lane.
        unsigned long long v[kStats] = {wc.dec, wc.cand, wc.scan, wc.heavy, wc.hop, wc.ops};
#pragma unroll
        for (int k = 2; k < kStats; k++)
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) v[k] += __shfl_xor_sync(kFull, v[k], off);
        if (lane == 0 && B.stats) {
#pragma unroll
            for (int k = 0; k < kStats; k++) atomicAdd(&B.stats[k], v[k]);
        }
    }
}

// Single-instance evaluator (the instance travels as a kernel parameter).
// RMOD: the batch has rules with rmod; the kernels without it carry no code
// for the power function, which would cost the others several percent.
// MINB: resident blocks per SM the registers are budgeted for --
// SIDR_MIN_BLOCKS (4: 128 registers) by default, or kMoreBlocks (5: 96
// registers, more warps to hide latency, more spills), which pays on
// populations that spend their time in ATRISK's long classification loops.
// LPP: lanes per pair (32: a warp per pair; 16: two pairs per warp).
constexpr int kMoreBlocks = 5;

template <bool COUNT, bool RMOD, int MINB, int LPP = 32>
__global__ void __launch_bounds__(32 * SIDR_WARPS_PER_BLOCK, MINB)
    eval_kernel(const DevInst I, const DevBatch B) {
    eval_body<COUNT, false, RMOD, false, LPP>(I, B);
}

// Decision-situation capture: one rule on B.T scenarios, every decision's
// candidate terminal tables recorded (DevBatch cap_* fields).
__global__ void __launch_bounds__(32 * SIDR_WARPS_PER_BLOCK, SIDR_MIN_BLOCKS)
    capture_kernel(const DevInst I, const DevBatch B, const CaptureBuf C) {
    eval_body<false, false, true, true>(I, B, &C);
}

// Multi-instance evaluator, one instantiation per block shape (warps per
// block x minimum resident blocks x lanes per pair); the autotuner picks
// among them for each class of instance sizes.
template <int WPB, int MINB, bool RMOD, int LPP = 32>
__global__ void __launch_bounds__(32 * WPB, MINB) eval_multi_kernel(const DevBatch B) {
    eval_body<false, true, RMOD, false, LPP>(DevInst{}, B);
}

}  // namespace sidr
