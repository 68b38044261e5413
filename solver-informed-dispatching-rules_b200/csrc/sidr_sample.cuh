// sidr_sample.cuh -- the Box-Muller step of scenario sampling (gauss and
// sample_duration, engine/rng.hpp:135-147, engine/sim_host.hpp:43-58) for the
// on-device sampler, in code that compiles for the host and the device.
//
// The reference draws each service time as max(0, mu + z * (sigma * mu)),
// z = cos(2 pi u1) * sqrt(-2 log(1 - u2)) (its pair partner uses sin), with the
// host C library's log, cos and sin.  Those are not correctly rounded, so the
// device cannot simply call its own.  Here each of the three values is
// computed in double-double arithmetic (about 2^-100 relative error):
// log by log(m 2^e) = e ln 2 + 2 atanh((m-1)/(m+1)), sin and cos by a
// three-part pi/2 reduction and their Taylor series.  The C library's result
// is one of the two doubles around the exact value; it is the nearer one
// (hi) unless the exact value lies within the library's error of the
// midpoint.  The bound used is 0.52 units in the last place for log (the
// published worst case of the C library's log is 0.519) and 0.56 for sin and
// cos (errors measured on this interval stay below 0.515); with a margin of
// 0.01, a value whose double-double tail lies within (1 - bound - 0.01) of a
// unit of hi has hi as its library result, and otherwise both neighbours are
// candidates.  A duration is settled when every combination of candidates
// gives the same double; the rest (a few percent of the pairs) are left to
// the host, which recomputes them with its own C library.
//
// Every operation keeps the reference's order and rounding: the files that
// include this one are compiled without multiply-add contraction; fma() is
// only called explicitly, for exact products.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>

#include "sidr_sample_consts.h"

#ifdef __CUDACC__
#define SIDR_HD __host__ __device__ __forceinline__
#else
#define SIDR_HD inline
#endif

namespace sidr {
namespace smp {

struct dd {
    double hi, lo;
};

SIDR_HD dd two_sum(double a, double b) {
    const double s = a + b;
    const double bb = s - a;
    return {s, (a - (s - bb)) + (b - bb)};
}
SIDR_HD dd quick_two_sum(double a, double b) {
    const double s = a + b;
    return {s, b - (s - a)};
}
SIDR_HD dd two_prod(double a, double b) {
    const double p = a * b;
    return {p, fma(a, b, -p)};
}
SIDR_HD dd add(dd x, dd y) {
    const dd s = two_sum(x.hi, y.hi);
    const dd t = two_sum(x.lo, y.lo);
    const dd u = quick_two_sum(s.hi, s.lo + t.hi);
    return quick_two_sum(u.hi, u.lo + t.lo);
}
SIDR_HD dd add_d(dd x, double y) {
    const dd s = two_sum(x.hi, y);
    return quick_two_sum(s.hi, s.lo + x.lo);
}
SIDR_HD dd neg(dd x) { return {-x.hi, -x.lo}; }
SIDR_HD dd mul(dd x, dd y) {
    const dd p = two_prod(x.hi, y.hi);
    return quick_two_sum(p.hi, p.lo + (x.hi * y.lo + x.lo * y.hi));
}
SIDR_HD dd mul_d(dd x, double y) {
    const dd p = two_prod(x.hi, y);
    return quick_two_sum(p.hi, p.lo + x.lo * y);
}
SIDR_HD dd div(dd x, dd y) {
    const double q1 = x.hi / y.hi;
    dd r = add(x, neg(mul_d(y, q1)));
    const double q2 = r.hi / y.hi;
    r = add(r, neg(mul_d(y, q2)));
    const double q3 = r.hi / y.hi;
    return add_d(quick_two_sum(q1, q2), q3);
}

struct DDConst {
    double hi, lo;
};

// log(x) for 0 < x <= 1 (x = 1 - u with u a 53-bit uniform draw).
SIDR_HD dd log_dd(double x) {
    constexpr DDConst kInvOdd[] = {SIDR_INV_ODD_TABLE};
    if (x == 1.0) return {0.0, 0.0};
    int e = 0;
    double m = frexp(x, &e);  // x = m 2^e, m in [0.5, 1)
    if (m < 0.70710678118654752440) {
        m *= 2.0;
        e -= 1;
    }
    // m in [sqrt(1/2), sqrt(2)): s = (m - 1) / (m + 1), |s| < 0.1716
    const dd s = div(dd{m - 1.0, 0.0}, two_sum(m, 1.0));
    const dd s2 = mul(s, s);
    // atanh(s) / s = sum over k of s^(2k) / (2k + 1); s^44 < 2^-110
    dd acc{kInvOdd[22].hi, kInvOdd[22].lo};
    for (int k = 21; k >= 0; k--) acc = add(mul(acc, s2), dd{kInvOdd[k].hi, kInvOdd[k].lo});
    const dd lm = mul_d(mul(acc, s), 2.0);
    const double ef = (double)e;
    const dd le = add_d(two_prod(ef, SIDR_LN2_HI), ef * SIDR_LN2_LO);
    return add(le, lm);
}

// sin(x) and cos(x) for 0 <= x < 2 pi.
SIDR_HD void sincos_dd(double x, dd& sn, dd& cs) {
    constexpr DDConst kInvFact[] = {SIDR_INV_FACT_TABLE};
    const double kf = rint(x * SIDR_TWO_OVER_PI);
    // r = x - k pi/2, pi/2 in three parts (k <= 4: each product exact or tiny)
    dd r = add(dd{x, 0.0}, neg(two_prod(kf, SIDR_PIO2_1)));
    r = add(r, neg(two_prod(kf, SIDR_PIO2_2)));
    r = add_d(r, -(kf * SIDR_PIO2_3));
    const dd r2 = mul(r, r);
    // |r| <= pi/4 + a little; with y = r^2, sin(r) / r = b0 - y (b1 - y (b2 - ...)),
    // b_j = 1 / (2j+1)!, to j = 15, and cos(r) the same with b_j = 1 / (2j)!, to
    // j = 16: the terms left out are below 2^-130
    dd s{kInvFact[31].hi, kInvFact[31].lo};
    for (int j = 14; j >= 0; j--) s = add(neg(mul(s, r2)), dd{kInvFact[2 * j + 1].hi, kInvFact[2 * j + 1].lo});
    dd c{kInvFact[32].hi, kInvFact[32].lo};
    for (int j = 15; j >= 0; j--) c = add(neg(mul(c, r2)), dd{kInvFact[2 * j].hi, kInvFact[2 * j].lo});
    s = mul(s, r);
    switch (((int)kf) & 3) {
    case 0: sn = s; cs = c; break;
    case 1: sn = c; cs = neg(s); break;
    case 2: sn = neg(s); cs = neg(c); break;
    default: sn = neg(c); cs = s; break;
    }
}

// The doubles the C library can return for the exact value v: v.hi, and its
// neighbour on the side of v.lo when v lies within `bound` units of the
// midpoint between them.  Returns how many (1 or 2).
// The double next to x (finite, nonzero) towards +infinity (up) or -infinity.
SIDR_HD double neighbour(double x, bool up) {
    uint64_t b;
    std::memcpy(&b, &x, 8);
    b = ((x > 0.0) == up) ? b + 1 : b - 1;  // away from zero: one more unit of the magnitude
    double r;
    std::memcpy(&r, &b, 8);
    return r;
}

SIDR_HD int candidates(dd v, double guard, double c[2]) {
    c[0] = c[1] = v.hi;
    if (v.lo == 0.0 || v.hi == 0.0) return 1;
    const double nb = neighbour(v.hi, v.lo > 0.0);
    const double u = fabs(nb - v.hi);
    if (fabs(v.lo) < guard * u) return 1;
    c[1] = nb;
    return 2;
}

constexpr double kGuardLog = 1.0 - 0.52 - 0.01;
constexpr double kGuardTrig = 1.0 - 0.56 - 0.01;

// sample_duration (engine/sim_host.hpp:43-47) from one Box-Muller value.
SIDR_HD double duration_of(double mu, double sd, double trig, double lg) {
    const double g2rad = sqrt(-2.0 * lg);
    const double z = trig * g2rad;
    const double v = mu + z * sd;
    return v > 0.0 ? v : 0.0;
}

// The two service times of one Box-Muller pair: d0 from cos (customer with
// mean mu0, sd0 = sigma * mu0), d1 from sin (has1: the pair's second value is
// used).  u1, u2: the pair's two 53-bit draws.  Returns true when both are
// settled (then d0, d1 are the reference's values); false leaves them to
// the host.
SIDR_HD bool gauss_pair_durations(double u1, double u2, double mu0, double sd0, bool has1, double mu1,
                                  double sd1, double& d0, double& d1) {
    constexpr double kTwoPi = 2.0 * 3.14159265358979323846;
    const double x2pi = u1 * kTwoPi;
    const dd lg = log_dd(1.0 - u2);
    dd sn, cs;
    sincos_dd(x2pi, sn, cs);
    double cl[2], cc[2], cn[2];
    const int nl = candidates(lg, kGuardLog, cl);
    const int nc = candidates(cs, kGuardTrig, cc);
    const int ns = has1 ? candidates(sn, kGuardTrig, cn) : 1;
    if (!has1) cn[0] = cn[1] = 0.0;
    bool ok = true;
    d0 = duration_of(mu0, sd0, cc[0], cl[0]);
    d1 = has1 ? duration_of(mu1, sd1, cn[0], cl[0]) : 0.0;
    for (int a = 0; a < nl; a++) {
        for (int b = 0; b < nc; b++)
            if (a + b > 0) {
                const double v = duration_of(mu0, sd0, cc[b], cl[a]);
                ok = ok && v == d0;  // both positive or +0
            }
        if (has1)
            for (int b = 0; b < ns; b++)
                if (a + b > 0) {
                    const double v = duration_of(mu1, sd1, cn[b], cl[a]);
                    ok = ok && v == d1;
                }
    }
    return ok;
}

// ---------------------------------------------------------------- MT19937
// The generator of engine/rng.hpp:13-83 in the pieces the sampler's warps run
// (on the device) and the tests replay (on the host).

constexpr int kMtN = 624, kMtM = 397;

// init_genrand(19650218) then init_by_array over the seed's 32-bit words,
// least significant first (a single zero word for seed 0): the sequential
// seeding recurrence, the previous word kept in a register.
SIDR_HD void mt_seed(uint32_t* mt, unsigned long long seed) {
    uint32_t key[2];
    int klen = 0;
    if (seed == 0) key[klen++] = 0u;
    while (seed) {
        key[klen++] = (uint32_t)(seed & 0xffffffffu);
        seed >>= 32;
    }
    uint32_t prev = 19650218u;
    mt[0] = prev;
    for (int i = 1; i < kMtN; i++) {
        prev = 1812433253u * (prev ^ (prev >> 30)) + (uint32_t)i;
        mt[i] = prev;
    }
    prev = mt[0];  // the word before mt[1]
    int i = 1, j = 0;
    for (int k = kMtN; k; k--) {
        prev = (mt[i] ^ ((prev ^ (prev >> 30)) * 1664525u)) + key[j] + (uint32_t)j;
        mt[i] = prev;
        i++;
        j++;
        if (i >= kMtN) {
            mt[0] = mt[kMtN - 1];
            i = 1;
        }
        if (j >= klen) j = 0;
    }
    for (int k = kMtN - 1; k; k--) {
        prev = (mt[i] ^ ((prev ^ (prev >> 30)) * 1566083941u)) - (uint32_t)i;
        mt[i] = prev;
        i++;
        if (i >= kMtN) {
            mt[0] = mt[kMtN - 1];
            i = 1;
        }
    }
    mt[0] = 0x80000000u;
}

SIDR_HD uint32_t mt_temper(uint32_t y) {
    y ^= (y >> 11);
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= (y >> 18);
    return y;
}

// The new value of word kk (kk < N - 1) in a state refresh, from the words
// as they are when its turn comes: mt[kk + M] for kk < N - M (not yet
// refreshed), mt[kk + M - N] otherwise (already refreshed); the last word is
// mt_refreshed_last.  The refresh runs in three phases, [0, N-M),
// [N-M, 2(N-M)) and [2(N-M), N-1), each reading only words that earlier
// phases finished or later ones have not touched yet.
SIDR_HD uint32_t mt_refreshed(const uint32_t* mt, int kk) {
    const uint32_t y = (mt[kk] & 0x80000000u) | (mt[kk + 1] & 0x7fffffffu);
    const uint32_t src = kk < kMtN - kMtM ? mt[kk + kMtM] : mt[kk + kMtM - kMtN];
    return src ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
}
SIDR_HD uint32_t mt_refreshed_last(const uint32_t* mt) {
    const uint32_t y = (mt[kMtN - 1] & 0x80000000u) | (mt[0] & 0x7fffffffu);
    return mt[kMtM - 1] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
}

// random(): a 53-bit draw from two tempered words (engine/rng.hpp:70-74).
SIDR_HD double mt_draw(uint32_t a, uint32_t b) {
    return ((double)(mt_temper(a) >> 5) * 67108864.0 + (double)(mt_temper(b) >> 6)) * (1.0 / 9007199254740992.0);
}

}  // namespace smp
}  // namespace sidr
