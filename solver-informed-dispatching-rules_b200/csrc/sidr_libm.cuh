// sidr_libm.cuh -- erf, erfc and exp with the results of the C library the
// reference simulator runs on, for host and device.
//
// The reference evaluates ATRISK's normal CDF with erf and PBUST with erfc
// (engine/sim_terms.hpp:221-223, :571) through glibc.  CUDA's erf and erfc are
// other approximations: they differ from glibc's in the last bit for a share
// of arguments, which changes a decision whenever a rule's priorities tie to
// within that bit (GP rules such as (SCORE/ATRISK)*ATRISK do).  So the
// evaluator computes them with the same published algorithms, evaluated in
// the same order, as glibc 2.39 on x86-64:
//
//   erf, erfc  fdlibm 5.3's rational approximations (Sun Microsystems, 1993):
//              x + x*P(x^2)/Q(x^2) below 0.84375; erx + P(s)/Q(s) with
//              s = |x|-1 below 1.25; exp(-z^2-0.5625)*exp((z-x)(z+x)+R/S)/x
//              with R/S in 1/x^2 (two coefficient sets split at 1/0.35) below
//              6 (erf) or 28 (erfc); the polynomials evaluated pairwise
//              (c0 + t*c1) + t^2*(c2 + t*c3) + ..., as glibc's s_erf.c does.
//   exp        the table-driven exponential of glibc 2.28+ (Szabolcs Nagy,
//              ARM optimized-routines): x = k*ln2/128 + r, 2^(k/128) from a
//              128-entry table (sidr_exp_table.h, generated by
//              gen_exp_table.py), exp(r)-1 by a degree-5 polynomial, with the
//              multiply-adds fused where glibc's FMA build (the one selected
//              on every x86-64 CPU with FMA) fuses them.
//   pow        glibc 2.28+'s power function from the same library (rmod,
//              engine/sim_core.hpp:30-35): x^y = exp(y*log(x)) with log(x) in
//              double-double from a 128-entry table of 1/c, log(c)
//              (sidr_pow_table.h, gen_pow_table.py) and a degree-8
//              polynomial of log1p(z/c - 1), the product y*log(x) split
//              exactly with a fused multiply-add, and the exponential above
//              taking the product's low part as a correction.
//
// Every other operation is a separately rounded IEEE operation (the device
// code is compiled with -fmad=false, the host code with -ffp-contract=off).
// tests/test_libm.py compares these functions with the host's glibc over
// random arguments in every interval, for the host and the device builds.
#pragma once
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "sidr_exp_table.h"
#include "sidr_pow_table.h"

#ifdef __CUDACC__
#define SIDR_HD __host__ __device__ __forceinline__
// erf and erfc stay out of line on the device: they run only for arguments
// whose result is not exactly 0 or 1, and inlining them into the neighbour
// scans would raise their register count
#define SIDR_HD_CALL static __host__ __device__ __noinline__  // one copy per translation unit
#else
#define SIDR_HD inline
#define SIDR_HD_CALL inline
#endif

namespace sidr {
namespace libm {

#ifdef __CUDACC__
__device__ const uint64_t kExpTableDev[256] = {SIDR_EXP_TABLE_ENTRIES};
#endif
static const uint64_t kExpTableHost[256] = {SIDR_EXP_TABLE_ENTRIES};
#ifdef __CUDACC__
__device__ const double kPowLogDev[384] = {SIDR_POW_LOG_TABLE_ENTRIES};
#endif
static const double kPowLogHost[384] = {SIDR_POW_LOG_TABLE_ENTRIES};

SIDR_HD uint64_t bits_of(double x) {
#ifdef __CUDA_ARCH__
    return (uint64_t)__double_as_longlong(x);
#else
    uint64_t u;
    memcpy(&u, &x, 8);
    return u;
#endif
}

SIDR_HD double double_of(uint64_t u) {
#ifdef __CUDA_ARCH__
    return __longlong_as_double((long long)u);
#else
    double x;
    memcpy(&x, &u, 8);
    return x;
#endif
}

SIDR_HD uint64_t exp_table(int i) {
#ifdef __CUDA_ARCH__
    return kExpTableDev[i];
#else
    return kExpTableHost[i];
#endif
}

SIDR_HD double pow_log_table(int i) {
#ifdef __CUDA_ARCH__
    return kPowLogDev[i];
#else
    return kPowLogHost[i];
#endif
}

// a*b + c with one rounding.
SIDR_HD double fused(double a, double b, double c) { return fma(a, b, c); }

// ------------------------------------------------------------------ exp

// exp(x).  The argument is reduced to r in about [-ln2/256, ln2/256]:
// k = round(x*128/ln2) through the 1.5*2^52 shift, r = x - k*ln2/128 with
// ln2/128 in two parts.  Then exp(x) = 2^(k/128) * exp(r)
// ~= S*(1 + tail + (exp(r)-1)) = S + S*tmp.
SIDR_HD double exp_(double x) {
    const double kInvLn2N = 0x1.71547652b82fep0 * 128.0;
    const double kNegLn2HiN = -0x1.62e42fefa0000p-8;
    const double kNegLn2LoN = -0x1.cf79abc9e3b3ap-47;
    const double kShift = 0x1.8p52;
    const double kC2 = 0x1.ffffffffffdbdp-2, kC3 = 0x1.555555555543cp-3;
    const double kC4 = 0x1.55555cf172b91p-5, kC5 = 0x1.1111167a4d017p-7;

    const uint32_t top = (uint32_t)(bits_of(x) >> 52) & 0x7ffu;  // biased exponent of |x|
    bool scaled = false;
    if (top - 0x3c9u >= 0x408u - 0x3c9u) {  // |x| < 2^-54 or |x| >= 512 (or not finite)
        if (top < 0x3c9u) return 1.0 + x;    // tiny: rounds to 1 (or 1 + x)
        if (top >= 0x409u) {                 // |x| >= 1024, inf, nan
            if (bits_of(x) == 0xfff0000000000000ull) return 0.0;
            if (top >= 0x7ffu) return 1.0 + x;
            return (bits_of(x) >> 63) ? 0.0 : HUGE_VAL;
        }
        scaled = true;  // 512 <= |x| < 1024: the result's scale needs care
    }
    double kd = fused(kInvLn2N, x, kShift);
    const uint64_t ki = bits_of(kd);
    kd -= kShift;
    const double r = fused(kd, kNegLn2LoN, fused(kd, kNegLn2HiN, x));
    const int idx = (int)(2 * (ki % 128));
    const double tail = double_of(exp_table(idx));
    uint64_t sbits = exp_table(idx + 1) + (ki << 45);
    const double r2 = r * r;
    const double tmp = fused(r2 * r2, fused(r, kC5, kC4), fused(r2, fused(r, kC3, kC2), tail + r));
    if (!scaled) {
        const double scale = double_of(sbits);
        return fused(scale, tmp, scale);
    }
    if ((ki & 0x80000000u) == 0) {  // k > 0: scale by 2^1009 afterwards
        sbits -= 1009ull << 52;
        const double scale = double_of(sbits);
        return 0x1p1009 * fused(scale, tmp, scale);
    }
    // k < 0: build the result at 2^1022 times its size and round it once to
    // the subnormal precision it will have (glibc's FMA build leaves these
    // products unfused)
    sbits += 1022ull << 52;
    const double scale = double_of(sbits);
    const double st = scale * tmp;
    double y = scale + st;
    if (y < 1.0) {
        double lo = scale - y + st;
        const double hi = 1.0 + y;
        lo = 1.0 - hi + y + lo;
        y = (hi + lo) - 1.0;
        if (y == 0.0) y = 0.0;
    }
    return 0x1p-1022 * y;
}

// ------------------------------------------------------------------ pow

// exp(x + xtail) * (sign_bias ? -1 : 1) for the power function: the
// exponential above with the low part of y*log(x) added to the reduced
// argument (|xtail| is far below ln2/128) and the result's sign carried in
// the scale's exponent bits.
SIDR_HD double exp_tail_(double x, double xtail, uint64_t sign_bias) {
    const double kInvLn2N = 0x1.71547652b82fep0 * 128.0;
    const double kNegLn2HiN = -0x1.62e42fefa0000p-8;
    const double kNegLn2LoN = -0x1.cf79abc9e3b3ap-47;
    const double kShift = 0x1.8p52;
    const double kC2 = 0x1.ffffffffffdbdp-2, kC3 = 0x1.555555555543cp-3;
    const double kC4 = 0x1.55555cf172b91p-5, kC5 = 0x1.1111167a4d017p-7;

    const uint32_t top = (uint32_t)(bits_of(x) >> 52) & 0x7ffu;
    bool scaled = false;
    if (top - 0x3c9u >= 0x408u - 0x3c9u) {  // |x| < 2^-54 or |x| >= 512
        if (top < 0x3c9u) {
            const double one = 1.0 + x;
            return sign_bias ? -one : one;
        }
        if (top >= 0x409u) {  // |x| >= 1024: overflow or underflow
            const bool neg = (bits_of(x) >> 63) != 0;
            const double v = neg ? 0.0 : HUGE_VAL;
            return sign_bias ? -v : v;
        }
        scaled = true;
    }
    double kd = fused(kInvLn2N, x, kShift);
    const uint64_t ki = bits_of(kd);
    kd -= kShift;
    double r = fused(kd, kNegLn2LoN, fused(kd, kNegLn2HiN, x));
    r += xtail;
    const int idx = (int)(2 * (ki % 128));
    const double tail = double_of(exp_table(idx));
    uint64_t sbits = exp_table(idx + 1) + ((ki + sign_bias) << 45);
    const double r2 = r * r;
    const double tmp = fused(r2 * r2, fused(r, kC5, kC4), fused(r2, fused(r, kC3, kC2), tail + r));
    if (!scaled) {
        const double scale = double_of(sbits);
        return fused(scale, tmp, scale);
    }
    if ((ki & 0x80000000u) == 0) {
        sbits -= 1009ull << 52;
        const double scale = double_of(sbits);
        return 0x1p1009 * fused(scale, tmp, scale);
    }
    sbits += 1022ull << 52;
    const double scale = double_of(sbits);
    const double st = scale * tmp;
    double y = scale + st;
    if (fabs(y) < 1.0) {  // round once at the subnormal precision
        const double one = y < 0.0 ? -1.0 : 1.0;
        double lo = scale - y + st;
        const double hi = one + y;
        lo = one - hi + y + lo;
        y = (hi + lo) - one;
        if (y == 0.0) y = double_of(sbits & 0x8000000000000000ull);
    }
    return 0x1p-1022 * y;
}

// log(x) for the bit pattern ix of a positive normal x (subnormals arrive
// normalised with a negative exponent), as hi + *tail.  x = 2^k z with z in
// [0x1.69555p-1, 0x1.69555p0); log(x) = k*ln2 + log(c) + log1p(z/c - 1),
// with r = z/c - 1 exact (one fused multiply-add) and log1p(r) = r - r^2/2 +
// r^3*q(r), q of degree 5.
SIDR_HD double log_tail_(uint64_t ix, double* tail) {
    const double kLn2Hi = 0x1.62e42fefa3800p-1, kLn2Lo = 0x1.ef35793c76730p-45;
    // log1p(r) - r = a0 r^2 + a1 r^3 + ... + a6 r^8, scaled for the evaluation below
    const double a0 = -0x1p-1, a1 = 0x1.555555555556p-2 * -2, a2 = -0x1.0000000000006p-2 * -2,
                 a3 = 0x1.999999959554ep-3 * 4, a4 = -0x1.555555529a47ap-3 * 4,
                 a5 = 0x1.2495b9b4845e9p-3 * -8, a6 = -0x1.0002b8b263fc3p-3 * -8;
    const uint64_t tmp = ix - 0x3fe6955500000000ull;
    const int i = (int)((tmp >> 45) % 128);
    const int k = (int)((int64_t)tmp >> 52);
    const double z = double_of(ix - (tmp & (0xfffull << 52)));
    const double kd = (double)k;
    const double invc = pow_log_table(3 * i), logc = pow_log_table(3 * i + 1);
    const double logctail = pow_log_table(3 * i + 2);
    const double r = fused(z, invc, -1.0);
    const double t1 = fused(kd, kLn2Hi, logc);
    const double t2 = t1 + r;
    const double lo1 = fused(kd, kLn2Lo, logctail);
    const double lo2 = t1 - t2 + r;
    const double ar = a0 * r;
    const double ar2 = r * ar;
    const double ar3 = r * ar2;
    const double hi = t2 + ar2;
    const double lo3 = fused(ar, r, -ar2);
    const double lo4 = t2 - hi + ar2;
    const double q = fused(ar2, fused(ar2, fused(r, a6, a5), fused(r, a4, a3)), fused(r, a2, a1));
    const double lo = fused(ar3, q, lo1 + lo2 + lo3 + lo4);
    const double y = hi + lo;
    *tail = hi - y + lo;
    return y;
}

// 0: y not an integer, 1: odd integer, 2: even integer (y finite, nonzero).
SIDR_HD int integer_kind(uint64_t iy) {
    const int e = (int)(iy >> 52 & 0x7ff);
    if (e < 0x3ff) return 0;
    if (e > 0x3ff + 52) return 2;
    if (iy & ((1ull << (0x3ff + 52 - e)) - 1)) return 0;
    if (iy & (1ull << (0x3ff + 52 - e))) return 1;
    return 2;
}

// x^y with the results of glibc's pow (round to nearest).
SIDR_HD_CALL double pow_(double x, double y) {
    const uint64_t kInf = 0x7ff0000000000000ull, kOne = 0x3ff0000000000000ull;
    uint64_t ix = bits_of(x), sign_bias = 0;
    const uint64_t iy = bits_of(y);
    uint32_t topx = (uint32_t)(ix >> 52);
    const uint32_t topy = (uint32_t)(iy >> 52);
    if (topx - 0x001u >= 0x7ffu - 0x001u || (topy & 0x7ffu) - 0x3beu >= 0x43eu - 0x3beu) {
        if (2 * iy - 1 >= 2 * kInf - 1) {  // y is 0, inf or nan
            if (2 * iy == 0) return 1.0;
            if (ix == kOne) return 1.0;
            if (2 * ix > 2 * kInf || 2 * iy > 2 * kInf) return x + y;
            if (2 * ix == 2 * kOne) return 1.0;
            if ((2 * ix < 2 * kOne) == !(iy >> 63)) return 0.0;
            return y * y;
        }
        if (2 * ix - 1 >= 2 * kInf - 1) {  // x is 0, inf or nan
            double x2 = x * x;
            if ((ix >> 63) && integer_kind(iy) == 1) x2 = -x2;
            return (iy >> 63) ? 1.0 / x2 : x2;
        }
        if (ix >> 63) {  // finite x < 0
            const int yk = integer_kind(iy);
            if (yk == 0) return (x - x) / (x - x);
            if (yk == 1) sign_bias = 0x800ull << 7;
            ix &= 0x7fffffffffffffffull;
            topx &= 0x7ffu;
        }
        if ((topy & 0x7ffu) - 0x3beu >= 0x43eu - 0x3beu) {  // |y| tiny or huge
            if (ix == kOne) return 1.0;
            if ((topy & 0x7ffu) < 0x3beu) return ix > kOne ? 1.0 + y : 1.0 - y;
            return (ix > kOne) == (topy < 0x800u) ? HUGE_VAL : 0.0;
        }
        if (topx == 0) {  // subnormal x: normalise, exponent becomes negative
            ix = bits_of(x * 0x1p52) & 0x7fffffffffffffffull;
            ix -= 52ull << 52;
        }
    }
    double lo;
    const double hi = log_tail_(ix, &lo);
    const double ehi = y * hi;
    const double elo = fused(y, lo, fused(y, hi, -ehi));
    return exp_tail_(ehi, elo, sign_bias);
}

// rmod's operation (engine/sim_core.hpp:30-35): pow(max(a, 0), 1 + clip(b, 0, 1)).
// On that domain (x >= +0, y in [1, 2] or NaN) glibc's pow reduces to: NaN y
// gives x + y (1 for x == 1), +0 and +inf give x * x, a subnormal x is
// normalised, and the rest is the main path of pow_ above; the branches for
// negative bases and for tiny or huge exponents are left out.
SIDR_HD_CALL double rmod_(double a, double b) {
    const double x = a > 0.0 ? a : 0.0;
    double e = b;
    if (e < 0.0) e = 0.0;
    else if (e > 1.0) e = 1.0;
    const double y = 1.0 + e;
    if (y != y) return x == 1.0 ? 1.0 : x + y;
    uint64_t ix = bits_of(x);
    if (x == 0.0 || ix >= 0x7ff0000000000000ull) return x * x;  // +0 and +inf
    if (ix < 0x0010000000000000ull) {  // subnormal: the exponent becomes negative
        ix = bits_of(x * 0x1p52) & 0x7fffffffffffffffull;
        ix -= 52ull << 52;
    }
    double lo;
    const double hi = log_tail_(ix, &lo);
    const double ehi = y * hi;
    const double elo = fused(y, lo, fused(y, hi, -ehi));
    return exp_tail_(ehi, elo, 0);
}

// ------------------------------------------------------------- erf, erfc

// fdlibm's coefficients.
struct ErfCoef {
    // erf(x) = x + x*PP(z)/QQ(z), z = x^2, |x| < 0.84375
    static constexpr double efx = 1.28379167095512586316e-01;
    static constexpr double pp0 = 1.28379167095512558561e-01, pp1 = -3.25042107247001499370e-01,
                            pp2 = -2.84817495755985104766e-02, pp3 = -5.77027029648944159157e-03,
                            pp4 = -2.37630166566501626084e-05;
    static constexpr double qq1 = 3.97917223959155352819e-01, qq2 = 6.50222499887672944485e-02,
                            qq3 = 5.08130628187576562776e-03, qq4 = 1.32494738004321644526e-04,
                            qq5 = -3.96022827877536812320e-06;
    // erf(x) = erx + PA(s)/QA(s), s = |x|-1, 0.84375 <= |x| < 1.25
    static constexpr double erx = 8.45062911510467529297e-01;
    static constexpr double pa0 = -2.36211856075265944077e-03, pa1 = 4.14856118683748331666e-01,
                            pa2 = -3.72207876035701323847e-01, pa3 = 3.18346619901161753674e-01,
                            pa4 = -1.10894694282396677476e-01, pa5 = 3.54783043256182359371e-02,
                            pa6 = -2.16637559486879084300e-03;
    static constexpr double qa1 = 1.06420880400844228286e-01, qa2 = 5.40397917702171048937e-01,
                            qa3 = 7.18286544141962662868e-02, qa4 = 1.26171219808761642112e-01,
                            qa5 = 1.36370839120290507362e-02, qa6 = 1.19844998467991074170e-02;
    // erfc(x) = exp(-x^2-0.5625+RA(t)/SA(t))/x, t = 1/x^2, 1.25 <= |x| < 1/0.35
    static constexpr double ra0 = -9.86494403484714822705e-03, ra1 = -6.93858572707181764372e-01,
                            ra2 = -1.05586262253232909814e+01, ra3 = -6.23753324503260060396e+01,
                            ra4 = -1.62396669462573470355e+02, ra5 = -1.84605092906711035994e+02,
                            ra6 = -8.12874355063065934246e+01, ra7 = -9.81432934416914548592e+00;
    static constexpr double sa1 = 1.96512716674392571292e+01, sa2 = 1.37657754143519042600e+02,
                            sa3 = 4.34565877475229228821e+02, sa4 = 6.45387271733267880336e+02,
                            sa5 = 4.29008140027567833386e+02, sa6 = 1.08635005541779435134e+02,
                            sa7 = 6.57024977031928170135e+00, sa8 = -6.04244152148580987438e-02;
    // the same with RB/SB, |x| >= 1/0.35
    static constexpr double rb0 = -9.86494292470009928597e-03, rb1 = -7.99283237680523006574e-01,
                            rb2 = -1.77579549177547519889e+01, rb3 = -1.60636384855821916062e+02,
                            rb4 = -6.37566443368389627722e+02, rb5 = -1.02509513161107724954e+03,
                            rb6 = -4.83519191608651397019e+02;
    static constexpr double sb1 = 3.03380607434824582924e+01, sb2 = 3.25792512996573918826e+02,
                            sb3 = 1.53672958608443695994e+03, sb4 = 3.19985821950859553908e+03,
                            sb5 = 2.55305040643316442583e+03, sb6 = 4.74528541206955367215e+02,
                            sb7 = -2.24409524465858183362e+01;
};

// The four rational approximations share one evaluation: every numerator
// and denominator above is a prefix of
//   ((((c0 + t*c1) + t2*(c2 + t*c3)) + t4*(c4 + t*c5)) + t6*(c6 + t*c7)) + t8*(c8 + t*c9)
// with t2 = t*t, t4 = t2*t2, t6 = t4*t2, t8 = t4*t4 (a trailing single term
// such as z4*pp4 is t4*(c4 + t*0)); the missing coefficients are zero, and a
// zero term adds +0, which changes no value, so the result is the same
// double.  One code path for all intervals keeps the lanes of a warp together
// when their arguments fall in different intervals.  Rows: small |x|, mid
// |x|, tail with RA/SA, tail with RB/SB; in each row 10 numerator then 10
// denominator coefficients.
#define SIDR_ERF_ROWS                                                                             \
    {ErfCoef::pp0, ErfCoef::pp1, ErfCoef::pp2, ErfCoef::pp3, ErfCoef::pp4, 0.0, 0.0, 0.0, 0.0, 0.0, \
     1.0, ErfCoef::qq1, ErfCoef::qq2, ErfCoef::qq3, ErfCoef::qq4, ErfCoef::qq5, 0.0, 0.0, 0.0, 0.0, \
     ErfCoef::pa0, ErfCoef::pa1, ErfCoef::pa2, ErfCoef::pa3, ErfCoef::pa4, ErfCoef::pa5,           \
     ErfCoef::pa6, 0.0, 0.0, 0.0,                                                                 \
     1.0, ErfCoef::qa1, ErfCoef::qa2, ErfCoef::qa3, ErfCoef::qa4, ErfCoef::qa5, ErfCoef::qa6,      \
     0.0, 0.0, 0.0,                                                                               \
     ErfCoef::ra0, ErfCoef::ra1, ErfCoef::ra2, ErfCoef::ra3, ErfCoef::ra4, ErfCoef::ra5,           \
     ErfCoef::ra6, ErfCoef::ra7, 0.0, 0.0,                                                        \
     1.0, ErfCoef::sa1, ErfCoef::sa2, ErfCoef::sa3, ErfCoef::sa4, ErfCoef::sa5, ErfCoef::sa6,      \
     ErfCoef::sa7, ErfCoef::sa8, 0.0,                                                             \
     ErfCoef::rb0, ErfCoef::rb1, ErfCoef::rb2, ErfCoef::rb3, ErfCoef::rb4, ErfCoef::rb5,           \
     ErfCoef::rb6, 0.0, 0.0, 0.0,                                                                 \
     1.0, ErfCoef::sb1, ErfCoef::sb2, ErfCoef::sb3, ErfCoef::sb4, ErfCoef::sb5, ErfCoef::sb6,      \
     ErfCoef::sb7, 0.0, 0.0}

#ifdef __CUDACC__
__device__ const double kErfRowsDev[80] = SIDR_ERF_ROWS;
#endif
static const double kErfRowsHost[80] = SIDR_ERF_ROWS;

SIDR_HD double erf_coef(int i) {
#ifdef __CUDA_ARCH__
    return kErfRowsDev[i];
#else
    return kErfRowsHost[i];
#endif
}

// Numerator / denominator of row `row` at t, both pairwise as above.
SIDR_HD double erf_ratio(int row, double t) {
    const int o = row * 20;
    const double t2 = t * t, t4 = t2 * t2, t6 = t4 * t2, t8 = t4 * t4;
    double pq[2];
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const int c = o + 10 * h;
        pq[h] = (erf_coef(c) + t * erf_coef(c + 1)) + t2 * (erf_coef(c + 2) + t * erf_coef(c + 3)) +
                t4 * (erf_coef(c + 4) + t * erf_coef(c + 5)) + t6 * (erf_coef(c + 6) + t * erf_coef(c + 7)) +
                t8 * (erf_coef(c + 8) + t * erf_coef(c + 9));
    }
    return pq[0] / pq[1];
}

// exp(-z^2-0.5625) * exp((z-ax)(z+ax) + rs), z = ax with its low 32 bits
// cleared (so z*z is exact): x*erfc(x) for the tail rows.
SIDR_HD double erf_tail(double ax, double rs) {
    const double z = double_of(bits_of(ax) & 0xffffffff00000000ull);
    return exp_(-z * z - 0.5625) * exp_((z - ax) * (z + ax) + rs);
}

SIDR_HD_CALL double erf_(double x) {
    using C = ErfCoef;
    const uint64_t u = bits_of(x);
    const bool neg = (u >> 63) != 0;
    const uint32_t ix = (uint32_t)(u >> 32) & 0x7fffffffu;  // high word of |x|
    if (ix >= 0x7ff00000u) return (neg ? -1.0 : 1.0) + 1.0 / x;  // nan, +-inf
    if (ix < 0x3e300000u) {                                      // |x| < 2^-28
        if (ix < 0x00800000u) return 0.0625 * (16.0 * x + (16.0 * C::efx) * x);
        return x + C::efx * x;
    }
    if (ix >= 0x40180000u) return neg ? 1e-300 - 1.0 : 1.0 - 1e-300;  // |x| >= 6
    const double ax = fabs(x);
    const int row = ix < 0x3feb0000u ? 0 : ix < 0x3ff40000u ? 1 : ix < 0x4006DB6Eu ? 2 : 3;
    const double t = row == 0 ? x * x : row == 1 ? ax - 1.0 : 1.0 / (ax * ax);
    const double pq = erf_ratio(row, t);
    if (row == 0) return x + x * pq;                              // |x| < 0.84375
    if (row == 1) return neg ? -C::erx - pq : C::erx + pq;        // |x| < 1.25
    const double r = erf_tail(ax, pq);                            // |x| < 6
    return neg ? r / ax - 1.0 : 1.0 - r / ax;
}

SIDR_HD_CALL double erfc_(double x) {
    using C = ErfCoef;
    const uint64_t u = bits_of(x);
    const bool neg = (u >> 63) != 0;
    const uint32_t hx = (uint32_t)(u >> 32);
    const uint32_t ix = hx & 0x7fffffffu;
    if (ix >= 0x7ff00000u) return (double)(neg ? 2 : 0) + 1.0 / x;  // nan, +-inf
    if (ix < 0x3c700000u) return 1.0 - x;                           // |x| < 2^-56
    if (ix >= 0x403c0000u) return neg ? 2.0 - 1e-300 : 1e-300 * 1e-300;  // |x| >= 28
    if (neg && ix >= 0x40180000u) return 2.0 - 1e-300;                // x <= -6
    const double ax = fabs(x);
    const int row = ix < 0x3feb0000u ? 0 : ix < 0x3ff40000u ? 1 : ix < 0x4006DB6Du ? 2 : 3;
    const double t = row == 0 ? x * x : row == 1 ? ax - 1.0 : 1.0 / (ax * ax);
    const double pq = erf_ratio(row, t);
    if (row == 0) {  // |x| < 0.84375
        if ((int32_t)hx < 0x3fd00000) return 1.0 - (x + x * pq);  // x < 1/4
        double r = x * pq;
        r += (x - 0.5);
        return 0.5 - r;
    }
    if (row == 1) return neg ? 1.0 + (C::erx + pq) : (1.0 - C::erx) - pq;  // |x| < 1.25
    const double r = erf_tail(ax, pq);                                     // |x| < 28
    return neg ? 2.0 - r / ax : r / ax;
}

}  // namespace libm
}  // namespace sidr
