// Compares sidr::libm::{erf_, erfc_, exp_, pow_} (csrc/sidr_libm.cuh) with the
// host C library bit for bit over random arguments in every interval of the
// algorithms.  Usage: libm_check <samples per interval> <seed>; prints one line
// per interval "name lo hi mismatches samples" and exits 1 on any mismatch.
// For pow the interval is a family of (x, y) pairs, named by its number.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "sidr_libm.cuh"

namespace {

uint64_t g_state = 88172645463325252ull;
uint64_t next_u64() {
    g_state ^= g_state << 13;
    g_state ^= g_state >> 7;
    g_state ^= g_state << 17;
    return g_state;
}
double uniform(double a, double b) { return a + (b - a) * ((next_u64() >> 11) * 0x1p-53); }
uint64_t bits(double x) {
    uint64_t u;
    std::memcpy(&u, &x, 8);
    return u;
}

struct Range {
    const char* fn;
    double lo, hi;
};

double ours(const char* fn, double x) {
    if (fn[1] == 'x') return sidr::libm::exp_(x);
    if (fn[3] == 'c') return sidr::libm::erfc_(x);
    return sidr::libm::erf_(x);
}
double theirs(const char* fn, double x) {
    if (fn[1] == 'x') return std::exp(x);
    if (fn[3] == 'c') return std::erfc(x);
    return std::erf(x);
}

}  // namespace

int main(int argc, char** argv) {
    const long n = argc > 1 ? std::atol(argv[1]) : 1000000;
    if (argc > 2) g_state ^= (uint64_t)std::atoll(argv[2]) * 0x9e3779b97f4a7c15ull;
    const Range ranges[] = {
        {"erf", -0x1p-1020, 0x1p-1020}, {"erf", -0x1p-27, 0x1p-27}, {"erf", -0.84375, 0.84375},
        {"erf", 0.84375, 1.25},         {"erf", -1.25, -0.84375},   {"erf", 1.25, 2.857142857142857},
        {"erf", 2.857142857142857, 6.0}, {"erf", -6.0, -1.25},      {"erf", -9.0, 9.0},
        {"erfc", -0x1p-55, 0x1p-55},    {"erfc", -0.25, 0.25},      {"erfc", 0.25, 0.84375},
        {"erfc", -0.84375, -0.25},      {"erfc", 0.84375, 1.25},    {"erfc", -1.25, -0.84375},
        {"erfc", 1.25, 2.857142857142857}, {"erfc", 2.857142857142857, 6.0}, {"erfc", 6.0, 28.0},
        {"erfc", -6.5, -1.25},          {"erfc", 26.0, 30.0},       {"erfc", -40.0, 40.0},
        {"exp", -0x1p-50, 0x1p-50},     {"exp", -1.0, 1.0},         {"exp", -40.0, 1.0},
        {"exp", -745.5, -512.0},        {"exp", 512.0, 709.7},      {"exp", -800.0, 800.0},
    };
    int bad_total = 0;
    for (const Range& r : ranges) {
        long bad = 0;
        for (long k = 0; k < n; k++) {
            const double x = uniform(r.lo, r.hi);
            const double a = ours(r.fn, x), b = theirs(r.fn, x);
            if (bits(a) != bits(b)) {
                if (bad < 2) std::printf("# %s(%a): ours %a libc %a\n", r.fn, x, a, b);
                bad++;
            }
        }
        const double special[] = {0.0, -0.0, 1.0, -1.0, 0.84375, 1.25, 6.0, -6.0, 28.0, 0x1p-1074,
                                  INFINITY, -INFINITY};
        for (double x : special)
            if (bits(ours(r.fn, x)) != bits(theirs(r.fn, x))) bad++;
        std::printf("%s %a %a %ld %ld\n", r.fn, r.lo, r.hi, bad, n);
        bad_total += bad != 0;
    }
    // pow: families of (x, y); the first ones cover rmod's arguments
    // (x >= 0, y = 1 + clip(b, 0, 1))
    auto pow_pair = [](int fam, double& x, double& y) {
        switch (fam) {
        case 0: x = std::exp2(uniform(-30.0, 30.0)); y = uniform(1.0, 2.0); break;
        case 1: x = uniform(0.5, 2.0); y = uniform(1.0, 2.0); break;
        case 2: x = std::exp2(uniform(-1074.0, 1023.9)); y = uniform(1.0, 2.0); break;
        case 3: x = (double)(1 + next_u64() % 1000000) / (double)(1 + next_u64() % 1000);
                y = 1.0 + (double)(next_u64() % 1001) / 1000.0; break;
        case 4: x = std::exp2(uniform(-1022.0, 1023.9)); y = uniform(-8.0, 8.0); break;
        case 5: { uint64_t u = next_u64() & 0x000fffffffffffffull; std::memcpy(&x, &u, 8); }
                y = uniform(0.5, 2.0); break;
        default: x = -std::exp2(uniform(-10.0, 10.0));
                 y = (double)(long)uniform(-10.0, 10.0) + ((next_u64() & 1) ? 0.5 : 0.0); break;
        }
    };
    for (int fam = 0; fam < 7; fam++) {
        long bad = 0;
        for (long k = 0; k < n; k++) {
            double x, y;
            pow_pair(fam, x, y);
            const double a = sidr::libm::pow_(x, y), b = std::pow(x, y);
            if (bits(a) != bits(b) && !(a != a && b != b)) {
                if (bad < 2) std::printf("# pow(%a, %a): ours %a libc %a\n", x, y, a, b);
                bad++;
            }
        }
        std::printf("pow family%d - %ld %ld\n", fam, bad, n);
        bad_total += bad != 0;
    }
    {  // special operands
        const double xs[] = {0.0, -0.0, 1.0, -1.0, 2.0, 0.5, 0x1p-1074, 0x1p-1022, 1e308, INFINITY,
                             -INFINITY, NAN, -2.0, 3.5};
        const double ys[] = {0.0, -0.0, 1.0, 2.0, 1.5, -1.0, 0.5, 3.0, 1e-300, 1e300, INFINITY,
                             -INFINITY, NAN, 1075.0, -1075.0};
        long bad = 0, cnt = 0;
        for (double x : xs)
            for (double y : ys) {
                const double a = sidr::libm::pow_(x, y), b = std::pow(x, y);
                cnt++;
                if (bits(a) != bits(b) && !(a != a && b != b)) {
                    std::printf("# pow(%a, %a): ours %a libc %a\n", x, y, a, b);
                    bad++;
                }
            }
        std::printf("pow specials - %ld %ld\n", bad, cnt);
        bad_total += bad != 0;
    }
    {  // rmod_ (a, b) -> pow(max(a, 0), 1 + clip(b, 0, 1)) on every kind of operand
        long bad = 0;
        const double special[] = {0.0, -0.0, 1.0, -1.0, 0.5, 2.0, 5e-324, 1e-310, 1e308, INFINITY,
                                  -INFINITY, NAN, -NAN, 1.5, 3.0};
        auto check = [&](double a, double b) {
            const double x = a > 0.0 ? a : 0.0;
            const double e = b < 0.0 ? 0.0 : (b > 1.0 ? 1.0 : b);
            // a volatile exponent: where the clamp gives 2, the compiler would otherwise
            // fold pow(x, 2.0) into x * x, which is not what the C library returns
            volatile double y = 1.0 + e;
            const double want = std::pow(x, (double)y), got = sidr::libm::rmod_(a, b);
            if (bits(got) != bits(want) && !(got != got && want != want)) {
                if (bad < 2) std::printf("# rmod(%a, %a): ours %a libc %a\n", a, b, got, want);
                bad++;
            }
        };
        for (double a : special)
            for (double b : special) check(a, b);
        for (long k = 0; k < n; k++) {
            const double mag = std::exp2(uniform(-1074.0, 1023.9));
            const double a = (next_u64() & 3) == 0 ? -mag : mag;
            const double b = uniform(-0.5, 1.5);
            check(a, b);
        }
        std::printf("rmod all - %ld %ld\n", bad, n);
        bad_total += bad != 0;
    }
    return bad_total ? 1 : 0;
}
