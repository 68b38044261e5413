// Host build of the on-device sampler's Box-Muller step (csrc/sidr_sample.cuh)
// against the C library, the way the reference computes it (engine/rng.hpp:
// 135-147, engine/sim_host.hpp:43-47):
//   * log, sin, cos: whenever the double-double value names one candidate, it
//     is the C library's result; when it names two, the result is one of them;
//   * durations: every pair the header settles equals the C library's pair.
// Arguments: pairs, seed.  Prints one row per check: name, checked, settled,
// mismatches; exits 1 on any mismatch.
#include <cstdio>
#include <cstdlib>
#include <random>

#include "sidr_gp_core.hpp"
#include "sidr_sample.cuh"

using namespace sidr::smp;

// The device generator's pieces replayed on the host -- the seeding, a state
// refresh in its three phases (each computes its words, then stores them),
// tempering and the 53-bit draw -- against the host generator's stream for
// two refreshes per seed.  Returns the number of differing outputs.
static long long check_generator(unsigned long long seed) {
    uint32_t mt[kMtN];
    mt_seed(mt, seed);
    sidr::gp::Mt19937 ref(seed);
    long long bad = 0;
    for (int blk = 0; blk < 2; blk++) {
        const int lo[3] = {0, kMtN - kMtM, 2 * (kMtN - kMtM)};
        const int hi[3] = {kMtN - kMtM, 2 * (kMtN - kMtM), kMtN - 1};
        for (int ph = 0; ph < 3; ph++) {
            uint32_t nv[kMtN];
            for (int kk = lo[ph]; kk < hi[ph]; kk++) nv[kk] = mt_refreshed(mt, kk);
            for (int kk = lo[ph]; kk < hi[ph]; kk++) mt[kk] = nv[kk];
        }
        mt[kMtN - 1] = mt_refreshed_last(mt);
        for (int k = 0; k < kMtN; k += 2) {
            const uint32_t a = ref.next(), b = ref.next();
            const double want = ((double)(a >> 5) * 67108864.0 + (double)(b >> 6)) * (1.0 / 9007199254740992.0);
            bad += mt_temper(mt[k]) != a || mt_temper(mt[k + 1]) != b || mt_draw(mt[k], mt[k + 1]) != want;
        }
    }
    return bad;
}

int main(int argc, char** argv) {
    const long long N = argc > 1 ? std::atoll(argv[1]) : 100000;
    const unsigned long long seed = argc > 2 ? std::strtoull(argv[2], nullptr, 10) : 1;
    std::mt19937_64 g(seed);
    auto u53 = [&]() { return (double)(g() >> 11) * (1.0 / 9007199254740992.0); };
    constexpr double kTwoPi = 2.0 * 3.14159265358979323846;
    const double mus[] = {10.0, 1.0, 37.5, 0.3, 90.0, 5.0, 20.0};
    long long fn_checked[3] = {0, 0, 0}, fn_one[3] = {0, 0, 0}, fn_bad[3] = {0, 0, 0};
    long long pairs = 0, settled = 0, bad = 0;
    for (long long i = 0; i < N + 8; i++) {
        double u1 = u53(), u2 = u53();
        if (i >= N) {  // edges: zero draws and the largest draw below 1
            const double edge[] = {0.0, 0.0, 1.0 - 1.0 / 9007199254740992.0, 0.25, 0.5, 0.75, 0.125, 0.999};
            u1 = edge[i - N];
            u2 = edge[(i - N + 3) % 8];
            if (i == N) u2 = 0.0;
        }
        const double x2pi = u1 * kTwoPi, y = 1.0 - u2;
        const dd lg = log_dd(y);
        dd sn, cs;
        sincos_dd(x2pi, sn, cs);
        const double lib[3] = {std::log(y), std::sin(x2pi), std::cos(x2pi)};
        const dd mine[3] = {lg, sn, cs};
        const double guard[3] = {kGuardLog, kGuardTrig, kGuardTrig};
        for (int f = 0; f < 3; f++) {
            double c[2];
            const int k = candidates(mine[f], guard[f], c);
            fn_checked[f]++;
            fn_one[f] += k == 1;
            if (lib[f] != c[0] && lib[f] != c[1]) {
                fn_bad[f]++;
                if (fn_bad[f] <= 3)
                    std::printf("# f%d arg %a lib %a mine %a + %a\n", f, f == 0 ? y : x2pi, lib[f], mine[f].hi,
                                mine[f].lo);
            }
        }
        // the reference's pair: z = cos * g2rad, then sin * g2rad
        const double g2rad = std::sqrt(-2.0 * std::log(1.0 - u2));
        const double z0 = std::cos(x2pi) * g2rad, z1 = std::sin(x2pi) * g2rad;
        for (double mu0 : mus) {
            const double mu1 = mus[(i + 3) % 7], sd0 = 0.2 * mu0, sd1 = 0.2 * mu1;
            const bool has1 = (i % 5) != 0;
            double v0 = mu0 + z0 * sd0, v1 = mu1 + z1 * sd1;
            v0 = v0 > 0.0 ? v0 : 0.0;
            v1 = v1 > 0.0 ? v1 : 0.0;
            double d0, d1;
            const bool ok = gauss_pair_durations(u1, u2, mu0, sd0, has1, mu1, sd1, d0, d1);
            pairs++;
            if (ok) {
                settled++;
                if (d0 != v0 || (has1 && d1 != v1)) {
                    bad++;
                    if (bad <= 3) std::printf("# pair u1 %a u2 %a mu %g: %a %a vs %a %a\n", u1, u2, mu0, d0, d1, v0, v1);
                }
            }
        }
    }
    long long gen_bad = 0;
    const unsigned long long seeds[] = {0ull, 1ull, 5ull, 123456789ull, 1000000ull, (1ull << 32) + 5ull,
                                        0xffffffffull, seed * 7919ull};
    for (unsigned long long sd : seeds) gen_bad += check_generator(sd);
    std::printf("generator %d %d %lld\n", (int)(sizeof seeds / sizeof seeds[0]), 2 * kMtN, gen_bad);
    const char* names[3] = {"log", "sin", "cos"};
    for (int f = 0; f < 3; f++) std::printf("%s %lld %lld %lld\n", names[f], fn_checked[f], fn_one[f], fn_bad[f]);
    std::printf("pairs %lld %lld %lld\n", pairs, settled, bad);
    return (bad || gen_bad || fn_bad[0] || fn_bad[1] || fn_bad[2]) ? 1 : 0;
}
