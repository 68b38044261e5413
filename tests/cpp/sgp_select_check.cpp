// Checks the surrogate driver's host rules (csrc/sidr_sgp_select.hpp) on
// fixed inputs; prints "ok" or the first failed check and exits non-zero.
#include <cmath>
#include <cstdio>
#include <vector>

#include "sidr_sgp_select.hpp"

using namespace sidr::sgp;

static int fails = 0;
#define CHECK(c)                                                   \
    do {                                                           \
        if (!(c)) {                                                \
            std::printf("failed: %s (line %d)\n", #c, __LINE__);   \
            fails++;                                               \
        }                                                          \
    } while (0)

int main() {
    // ranks with ties averaged
    const std::vector<double> x = {3.0, 1.0, 3.0, 2.0, 5.0};
    const std::vector<double> r = ranks_of(x);
    CHECK(r[1] == 0.0 && r[3] == 1.0 && r[0] == 2.5 && r[2] == 2.5 && r[4] == 4.0);

    // Spearman: monotone maps give 1, reversal -1, a constant side 0
    const std::vector<double> a = {1, 2, 3, 4, 5, 6}, b = {10, 20, 25, 40, 41, 90};
    std::vector<double> rev(a.rbegin(), a.rend()), flat(6, 7.0);
    CHECK(std::fabs(spearman(a, b) - 1.0) < 1e-15);
    CHECK(std::fabs(spearman(a, rev) + 1.0) < 1e-15);
    CHECK(spearman(a, flat) == 0.0);

    // rank targets: order kept, mean 0, variance 1 without ties, skew gone
    std::vector<double> fit = {0.0, 0.0001, 2400.0, 2350.0, 1.0, 2410.0, 2300.0, 5.0};
    const std::vector<float> y = training_targets(fit, 1);
    double m = 0, v = 0;
    for (float t : y) m += t;
    m /= y.size();
    for (float t : y) v += (t - m) * (t - m);
    v /= y.size();
    CHECK(std::fabs(m) < 1e-6);
    CHECK(std::fabs(v - (1.0 - 1.0 / 64.0)) < 1e-5);  // uniform scores of n = 8: 1 - 1/n^2
    const std::vector<double> rf = ranks_of(fit);
    for (size_t i = 0; i < fit.size(); i++)
        for (size_t j = 0; j < fit.size(); j++)
            if (fit[i] < fit[j]) CHECK(y[i] < y[j]);
    const std::vector<float> z = training_targets(fit, 0);
    double mz = 0;
    for (float t : z) mz += t;
    CHECK(std::fabs(mz / z.size()) < 1e-6);

    // best distinct: one per key in prediction order, ties by index, then the rest
    const std::vector<float> pred = {0.5f, 0.9f, 0.9f, 0.1f, 0.7f, 0.3f};
    const std::vector<int> key = {0, 1, 1, 2, 1, 3};  // offspring 1, 2 and 4 behave alike
    std::vector<int> pick = best_distinct<int>(pred, 4, [&](int c) { return key[c]; });
    CHECK((pick == std::vector<int>{1, 0, 5, 3}));
    pick = best_distinct<int>(pred, 6, [&](int c) { return key[c]; });
    CHECK((pick == std::vector<int>{1, 0, 5, 3, 2, 4}));
    pick = best_distinct<int>(pred, 2, [&](int c) { return c; });
    CHECK((pick == std::vector<int>{1, 2}));
    CHECK(best_distinct<int>(pred, 0, [&](int c) { return c; }).empty());

    // pre-selection: best of each group of count / need
    const std::vector<float> p2 = {0.1f, 0.4f, 0.4f, 0.2f, 0.9f, 0.0f, 0.3f, 0.3f};
    CHECK((preselect(p2, 4) == std::vector<int>{1, 2, 4, 6}));
    CHECK((preselect(p2, 2) == std::vector<int>{1, 4}));
    CHECK((preselect(p2, 8) == std::vector<int>{0, 1, 2, 3, 4, 5, 6, 7}));
    CHECK(preselect(p2, 0).empty());

    if (fails) return 1;
    std::printf("ok\n");
    return 0;
}
