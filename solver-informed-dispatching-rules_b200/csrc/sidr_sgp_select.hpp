// sidr_sgp_select.hpp -- the host-side statistics and screening rules of the
// surrogate-assisted GP driver (sidr_sgp.cpp): ranks, Spearman's rho, the
// model's training targets and the choice of screened offspring.  Header-only
// so that a CPU test program can check them directly.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <numeric>
#include <set>
#include <vector>

namespace sidr {
namespace sgp {

// Ranks (0-based) with ties sharing their average rank.
inline std::vector<double> ranks_of(const std::vector<double>& x) {
    const size_t n = x.size();
    std::vector<size_t> o(n);
    std::iota(o.begin(), o.end(), 0);
    std::stable_sort(o.begin(), o.end(), [&](size_t a, size_t b) { return x[a] < x[b]; });
    std::vector<double> r(n);
    for (size_t i = 0; i < n;) {
        size_t j = i;
        while (j + 1 < n && x[o[j + 1]] == x[o[i]]) j++;
        const double avg = 0.5 * (double)(i + j);
        for (size_t k = i; k <= j; k++) r[o[k]] = avg;
        i = j + 1;
    }
    return r;
}

// Spearman's rank correlation (Pearson correlation of the ranks); 0 when
// either side is constant.
inline double spearman(const std::vector<double>& a, const std::vector<double>& b) {
    const std::vector<double> ra = ranks_of(a), rb = ranks_of(b);
    const double n = (double)a.size();
    double ma = 0, mb = 0;
    for (size_t i = 0; i < a.size(); i++) {
        ma += ra[i];
        mb += rb[i];
    }
    ma /= n;
    mb /= n;
    double sab = 0, saa = 0, sbb = 0;
    for (size_t i = 0; i < a.size(); i++) {
        sab += (ra[i] - ma) * (rb[i] - mb);
        saa += (ra[i] - ma) * (ra[i] - ma);
        sbb += (rb[i] - mb) * (rb[i] - mb);
    }
    if (saa <= 0 || sbb <= 0) return 0.0;
    return sab / std::sqrt(saa * sbb);
}

// Training targets from simulated fitness: target 1, the ranks as uniform
// scores ((r + 0.5) / n - 0.5) * sqrt(12) (mean 0, variance 1 without ties);
// otherwise the fitness standardised by its mean and standard deviation.
inline std::vector<float> training_targets(const std::vector<double>& fit, int target) {
    std::vector<float> y;
    y.reserve(fit.size());
    const double cnt = (double)fit.size();
    if (target == 1) {
        for (double r : ranks_of(fit)) y.push_back((float)(((r + 0.5) / cnt - 0.5) * std::sqrt(12.0)));
        return y;
    }
    double mu = 0, sd = 0;
    for (double v : fit) mu += v;
    mu /= cnt;
    for (double v : fit) sd += (v - mu) * (v - mu);
    sd = std::sqrt(sd / cnt) + 1e-9;
    for (double v : fit) y.push_back((float)((v - mu) / sd));
    return y;
}

// Up to `need` offspring indices in order of decreasing prediction (ties in
// index order), at most one per key(c); when fewer distinct keys exist than
// slots, the best-predicted of the remaining offspring fill the rest.
template <class Key, class KeyOf>
std::vector<int> best_distinct(const std::vector<float>& pred, size_t need, KeyOf key_of) {
    std::vector<int> co(pred.size());
    std::iota(co.begin(), co.end(), 0);
    std::stable_sort(co.begin(), co.end(), [&](int a, int b) { return pred[a] > pred[b]; });
    std::set<Key> seen;
    std::vector<char> taken(pred.size(), 0);
    std::vector<int> out;
    for (size_t k = 0; out.size() < need && k < co.size(); k++)
        if (seen.insert(key_of(co[k])).second) {
            out.push_back(co[k]);
            taken[co[k]] = 1;
        }
    for (size_t k = 0; out.size() < need && k < co.size(); k++)
        if (!taken[co[k]]) out.push_back(co[k]);
    return out;
}

// Pre-selection: for q < need, the best-predicted offspring (first on ties)
// of the group [q*per, (q+1)*per), per = max(1, count / need).
inline std::vector<int> preselect(const std::vector<float>& pred, int need) {
    std::vector<int> out;
    const int count = (int)pred.size();
    const int per = std::max(1, count / std::max(need, 1));
    for (int q = 0; q < need; q++) {
        int b = q * per;
        if (b >= count) break;
        for (int c = q * per + 1; c < (q + 1) * per && c < count; c++)
            if (pred[c] > pred[b]) b = c;
        out.push_back(b);
    }
    return out;
}

}  // namespace sgp
}  // namespace sidr
