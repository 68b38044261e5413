// sidr_host.cpp -- host-side preparation for the evaluator (see sidr_host.hpp).
// Build with -ffp-contract=off: the tables must reproduce the reference's
// IEEE operations one by one.
#include "sidr_host.hpp"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <map>
#include <thread>

namespace sidr {

namespace {

// Monotone map of doubles onto uint64 (total order, -0 just below +0).
inline uint64_t okey(double x) {
    uint64_t u;
    std::memcpy(&u, &x, 8);
    return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}
inline double from_okey(uint64_t k) {
    uint64_t u = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
    double x;
    std::memcpy(&x, &u, 8);
    return x;
}

// Largest finite double x with pred(x), for a predicate that holds on a
// down-set; -inf when it holds nowhere.
template <class Pred>
double largest_true(Pred pred) {
    if (!pred(-DBL_MAX)) return -INFINITY;
    if (pred(DBL_MAX)) return DBL_MAX;
    uint64_t lo = okey(-DBL_MAX), hi = okey(DBL_MAX);
    while (hi - lo > 1) {
        const uint64_t mid = lo + (hi - lo) / 2;
        if (pred(from_okey(mid))) lo = mid;
        else hi = mid;
    }
    return from_okey(lo);
}

// The standard and robust neighbour tests of engine/sim_terms.hpp, verbatim in
// their arithmetic: true when the neighbour can be served after arriving at a.
struct Tests {
    const HostInstance& h;
    bool std_ok(int j, double a) const {
        if (a > h.close_t[j]) return false;
        const double st = a > h.open_t[j] ? a : h.open_t[j];
        return !(st + h.durations[j] + h.d2d[j] > h.tmax);
    }
    bool rob_ok(int j, double a) const {
        if (a > h.close_t[j]) return false;
        const double st = a > h.open_t[j] ? a : h.open_t[j];
        return !(st + h.durations[j] * (1.0 + kSigma) + h.d2d[j] > h.tmax);
    }
};

inline double D(const HostInstance& h, int a, int b) { return h.dist[(size_t)a * (h.n + 1) + b]; }

// t_reach2 / t_regret / t_eloss_chance at the initial state, for zstats
// (engine/sim_terms.hpp:95-127, 36-54, 225-257; nothing visited).
double z_reach2(const HostInstance& h, int i, double fin) {
    const Tests T{h};
    double bv = 0.0, fj = 0.0;
    int bj = -1;
    for (int j = 0; j < h.n; j++) {
        if (j == i) continue;
        const double t = D(h, i + 1, j + 1);
        if (t < 1e-10) continue;
        const double a = fin + t;
        if (!T.std_ok(j, a)) continue;
        const double v = h.scores[j] / t;
        if (v > bv) {
            bv = v;
            bj = j;
            const double st = a > h.open_t[j] ? a : h.open_t[j];
            fj = st + h.durations[j];
        }
    }
    if (bj < 0) return 0.0;
    double bv2 = 0.0, s2 = 0.0;
    for (int k = 0; k < h.n; k++) {
        if (k == i || k == bj) continue;
        const double t = D(h, bj + 1, k + 1);
        if (t < 1e-10) continue;
        if (!T.std_ok(k, fj + t)) continue;
        const double v = h.scores[k] / t;
        if (v > bv2) {
            bv2 = v;
            s2 = h.scores[k];
        }
    }
    return h.scores[bj] + s2;
}

double z_regret(const HostInstance& h, int i, double fin) {
    const Tests T{h};
    double acc = 0.0;
    for (int j = 0; j < h.n; j++) {
        if (j == i) continue;
        if (!T.std_ok(j, 0.0 + D(h, 0, j + 1))) continue;
        if (!T.std_ok(j, fin + D(h, i + 1, j + 1))) acc += h.scores[j];
    }
    return acc;
}

double z_atrisk(const HostInstance& h, int c) {
    const double arr_c = 0.0 + D(h, 0, c + 1);
    const double st_c = arr_c > h.open_t[c] ? arr_c : h.open_t[c];
    const double mfin = st_c + h.durations[c];
    const double sd_c = kSigma * h.durations[c];
    double acc = 0.0;
    for (int j = 0; j < h.n; j++) {
        if (j == c) continue;
        if (0.0 + D(h, 0, j + 1) > h.close_t[j]) continue;
        const double marr = mfin + D(h, c + 1, j + 1);
        double pw;
        if (sd_c > 1e-9) pw = 0.5 * (1.0 + std::erf(((h.close_t[j] - marr) / sd_c) * 0.7071067811865476));
        else pw = marr <= h.close_t[j] ? 1.0 : 0.0;
        double mst, vst;
        if (marr > h.open_t[j]) {
            mst = marr;
            vst = sd_c * sd_c;
        } else {
            mst = h.open_t[j];
            vst = 0.0;
        }
        const double sd_j = kSigma * h.durations[j];
        const double vb = vst + sd_j * sd_j;
        const double mb = mst + h.durations[j] + h.d2d[j];
        double pb;
        if (vb > 1e-18) pb = 0.5 * (1.0 + std::erf(((h.tmax - mb) / std::pow(vb, 0.5)) * 0.7071067811865476));
        else pb = mb <= h.tmax ? 1.0 : 0.0;
        acc += h.scores[j] * (1.0 - pw * pb);
    }
    return acc;
}

// ATRISK's classification of the pair (candidate c, customer j) when the
// candidate finishes at f: the kernel's at_risk_compute, operation for
// operation.  0: the term is +0 (both factors exactly 1); 1: the term is
// s_j (a factor exactly 0); 2: a factor needs erf.
int atrisk_outcome(const HostInstance& h, int c, int j, double f) {
    const double sd_c = kSigma * h.durations[c];
    const double hw = 8.5 * sd_c, lw = -8.5 * sd_c;
    const double cj = h.close_t[j], oj = h.open_t[j], dj = h.durations[j], ej = h.d2d[j];
    const double marr = f + D(h, c + 1, j + 1);
    const double dw = cj - marr;
    const bool sdv = sd_c > 1e-9;
    const bool ew = sdv && !(dw >= hw) && !(dw <= lw);
    const bool pw1 = sdv ? dw >= hw : marr <= cj;
    const bool late = marr > oj;
    const double mst = late ? marr : oj;
    const double pv = late ? h.P1[(size_t)c * h.n + j] : h.P0[j];
    const double mb = mst + dj + ej;
    const double db = h.tmax - mb;
    const bool pvv = pv >= 0.0;
    const double hb = 8.5 * pv, lb = -8.5 * pv;
    const bool eb = (ew || pw1) && pvv && !(db >= hb) && !(db <= lb);
    const bool pb1 = pvv ? db >= hb : mb <= h.tmax;
    if (ew || eb) return 2;
    return (pw1 && pb1) ? 0 : 1;
}

// The outcome of a pair as a step function of f.  Every test above is a
// monotone function of f (each operation is round-to-nearest and monotone),
// and so are the late branch's tests taken on their own; the outcome only
// changes where one of them does.  Those points are found by bisection; the
// outcome between them is taken at one point of each interval.  Stored as
// {k0, k1} and a code byte: interval i is (k_{i-1}, k_i] (k_{-1} = -inf,
// k_2 = +inf, unused points +inf) and its outcome is bits 2i..2i+1 of the
// byte; when more than three intervals remain after merging equal neighbours,
// the last kept interval is given outcome 2 (the kernel then classifies the
// pair itself).
void atrisk_steps(const HostInstance& h, int c, int j, double* ks_out, uint8_t* code_out) {
    const double t = D(h, c + 1, j + 1);
    const double sd_c = kSigma * h.durations[c];
    const double hw = 8.5 * sd_c, lw = -8.5 * sd_c;
    const double cj = h.close_t[j], oj = h.open_t[j], dj = h.durations[j], ej = h.d2d[j];
    const double p1 = h.P1[(size_t)c * h.n + j];
    const bool sdv = sd_c > 1e-9;
    std::vector<double> pts;
    auto add_pt = [&](double k) {
        if (k > -DBL_MAX && k < DBL_MAX) pts.push_back(k);
    };
    // p_win exactly 1 (a down-set), exactly 0 (an up-set)
    add_pt(largest_true([&](double f) {
        const double m = f + t;
        return sdv ? (cj - m) >= hw : m <= cj;
    }));
    if (sdv) add_pt(largest_true([&](double f) { return !((cj - (f + t)) <= lw); }));
    // late arrival (an up-set) and, on the late branch, p_bud exactly 1 (down) or 0 (up)
    add_pt(largest_true([&](double f) { return !((f + t) > oj); }));
    add_pt(largest_true([&](double f) {
        const double mb = (f + t) + dj + ej;
        return p1 >= 0.0 ? (h.tmax - mb) >= 8.5 * p1 : mb <= h.tmax;
    }));
    if (p1 >= 0.0) add_pt(largest_true([&](double f) { return !((h.tmax - ((f + t) + dj + ej)) <= -8.5 * p1); }));
    std::sort(pts.begin(), pts.end());
    pts.erase(std::unique(pts.begin(), pts.end()), pts.end());
    // outcome of each interval at one of its points (interval i ends at pts[i],
    // the last one at +inf), then equal neighbours merged
    std::vector<int> codes;
    std::vector<double> ends;  // right end of each merged interval
    for (size_t i = 0; i <= pts.size(); i++) {
        const double end = i < pts.size() ? pts[i] : INFINITY;
        const double rep = i < pts.size() ? pts[i] : (pts.empty() ? 0.0 : std::nextafter(pts.back(), INFINITY));
        const int o = atrisk_outcome(h, c, j, rep);
        if (!codes.empty() && codes.back() == o) {
            ends.back() = end;
        } else {
            codes.push_back(o);
            ends.push_back(end);
        }
    }
    std::vector<double> ks(ends.begin(), ends.end() - 1);  // the last interval ends at +inf
    if (codes.size() > 3) {
        codes.resize(3);
        codes[2] = 2;
        ks.resize(2);
    }
    uint32_t code = 0;
    for (size_t i = 0; i < codes.size(); i++) code |= (uint32_t)codes[i] << (2 * i);
    for (int i = 0; i < 2; i++) ks_out[i] = i < (int)ks.size() ? ks[i] : INFINITY;
    *code_out = (uint8_t)code;
}

}  // namespace

void atrisk_table_check(const HostInstance& h, int seed, long long& checked, long long& bad) {
    checked = bad = 0;
    uint64_t x = 0x9e3779b97f4a7c15ull * (uint64_t)(seed + 1);
    auto rnd = [&]() {  // splitmix64 in [0, 1)
        x += 0x9e3779b97f4a7c15ull;
        uint64_t z = x;
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
        z ^= z >> 31;
        return (double)(z >> 11) * (1.0 / 9007199254740992.0);
    };
    const int n = h.n;
    for (int c = 0; c < n; c++)
        for (int j = 0; j < n; j++) {
            if (c == j) continue;
            const double* ta = &h.TK[2 * ((size_t)j * n + c)];
            std::vector<double> fs = {0.0};
            for (int k = 0; k < 2; k++)
                if (std::isfinite(ta[k]))
                    for (double v : {std::nextafter(ta[k], -INFINITY), ta[k], std::nextafter(ta[k], INFINITY)})
                        if (v >= 0.0) fs.push_back(v);
            for (int r = 0; r < 6; r++) fs.push_back(rnd() * 2.0 * h.tmax);
            const int codes = h.TC[(size_t)j * n + c];
            for (double f : fs) {
                const int iv = (f > ta[0]) + (f > ta[1]);
                const int code = (codes >> (2 * iv)) & 3;
                checked++;
                if (code != 2 && code != atrisk_outcome(h, c, j, f)) bad++;
            }
        }
}

std::string build_instance(int n, int m, double tmax, const double* scores,
                           const double* durations, const double* open_t, const double* close_t,
                           const double* dist, const double* d2d, HostInstance& h,
                           bool tables) {
    if (n < 1 || n > kMaxN) return "n must be in 1..512";
    if (m < 0 || m > (1 << 20)) return "m must be in 0..2^20";
    if (!scores || !durations || !open_t || !close_t || !dist || !d2d) return "null instance array";
    if (!std::isfinite(tmax)) return "tmax is not finite";
    const int ld = n + 1;
    h.n = n;
    h.m = m;
    h.nw = (n + 31) / 32;
    h.tmax = tmax;
    h.scores.assign(scores, scores + n);
    h.durations.assign(durations, durations + n);
    h.open_t.assign(open_t, open_t + n);
    h.close_t.assign(close_t, close_t + n);
    h.d2d.assign(d2d, d2d + n);
    h.dist.assign(dist, dist + (size_t)ld * ld);
    for (int i = 0; i < n; i++)
        if (!std::isfinite(scores[i]) || !std::isfinite(durations[i]) || !std::isfinite(open_t[i]) ||
            !std::isfinite(close_t[i]) || !std::isfinite(d2d[i]))
            return "non-finite instance value";
    for (size_t k = 0; k < h.dist.size(); k++)
        if (!std::isfinite(h.dist[k])) return "non-finite distance";
    if (!tables) return "";

    const Tests T{h};
    const size_t rows = (size_t)ld * n;
    h.F.assign(rows, 0.0);
    h.G.assign(rows, 0.0);
    h.R.assign(rows, 0.0);
    h.zlt.assign((size_t)ld * h.nw, 0u);
    h.zle.assign((size_t)ld * h.nw, 0u);
    for (int o = 0; o < ld; o++) {
        for (int j = 0; j < n; j++) {
            const double t = D(h, o, j + 1);
            h.F[(size_t)o * n + j] = largest_true([&](double f) { return T.std_ok(j, f + t); });
            h.G[(size_t)o * n + j] = largest_true([&](double f) { return T.rob_ok(j, f + t); });
            h.R[(size_t)o * n + j] = h.scores[j] / (t > 1e-10 ? t : 1e-10);
            if (t < 1e-10) h.zlt[(size_t)o * h.nw + (j >> 5)] |= 1u << (j & 31);
            if (!(t > 1e-10)) h.zle[(size_t)o * h.nw + (j >> 5)] |= 1u << (j & 31);
        }
    }
    h.P1.assign((size_t)n * n, -1.0);
    h.P0.assign(n, -1.0);
    for (int j = 0; j < n; j++) {
        const double sd_j = kSigma * h.durations[j];
        const double vb0 = 0.0 + sd_j * sd_j;
        h.P0[j] = vb0 > 1e-18 ? std::pow(vb0, 0.5) : -1.0;
    }
    for (int c = 0; c < n; c++) {
        const double sd_c = kSigma * h.durations[c];
        const double vs = sd_c * sd_c;
        for (int j = 0; j < n; j++) {
            const double sd_j = kSigma * h.durations[j];
            const double vb = vs + sd_j * sd_j;
            h.P1[(size_t)c * n + j] = vb > 1e-18 ? std::pow(vb, 0.5) : -1.0;
        }
    }
    // Neighbour-major pair tables: {F, R} and {G, dist} of (origin o,
    // neighbour j) at pair index j*ld + o.
    h.FR.assign(2 * rows, 0.0);
    h.GD.assign(2 * rows, 0.0);
    h.DP.assign(2 * (size_t)n * n, 0.0);
    h.CU.assign(6 * (size_t)n, 0.0);
    for (int j = 0; j < n; j++) {
        double* u = &h.CU[6 * (size_t)j];
        u[0] = h.close_t[j];
        u[1] = h.open_t[j];
        u[2] = h.P0[j];
        u[3] = h.durations[j];
        u[4] = h.d2d[j];
        u[5] = h.scores[j];
    }
    for (int o = 0; o < ld; o++)
        for (int j = 0; j < n; j++) {
            const size_t a = (size_t)o * n + j, t = 2 * ((size_t)j * ld + o);
            h.FR[t] = h.F[a];
            h.FR[t + 1] = h.R[a];
            h.GD[t] = h.G[a];
            h.GD[t + 1] = D(h, o, j + 1);
        }
    for (int c = 0; c < n; c++)
        for (int j = 0; j < n; j++) {
            const size_t t = 2 * ((size_t)j * n + c);
            h.DP[t] = D(h, c + 1, j + 1);
            h.DP[t + 1] = h.P1[(size_t)c * n + j];
        }
    // ATRISK's step functions at pair index j*n + c, candidates split over threads
    h.TK.assign(2 * (size_t)n * n, 0.0);
    h.TC.assign((size_t)n * n, 0);
    {
        const int nt = std::max(1, std::min<int>((int)std::thread::hardware_concurrency(), (n + 7) / 8));
        std::vector<std::thread> pool;
        for (int w = 0; w < nt; w++)
            pool.emplace_back([&, w] {
                for (int c = w; c < n; c += nt)
                    for (int j = 0; j < n; j++)
                        if (j != c)
                            atrisk_steps(h, c, j, &h.TK[2 * ((size_t)j * n + c)], &h.TC[(size_t)j * n + c]);
            });
        for (std::thread& th : pool) th.join();
    }
    // Per-origin neighbour lists by (R desc, index asc), rows padded to a
    // multiple of 4 entries; bit 14 of an index marks a coincident location.
    // cnt_pos / cnt_gm1 = how many leading entries have a ratio > 0 / > -1.
    h.ns = (n + 3) / 4 * 4;
    const size_t srows = (size_t)ld * h.ns;
    h.ord.assign(srows, 0);
    h.sF.assign(srows, -INFINITY);
    h.sG.assign(srows, -INFINITY);
    h.cnt_pos.assign(ld, 0);
    h.cnt_gm1.assign(ld, 0);
    std::vector<int> idx(n);
    for (int o = 0; o < ld; o++) {
        const double* Ro = h.R.data() + (size_t)o * n;
        for (int j = 0; j < n; j++) idx[j] = j;
        std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return Ro[a] > Ro[b]; });
        for (int k = 0; k < n; k++) {
            const int j = idx[k];
            const size_t a = (size_t)o * n + j, s = (size_t)o * h.ns + k;
            const bool coincident = (h.zlt[(size_t)o * h.nw + (j >> 5)] >> (j & 31)) & 1u;
            h.ord[s] = (int16_t)(j | (coincident ? kOrdCoincident : 0));
            h.sF[s] = h.F[a];
            h.sG[s] = h.G[a];
            if (Ro[j] > 0.0) h.cnt_pos[o] = k + 1;
            if (Ro[j] > -1.0) h.cnt_gm1[o] = k + 1;
        }
    }
    const int nc = h.ns / 4;
    h.bF.assign(2 * (size_t)ld * nc, -INFINITY);
    h.bG.assign(2 * (size_t)ld * nc, -INFINITY);
    for (int o = 0; o < ld; o++)
        for (int pass = 0; pass < 2; pass++) {
            const double* src = (pass ? h.sG : h.sF).data() + (size_t)o * h.ns;
            double* dst = (pass ? h.bG : h.bF).data() + 2 * (size_t)o * nc;
            double suffix = -INFINITY;
            for (int c = nc - 1; c >= 0; c--) {
                double mx = -INFINITY;
                for (int e = 0; e < 4; e++) mx = src[4 * c + e] > mx ? src[4 * c + e] : mx;
                suffix = mx > suffix ? mx : suffix;
                dst[2 * c] = mx;
                dst[2 * c + 1] = suffix;
            }
        }
    return "";
}

void host_zstats(const HostInstance& h, double zp[10]) {
    const Tests T{h};
    double zsum[5] = {0, 0, 0, 0, 0}, zsq[5] = {0, 0, 0, 0, 0};
    double cnt = 0.0;
    for (int i = 0; i < h.n; i++) {
        const double ta = D(h, 0, i + 1);
        if (!T.std_ok(i, ta)) continue;
        const double to = h.open_t[i];
        const double tsv = to > ta ? to : ta;
        const double fin = tsv + h.durations[i];
        const double f[5] = {h.close_t[i], z_reach2(h, i, fin), z_regret(h, i, fin), z_atrisk(h, i),
                             h.d2d[i]};
        for (int k = 0; k < 5; k++) {
            zsum[k] += f[k];
            zsq[k] += f[k] * f[k];
        }
        cnt += 1.0;
    }
    if (cnt < 1.0) cnt = 1.0;
    for (int k = 0; k < 5; k++) {
        const double mean = zsum[k] / cnt;
        double var = zsq[k] / cnt - mean * mean;
        if (var < 0.0) var = 0.0;
        zp[k] = mean;
        zp[5 + k] = std::sqrt(var) + 1e-9;
    }
}

bool slot_active(int s, const int64_t* M) {
    if (s < 10) return true;
    if (s == 11) return M[11] || M[33];
    if (s == 14) return M[14] || M[32];
    if (s == 30) return M[30] || M[34];
    return M[s] != 0;
}

namespace {

// Need bits and deepest REACH-k step for one active slot (the dependencies of
// terms[] in engine/sim_core.hpp:84-197).
void slot_needs(int s, uint32_t& need, int& reach_k, uint64_t& explore) {
    switch (s) {
    case 10: need |= kNeedNS; break;
    case 11: case 33: need |= kNeedRegret; break;
    case 12: need |= kNeedNSRob; break;
    case 13: need |= kNeedMaxN; break;
    case 14: case 32: need |= kNeedReach2; break;
    case 15: need |= kNeedNSTW; break;
    case 17: case 18: case 19: need |= kNeedStruct; break;
    case 20: need |= kNeedPBust; break;
    case 21: need |= kNeedReachK; reach_k = reach_k > 1 ? reach_k : 1; break;
    case 22: need |= kNeedReachK; reach_k = reach_k > 3 ? reach_k : 3; break;
    case 23: need |= kNeedReachK; reach_k = 5; break;
    case 25: case 26: need |= kNeedAgg; break;
    case 28: case 29: need |= kNeedNS | kNeedStruct; break;
    case 30: case 34: need |= kNeedAtRisk; break;
    case 41: need |= kNeedReach2Rob; break;
    case 43: need |= kNeedReach2Rob | kNeedRegret; break;
    case 45: need |= kNeedNS | kNeedNSRob; break;
    case 46: need |= kNeedNSRob; break;
    case 51: need |= kNeedAgg | kNeedFScore; break;
    case 52: need |= kNeedAgg | kNeedNFeasRob; break;
    case 44: case 47: case 48: case 49: case 50: case 53: case 54: case 55: case 56: case 57:
    case 59: case 60:
        need |= kNeedExplore;
        explore |= 1ull << s;
        break;
    default: break;
    }
}

}  // namespace

std::string compile_rule(const int32_t* ops, const int32_t* args, int len, const int64_t* M,
                         CompiledRule& out, bool all_active_rows) {
    out = CompiledRule();
    if (len < 1) return "empty rule";
    if (len > kMaxTree) return "rule longer than MAX_TREE (1024)";
    // Pass 1: stack discipline and the set of active slots read.
    int sp = 0, maxsp = 0;
    int slot_row[kTerms];
    for (int s = 0; s < kTerms; s++) slot_row[s] = -1;
    if (all_active_rows)
        for (int s = 0; s < kTerms; s++)
            if (slot_active(s, M) && !(s >= 36 && s <= 40)) {
                slot_row[s] = out.K++;
                out.slots.push_back((uint8_t)s);
            }
    for (int k = 0; k < len; k++) {
        const int o = ops[k];
        if (o == -1) {
            const int s = args[2 * k];
            if (s < 0 || s >= kTerms) return "terminal slot out of range 0..60";
            if (slot_active(s, M) && !(s >= 36 && s <= 40) && slot_row[s] < 0) {
                slot_row[s] = out.K++;
                out.slots.push_back((uint8_t)s);
            }
            sp++;
        } else if (o == -2) {
            sp++;
        } else if (o >= 0 && o <= 6) {
            if (sp < 2) return "operator with fewer than two operands";
            sp--;
        } else {
            return "unknown opcode";
        }
        if (sp > maxsp) maxsp = sp;
        if (sp > kMaxStack) return "stack deeper than MAX_STACK (32)";
    }
    if (sp != 1) return "rule leaves more than one value";
    // Needs of the slots read.
    for (int s : out.slots) slot_needs(s, out.need, out.reach_k, out.explore);
    // Pass 2: three-address code.  Operand descriptors: row index, or
    // kOpConst | constant index.
    std::map<uint64_t, int> cidx;
    auto konst = [&](double v) -> uint32_t {
        uint64_t u;
        std::memcpy(&u, &v, 8);
        auto it = cidx.find(u);
        if (it != cidx.end()) return kOpConst | (uint32_t)it->second;
        const int c = (int)out.consts.size();
        cidx[u] = c;
        out.consts.push_back(v);
        return kOpConst | (uint32_t)c;
    };
    std::vector<uint32_t> st;
    st.reserve(kMaxStack);
    int maxtemp = 0;
    for (int k = 0; k < len; k++) {
        const int o = ops[k];
        if (o == -1) {
            const int s = args[2 * k];
            if (!slot_active(s, M)) st.push_back(konst(0.0));
            else if (s >= 36 && s <= 40) {
                // C1..C5: the literals of terms[36..40] (engine/sim_core.hpp:152-156)
                static const double kC[5] = {0.1, 0.2, 0.3, 0.4, 0.5};
                st.push_back(konst(kC[s - 36]));
            }
            else st.push_back((uint32_t)slot_row[s]);
        } else if (o == -2) {
            st.push_back(konst(args[2 * k] / 1000.0));
        } else {
            const uint32_t b = st.back();
            st.pop_back();
            const uint32_t a = st.back();
            st.pop_back();
            const int pos = (int)st.size();  // result stack position
            const uint32_t dst = (uint32_t)(out.K + pos);
            if (pos + 1 > maxtemp) maxtemp = pos + 1;
            out.prog.push_back((uint32_t)o | (a << 3) | (b << 13) | (dst << 23));
            if (o == 6) out.need |= kNeedRmod;
            st.push_back(dst);
        }
    }
    out.D = maxtemp;
    out.res = (int)st.back();
    if (out.consts.size() > 511) return "more than 511 distinct constants";
    (void)maxsp;
    return "";
}

}  // namespace sidr
