/*
 * sidr_oracle.c -- CPU oracle (test infrastructure only; see sidr_oracle.h).
 *
 * A restatement, in C, of the reference simulator.  Each function names the
 * reference lines it follows.  The FP expressions keep the reference's operand
 * order; compile with -O2 -ffp-contract=off.
 */
#include "sidr_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#define SIG 0.2 /* SIM_SIGMA, engine/sim_terms.hpp:15 */
#define SQRT2_C 1.4142135623730951

/* ------------------------------------------------------------------ data */

void so_build_dist(int n, const double* x, const double* y, double* dist, double* d2d) {
    /* engine/sim_host.hpp:32-38 */
    int ld = n + 1;
    for (int a = 0; a < ld; a++)
        for (int b = 0; b < ld; b++) {
            double dx = x[a] - x[b], dy = y[a] - y[b];
            dist[(size_t)a * ld + b] = sqrt(dx * dx + dy * dy);
        }
    for (int i = 0; i < n; i++) d2d[i] = dist[(size_t)(i + 1) * ld + 0];
}

/* Standard neighbour test: arrive, start no earlier than open, finish and
 * return to the depot by tmax (the loop bodies of engine/sim_terms.hpp). */
static inline int fits_std(const so_simdata* s, int j, double arrive) {
    if (arrive > s->close_t[j]) return 0;
    double st = arrive > s->open_t[j] ? arrive : s->open_t[j];
    if (st + s->durations[j] + s->dist_to_depot[j] > s->tmax) return 0;
    return 1;
}

/* Robust test: the service time inflated by (1 + SIM_SIGMA). */
static inline int fits_rob(const so_simdata* s, int j, double arrive) {
    if (arrive > s->close_t[j]) return 0;
    double st = arrive > s->open_t[j] ? arrive : s->open_t[j];
    if (st + s->durations[j] * (1.0 + SIG) + s->dist_to_depot[j] > s->tmax) return 0;
    return 1;
}

static inline double D(const so_simdata* s, int a, int b) { return s->dist[(size_t)a * s->ld + b]; }

/* ------------------------------------------------------------ terminals */

/* NS, engine/sim_terms.hpp:18-34 */
static double t_ns(const so_simdata* s, const unsigned char* vis, int i, double fin) {
    double acc = 0.0;
    for (int j = 0; j < s->n; j++) {
        if (j == i || vis[j]) continue;
        double t = D(s, i + 1, j + 1);
        if (t < 1e-10) continue;
        if (!fits_std(s, j, fin + t)) continue;
        acc += s->scores[j] / t;
    }
    return acc;
}

/* REGRET, engine/sim_terms.hpp:36-54 */
static double t_regret(const so_simdata* s, const unsigned char* vis, int i, int cur, double ct,
                       double fin) {
    double acc = 0.0;
    for (int j = 0; j < s->n; j++) {
        if (j == i || vis[j]) continue;
        if (!fits_std(s, j, ct + D(s, cur, j + 1))) continue;
        double after = fin + D(s, i + 1, j + 1);
        if (after > s->close_t[j]) {
            acc += s->scores[j];
            continue;
        }
        double st = after > s->open_t[j] ? after : s->open_t[j];
        if (st + s->durations[j] + s->dist_to_depot[j] > s->tmax) acc += s->scores[j];
    }
    return acc;
}

/* NSROB, engine/sim_terms.hpp:56-74 */
static double t_ns_rob(const so_simdata* s, const unsigned char* vis, int i, double fin) {
    double frob = fin + s->durations[i] * SIG;
    double acc = 0.0;
    for (int j = 0; j < s->n; j++) {
        if (j == i || vis[j]) continue;
        double t = D(s, i + 1, j + 1);
        if (t < 1e-10) continue;
        if (!fits_rob(s, j, frob + t)) continue;
        acc += s->scores[j] / t;
    }
    return acc;
}

/* MAXN, engine/sim_terms.hpp:76-93 */
static double t_maxn(const so_simdata* s, const unsigned char* vis, int i, double fin) {
    double best = 0.0;
    for (int j = 0; j < s->n; j++) {
        if (j == i || vis[j]) continue;
        double t = D(s, i + 1, j + 1);
        if (t < 1e-10) continue;
        if (!fits_std(s, j, fin + t)) continue;
        double v = s->scores[j] / t;
        if (v > best) best = v;
    }
    return best;
}

/* Greedy best neighbour by score/time from node `from` (1-based node id) at
 * time `tm`, skipping ex1/ex2; shared by the two REACH2 loops
 * (engine/sim_terms.hpp:95-127, 156-190).  rob selects the robust test;
 * *fin_out receives the neighbour's finish time (robust duration if rob). */
static int reach_pick(const so_simdata* s, const unsigned char* vis, int from, double tm, int ex1,
                      int ex2, int rob, double* fin_out) {
    double best_v = 0.0, fj = 0.0;
    int bj = -1;
    for (int j = 0; j < s->n; j++) {
        if (j == ex1 || j == ex2 || vis[j]) continue;
        double t = D(s, from, j + 1);
        if (t < 1e-10) continue;
        double arrive = tm + t;
        if (arrive > s->close_t[j]) continue;
        double st = arrive > s->open_t[j] ? arrive : s->open_t[j];
        double fin = rob ? st + s->durations[j] * (1.0 + SIG) : st + s->durations[j];
        if ((rob ? st + s->durations[j] * (1.0 + SIG) + s->dist_to_depot[j]
                 : st + s->durations[j] + s->dist_to_depot[j]) > s->tmax)
            continue;
        double v = s->scores[j] / t;
        if (v > best_v) {
            best_v = v;
            bj = j;
            fj = fin;
        }
    }
    *fin_out = fj;
    return bj;
}

/* REACH2, engine/sim_terms.hpp:95-127 */
static double t_reach2(const so_simdata* s, const unsigned char* vis, int i, double fin) {
    double fj;
    int bj = reach_pick(s, vis, i + 1, fin, i, i, 0, &fj);
    if (bj < 0) return 0.0;
    double f2;
    int bk = reach_pick(s, vis, bj + 1, fj, i, bj, 0, &f2);
    double s2 = bk >= 0 ? s->scores[bk] : 0.0;
    return s->scores[bj] + s2;
}

/* REACH2ROB, engine/sim_terms.hpp:156-190 */
static double t_reach2_rob(const so_simdata* s, const unsigned char* vis, int i, double fin) {
    double frob = fin + s->durations[i] * SIG;
    double fj;
    int bj = reach_pick(s, vis, i + 1, frob, i, i, 1, &fj);
    if (bj < 0) return 0.0;
    double f2;
    int bk = reach_pick(s, vis, bj + 1, fj, i, bj, 1, &f2);
    double s2 = bk >= 0 ? s->scores[bk] : 0.0;
    return s->scores[bj] + s2;
}

/* SKIPLOSS, engine/sim_terms.hpp:129-154 */
static double t_skiploss(const so_simdata* s, const unsigned char* vis, int i, int cur, double ct) {
    double best_v = 0.0, fq = 0.0;
    int bq = -1;
    for (int q = 0; q < s->n; q++) {
        if (q == i || vis[q]) continue;
        double t = D(s, cur, q + 1);
        if (t < 1e-10) continue;
        double arrive = ct + t;
        if (arrive > s->close_t[q]) continue;
        double st = arrive > s->open_t[q] ? arrive : s->open_t[q];
        if (st + s->durations[q] + s->dist_to_depot[q] > s->tmax) continue;
        double v = s->scores[q] / t;
        if (v > best_v) {
            best_v = v;
            bq = q;
            fq = st + s->durations[q];
        }
    }
    if (bq < 0) return 0.0;
    double arr_i = fq + D(s, bq + 1, i + 1);
    if (arr_i > s->close_t[i]) return s->scores[i];
    double st_i = arr_i > s->open_t[i] ? arr_i : s->open_t[i];
    if (st_i + s->durations[i] + s->dist_to_depot[i] > s->tmax) return s->scores[i];
    return 0.0;
}

/* NSTW, engine/sim_terms.hpp:192-213 */
static double t_nstw(const so_simdata* s, const unsigned char* vis, int i, double fin) {
    double acc = 0.0;
    for (int j = 0; j < s->n; j++) {
        if (j == i || vis[j]) continue;
        double t = D(s, i + 1, j + 1);
        if (t < 1e-10) continue;
        double arrive = fin + t;
        if (!fits_std(s, j, arrive)) continue;
        double wait = s->open_t[j] - arrive;
        if (wait < 0.0) wait = 0.0;
        double win = s->close_t[j] - s->open_t[j];
        double w = win > 1e-10 ? 1.0 - wait / win : 1.0;
        if (w < 0.0) w = 0.0;
        acc += (s->scores[j] / t) * w;
    }
    return acc;
}

/* RAND, engine/sim_terms.hpp:215-219 */
static double t_rand(int i) {
    long long x = (((long long)i + 1) * 1103515245LL + 12345LL) & 0x7FFFFFFFLL;
    x = (x * 1103515245LL + 12345LL) & 0x7FFFFFFFLL;
    return (double)(x % 100000LL) / 1000.0;
}

/* norm_cdf, engine/sim_terms.hpp:221-223 */
static double ncdf(double z) { return 0.5 * (1.0 + erf(z * 0.7071067811865476)); }

/* ATRISK, engine/sim_terms.hpp:225-257 */
static double t_atrisk(const so_simdata* s, const unsigned char* vis, int c, int cur, double ct) {
    double arr_c = ct + D(s, cur, c + 1);
    double st_c = arr_c > s->open_t[c] ? arr_c : s->open_t[c];
    double mfin = st_c + s->durations[c];
    double sd_c = SIG * s->durations[c];
    double acc = 0.0;
    for (int j = 0; j < s->n; j++) {
        if (vis[j] || j == c) continue;
        if (ct + D(s, cur, j + 1) > s->close_t[j]) continue;
        double marr = mfin + D(s, c + 1, j + 1);
        double pw;
        if (sd_c > 1e-9) pw = ncdf((s->close_t[j] - marr) / sd_c);
        else pw = marr <= s->close_t[j] ? 1.0 : 0.0;
        double mst, vst;
        if (marr > s->open_t[j]) {
            mst = marr;
            vst = sd_c * sd_c;
        } else {
            mst = s->open_t[j];
            vst = 0.0;
        }
        double sd_j = SIG * s->durations[j];
        double vb = vst + sd_j * sd_j;
        double mb = mst + s->durations[j] + s->dist_to_depot[j];
        double pb;
        if (vb > 1e-18) pb = ncdf((s->tmax - mb) / pow(vb, 0.5));
        else pb = mb <= s->tmax ? 1.0 : 0.0;
        acc += s->scores[j] * (1.0 - pw * pb);
    }
    return acc;
}

/* NSA2 / NSA05, engine/sim_terms.hpp:259-293: kind 2 -> score/t^2, kind 1 -> score/sqrt(t) */
static double t_ns_pow(const so_simdata* s, const unsigned char* vis, int i, double fin, int kind) {
    double acc = 0.0;
    for (int j = 0; j < s->n; j++) {
        if (j == i || vis[j]) continue;
        double t = D(s, i + 1, j + 1);
        if (t < 1e-10) continue;
        if (!fits_std(s, j, fin + t)) continue;
        if (kind == 2) acc += s->scores[j] / (t * t);
        else acc += s->scores[j] / sqrt(t);
    }
    return acc;
}

/* NSROB05 / NSROB2, engine/sim_terms.hpp:295-314 */
static double t_ns_rob_m(const so_simdata* s, const unsigned char* vis, int i, double fin, double m) {
    double ms = m * SIG;
    double frob = fin + s->durations[i] * ms;
    double acc = 0.0;
    for (int j = 0; j < s->n; j++) {
        if (j == i || vis[j]) continue;
        double t = D(s, i + 1, j + 1);
        if (t < 1e-10) continue;
        double arrive = frob + t;
        if (arrive > s->close_t[j]) continue;
        double st = arrive > s->open_t[j] ? arrive : s->open_t[j];
        if (st + s->durations[j] * (1.0 + ms) + s->dist_to_depot[j] > s->tmax) continue;
        acc += s->scores[j] / t;
    }
    return acc;
}

/* NNFWD, engine/sim_terms.hpp:316-334 */
static double t_nnfwd(const so_simdata* s, const unsigned char* vis, int i, double fin) {
    double dmin = -1.0;
    for (int j = 0; j < s->n; j++) {
        if (j == i || vis[j]) continue;
        double t = D(s, i + 1, j + 1);
        if (t < 1e-10) continue;
        if (!fits_std(s, j, fin + t)) continue;
        if (dmin < 0.0 || t < dmin) dmin = t;
    }
    if (dmin < 0.0) return 0.0;
    return 1.0 / (1.0 + dmin);
}

/* NNK3, engine/sim_terms.hpp:336-358 */
static double t_nnk3(const so_simdata* s, const unsigned char* vis, int i, double fin) {
    double d1 = -1.0, d2 = -1.0, d3 = -1.0;
    for (int j = 0; j < s->n; j++) {
        if (j == i || vis[j]) continue;
        double t = D(s, i + 1, j + 1);
        if (t < 1e-10) continue;
        if (!fits_std(s, j, fin + t)) continue;
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
    }
    if (d1 < 0.0) return 0.0;
    double tot = d1, k = 1.0;
    if (d2 >= 0.0) {
        tot += d2;
        k += 1.0;
    }
    if (d3 >= 0.0) {
        tot += d3;
        k += 1.0;
    }
    return 1.0 / (1.0 + tot / k);
}

/* DETOUR, engine/sim_terms.hpp:360-380 */
static double t_detour(const so_simdata* s, const unsigned char* vis, int i, int cur, double fin,
                       double ta_i) {
    double tot = 0.0, cnt = 0.0;
    for (int j = 0; j < s->n; j++) {
        if (j == i || vis[j]) continue;
        double t = D(s, i + 1, j + 1);
        if (t < 1e-10) continue;
        if (!fits_std(s, j, fin + t)) continue;
        tot += ta_i + t - D(s, cur, j + 1);
        cnt += 1.0;
    }
    if (cnt == 0.0) return 0.0;
    return tot / cnt;
}

/* SCORERANK, engine/sim_terms.hpp:382-401 */
static double t_scorerank(const so_simdata* s, const unsigned char* vis, int i, double fin) {
    double below = 0.0, tot = 0.0;
    for (int j = 0; j < s->n; j++) {
        if (j == i || vis[j]) continue;
        double t = D(s, i + 1, j + 1);
        if (t < 1e-10) continue;
        if (!fits_std(s, j, fin + t)) continue;
        tot += 1.0;
        if (s->scores[j] < s->scores[i]) below += 1.0;
    }
    if (tot == 0.0) return 1.0;
    return below / tot;
}

/* REACH-k and REACH-k-ROB, engine/sim_terms.hpp:405-479.  The visited copy
 * is `scr` (caller buffer of n bytes). */
static double t_reach_k(const so_simdata* s, const unsigned char* vis, int c, int cur, double ct,
                        int K, int rob, unsigned char* scr) {
    memcpy(scr, vis, (size_t)s->n);
    scr[c] = 1;
    double arr_c = ct + D(s, cur, c + 1);
    double st_c = arr_c > s->open_t[c] ? arr_c : s->open_t[c];
    int at = c + 1;
    double tm = rob ? st_c + s->durations[c] * (1.0 + SIG) : st_c + s->durations[c];
    double acc = 0.0;
    for (int step = 0; step < K; step++) {
        int best = -1;
        double best_v = -1.0;
        for (int q = 0; q < s->n; q++) {
            if (scr[q]) continue;
            double ta = D(s, at, q + 1);
            double arrive = tm + ta;
            if (rob ? !fits_rob(s, q, arrive) : !fits_std(s, q, arrive)) continue;
            double tt = ta > 1e-10 ? ta : 1e-10;
            double v = s->scores[q] / tt;
            if (v > best_v) {
                best_v = v;
                best = q;
            }
        }
        if (best < 0) break;
        double arrive = tm + D(s, at, best + 1);
        double st = arrive > s->open_t[best] ? arrive : s->open_t[best];
        tm = rob ? st + s->durations[best] * (1.0 + SIG) : st + s->durations[best];
        at = best + 1;
        acc += s->scores[best];
        scr[best] = 1;
    }
    return acc;
}

/* NNCHAIN, engine/sim_terms.hpp:481-519 */
static double t_nnchain(const so_simdata* s, const unsigned char* vis, int c, int cur, double ct,
                        int K, unsigned char* scr) {
    memcpy(scr, vis, (size_t)s->n);
    scr[c] = 1;
    double arr_c = ct + D(s, cur, c + 1);
    double st_c = arr_c > s->open_t[c] ? arr_c : s->open_t[c];
    int at = c + 1;
    double tm = st_c + s->durations[c];
    double tot = 0.0;
    int done = 0;
    for (int step = 0; step < K; step++) {
        int best = -1;
        double best_d = -1.0;
        for (int q = 0; q < s->n; q++) {
            if (scr[q]) continue;
            double ta = D(s, at, q + 1);
            if (ta < 1e-10) continue;
            if (!fits_std(s, q, tm + ta)) continue;
            if (best_d < 0.0 || ta < best_d) {
                best_d = ta;
                best = q;
            }
        }
        if (best < 0) break;
        double arrive = tm + best_d;
        double st = arrive > s->open_t[best] ? arrive : s->open_t[best];
        tm = st + s->durations[best];
        at = best + 1;
        tot += best_d;
        done++;
        scr[best] = 1;
    }
    if (done == 0) return 0.0;
    return 1.0 / (1.0 + tot / done);
}

/* FRAGCNT / FRAGSCORE / DOWNSLACK / PBUST, engine/sim_terms.hpp:522-580 */
static void struct_feats(const so_simdata* s, const unsigned char* vis, int c, int cur, double ct,
                         double* out) {
    double arr_c = ct + D(s, cur, c + 1);
    double st_c = arr_c > s->open_t[c] ? arr_c : s->open_t[c];
    double fin_c = st_c + s->durations[c];
    int cp = c + 1;
    double fcnt = 0.0, fsc = 0.0, slackmin = 1e18, best_v = -1.0;
    int bq = -1;
    for (int q = 0; q < s->n; q++) {
        if (vis[q] || q == c) continue;
        int now = fits_std(s, q, ct + D(s, cur, q + 1));
        int after = fits_std(s, q, fin_c + D(s, cp, q + 1));
        if (now && !after) {
            fcnt += 1.0;
            fsc += s->scores[q];
        }
        if (after) {
            double aq = fin_c + D(s, cp, q + 1);
            double slack = s->close_t[q] - aq;
            if (slack < slackmin) slackmin = slack;
            double t = D(s, cp, q + 1);
            if (t > 1e-10) {
                double v = s->scores[q] / t;
                if (v > best_v) {
                    best_v = v;
                    bq = q;
                }
            }
        }
    }
    if (slackmin > 1e17) slackmin = 0.0;
    double pbust = 0.0;
    if (bq >= 0) {
        double ab = fin_c + D(s, cp, bq + 1);
        double sd = SIG * s->durations[c];
        if (sd > 1e-12) {
            double z = (s->close_t[bq] - ab) / (sd * SQRT2_C);
            pbust = 0.5 * erfc(z);
        } else {
            pbust = ab > s->close_t[bq] ? 1.0 : 0.0;
        }
    }
    out[0] = fcnt;
    out[1] = fsc;
    out[2] = slackmin;
    out[3] = pbust;
}

/* ------------------------------------------------------------ interpreter */

double so_eval_tree(const int32_t* ops, const int32_t* args, int len, const double* terms,
                    double* stack) {
    /* engine/sim_core.hpp:11-41 */
    int sp = 0;
    for (int k = 0; k < len; k++) {
        int o = ops[k];
        if (o == -1) {
            stack[sp++] = terms[args[2 * k]];
            continue;
        }
        if (o == -2) {
            stack[sp++] = args[2 * k] / 1000.0;
            continue;
        }
        double b = stack[--sp];
        double a = stack[--sp];
        double r;
        switch (o) {
        case 0: r = a + b; break;
        case 1: r = a - b; break;
        case 2: r = a * b; break;
        case 3: r = fabs(b) < 1e-10 ? 1.0 : a / b; break;
        case 4: r = a < b ? a : b; break;
        case 5: r = a > b ? a : b; break;
        default: {
            double base = a > 0.0 ? a : 0.0;
            double e = b;
            if (e < 0.0) e = 0.0;
            else if (e > 1.0) e = 1.0;
            r = pow(base, 1.0 + e);
        }
        }
        stack[sp++] = r;
    }
    return stack[0];
}

/* ------------------------------------------------------------- decision */

typedef struct {
    const so_simdata* s;
    const int64_t* mask;
    const double* zp;
    const int32_t *ops, *args;
    int len;
    unsigned char* vis;
    unsigned char* scr;
    so_counts cnt;
} so_run;

/* pick_best, engine/sim_core.hpp:43-204 */
static int pick_best(so_run* R, int cur, double ct, int remaining) {
    const so_simdata* s = R->s;
    const int64_t* M = R->mask;
    const double* zp = R->zp;
    const unsigned char* vis = R->vis;
    int n = s->n;
    double tmax = s->tmax;
    double terms[SO_N_TERMS], stack[SO_MAX_STACK], sb[4] = {0, 0, 0, 0};
    memset(terms, 0, sizeof terms);
    R->cnt.decisions++;

    int need_ns = M[10] || M[28] || M[29];
    int need_struct = M[17] || M[18] || M[19] || M[20] || M[28] || M[29];

    double sat = tmax > 0.0 ? ct / tmax : 0.0;
    double vfrac = 0.0, nfeas = 0.0, fscore = 0.0, nfeasrob = 0.0;
    if (M[25] || M[26] || M[51] || M[52]) {
        double nvis = 0.0;
        for (int j = 0; j < n; j++) {
            if (vis[j]) {
                nvis += 1.0;
                continue;
            }
            double arr = ct + D(s, cur, j + 1);
            if (arr > s->close_t[j]) continue;
            double st = arr > s->open_t[j] ? arr : s->open_t[j];
            if (st + s->durations[j] + s->dist_to_depot[j] > tmax) continue;
            nfeas += 1.0;
            fscore += s->scores[j];
            if (st + s->durations[j] * (1.0 + SIG) + s->dist_to_depot[j] <= tmax) nfeasrob += 1.0;
        }
        vfrac = nvis / n;
    }

    int best = -1;
    double best_pri = -1e300;
    for (int i = 0; i < n; i++) {
        if (vis[i]) continue;
        double ta = D(s, cur, i + 1);
        double arrival = ct + ta;
        if (arrival > s->close_t[i]) continue;
        double start = arrival > s->open_t[i] ? arrival : s->open_t[i];
        if (start + s->durations[i] + s->dist_to_depot[i] > tmax) continue;
        R->cnt.candidates++;

        double to = s->open_t[i] - ct;
        double tc = s->close_t[i] - ct;
        double tsv = to > ta ? to : ta;
        double tfv = tsv + s->durations[i];
        terms[0] = s->scores[i];
        terms[1] = s->durations[i];
        terms[2] = to;
        terms[3] = tc;
        terms[4] = ta;
        terms[5] = s->dist_to_depot[i];
        terms[6] = tsv;
        terms[7] = tfv;
        terms[8] = tc - ta;
        terms[9] = remaining * tmax + (tmax - ct);

        double fin = ct + tfv;
        double ns_val = need_ns ? t_ns(s, vis, i, fin) : 0.0;
        terms[10] = M[10] ? ns_val : 0.0;
        terms[11] = (M[11] || M[33]) ? t_regret(s, vis, i, cur, ct, fin) : 0.0;
        terms[12] = M[12] ? t_ns_rob(s, vis, i, fin) : 0.0;
        terms[13] = M[13] ? t_maxn(s, vis, i, fin) : 0.0;
        terms[14] = (M[14] || M[32]) ? t_reach2(s, vis, i, fin) : 0.0;
        terms[15] = M[15] ? t_nstw(s, vis, i, fin) : 0.0;
        terms[16] = M[16] ? t_rand(i) : 0.0;
        double frag_score = 0.0;
        if (need_struct) {
            struct_feats(s, vis, i, cur, ct, sb);
            frag_score = sb[1];
        }
        terms[17] = M[17] ? sb[0] : 0.0;
        terms[18] = M[18] ? sb[1] : 0.0;
        terms[19] = M[19] ? sb[2] : 0.0;
        terms[20] = M[20] ? sb[3] : 0.0;
        terms[21] = M[21] ? t_reach_k(s, vis, i, cur, ct, 1, 0, R->scr) : 0.0;
        terms[22] = M[22] ? t_reach_k(s, vis, i, cur, ct, 3, 0, R->scr) : 0.0;
        terms[23] = M[23] ? t_reach_k(s, vis, i, cur, ct, 5, 0, R->scr) : 0.0;
        terms[24] = M[24] ? sat : 0.0;
        terms[25] = M[25] ? vfrac : 0.0;
        terms[26] = M[26] ? nfeas : 0.0;
        terms[27] = M[27] ? (double)remaining : 0.0;
        terms[28] = M[28] ? frag_score / (ns_val + 1.0) : 0.0;
        terms[29] = M[29] ? frag_score - ns_val : 0.0;
        terms[30] = (M[30] || M[34]) ? t_atrisk(s, vis, i, cur, ct) : 0.0;
        terms[31] = M[31] ? (terms[3] - zp[0]) / zp[5] : 0.0;
        terms[32] = M[32] ? (terms[14] - zp[1]) / zp[6] : 0.0;
        terms[33] = M[33] ? (terms[11] - zp[2]) / zp[7] : 0.0;
        terms[34] = M[34] ? (terms[30] - zp[3]) / zp[8] : 0.0;
        terms[35] = M[35] ? (terms[5] - zp[4]) / zp[9] : 0.0;
        terms[36] = M[36] ? 0.1 : 0.0;
        terms[37] = M[37] ? 0.2 : 0.0;
        terms[38] = M[38] ? 0.3 : 0.0;
        terms[39] = M[39] ? 0.4 : 0.0;
        terms[40] = M[40] ? 0.5 : 0.0;
        terms[41] = M[41] ? t_reach2_rob(s, vis, i, fin) : 0.0;
        {
            double den = tmax - ct;
            if (den < 1.0) den = 1.0;
            terms[42] = M[42] ? (ta + s->durations[i]) / den : 0.0;
        }
        terms[43] = M[43] ? (t_reach2_rob(s, vis, i, fin) - t_regret(s, vis, i, cur, ct, fin)) : 0.0;
        terms[44] = M[44] ? t_skiploss(s, vis, i, cur, ct) : 0.0;
        terms[45] = M[45] ? (t_ns(s, vis, i, fin) - t_ns_rob(s, vis, i, fin)) : 0.0;
        {
            double den = ta + s->dist_to_depot[i];
            if (den < 1.0) den = 1.0;
            terms[46] = M[46] ? (s->scores[i] + t_ns_rob(s, vis, i, fin)) / den : 0.0;
        }
        terms[47] = M[47] ? t_reach_k(s, vis, i, cur, ct, 3, 1, R->scr) : 0.0;
        terms[48] = M[48] ? t_reach_k(s, vis, i, cur, ct, 5, 1, R->scr) : 0.0;
        terms[49] = M[49] ? t_ns_pow(s, vis, i, fin, 2) : 0.0;
        terms[50] = M[50] ? t_ns_pow(s, vis, i, fin, 1) : 0.0;
        terms[51] = M[51] ? fscore : 0.0;
        terms[52] = M[52] ? nfeasrob : 0.0;
        terms[53] = M[53] ? t_ns_rob_m(s, vis, i, fin, 0.5) : 0.0;
        terms[54] = M[54] ? t_ns_rob_m(s, vis, i, fin, 2.0) : 0.0;
        terms[55] = M[55] ? t_nnfwd(s, vis, i, fin) : 0.0;
        terms[56] = M[56] ? t_nnk3(s, vis, i, fin) : 0.0;
        terms[57] = M[57] ? t_nnchain(s, vis, i, cur, ct, 3, R->scr) : 0.0;
        terms[58] = M[58] ? (D(s, cur, 0) + s->dist_to_depot[i] - ta) : 0.0;
        terms[59] = M[59] ? t_detour(s, vis, i, cur, fin, ta) : 0.0;
        terms[60] = M[60] ? t_scorerank(s, vis, i, fin) : 0.0;

        R->cnt.tokens += R->len;
        double pri = so_eval_tree(R->ops, R->args, R->len, terms, stack);
        if (pri != pri) pri = -1e300;
        if (pri > best_pri) {
            best_pri = pri;
            best = i;
        }
    }
    return best;
}

/* sim_one, engine/sim_core.hpp:207-238 */
static double sim_one_run(so_run* R, const double* sampled) {
    const so_simdata* s = R->s;
    memset(R->vis, 0, (size_t)s->n);
    double total = 0.0;
    for (int v = 0; v < s->m; v++) {
        int remaining = s->m - v - 1;
        int cur = 0;
        double ct = 0.0;
        for (;;) {
            int b = pick_best(R, cur, ct, remaining);
            if (b < 0) break;
            double arrival = ct + D(s, cur, b + 1);
            double start = arrival > s->open_t[b] ? arrival : s->open_t[b];
            ct = start + sampled[b];
            cur = b + 1;
            total += s->scores[b];
            R->vis[b] = 1;
        }
    }
    return total;
}

double so_sim_one(const so_simdata* sd, const int32_t* ops, const int32_t* args, int len,
                  const double* sampled, const int64_t* term_mask, const double* zp) {
    unsigned char vis[SO_MAX_N], scr[SO_MAX_N];
    so_run R;
    memset(&R, 0, sizeof R);
    R.s = sd;
    R.mask = term_mask;
    R.zp = zp;
    R.ops = ops;
    R.args = args;
    R.len = len;
    R.vis = vis;
    R.scr = scr;
    return sim_one_run(&R, sampled);
}

/* ---------------------------------------------------------------- z-stats */

void so_zstats(const so_simdata* s, double* zp) {
    /* engine/sim_core.hpp:277-312 */
    unsigned char vis[SO_MAX_N];
    memset(vis, 0, sizeof vis);
    double zsum[5] = {0, 0, 0, 0, 0}, zsq[5] = {0, 0, 0, 0, 0};
    double cnt = 0.0;
    for (int i = 0; i < s->n; i++) {
        double ta = D(s, 0, i + 1);
        double arr = ta;
        if (arr > s->close_t[i]) continue;
        double start = arr > s->open_t[i] ? arr : s->open_t[i];
        if (start + s->durations[i] + s->dist_to_depot[i] > s->tmax) continue;
        double to = s->open_t[i];
        double tsv = to > ta ? to : ta;
        double fin = tsv + s->durations[i];
        double f[5];
        f[0] = s->close_t[i];
        f[1] = t_reach2(s, vis, i, fin);
        f[2] = t_regret(s, vis, i, 0, 0.0, fin);
        f[3] = t_atrisk(s, vis, i, 0, 0.0);
        f[4] = s->dist_to_depot[i];
        for (int k = 0; k < 5; k++) {
            zsum[k] += f[k];
            zsq[k] += f[k] * f[k];
        }
        cnt += 1.0;
    }
    if (cnt < 1.0) cnt = 1.0;
    for (int k = 0; k < 5; k++) {
        double mean = zsum[k] / cnt;
        double var = zsq[k] / cnt - mean * mean;
        if (var < 0.0) var = 0.0;
        zp[k] = mean;
        zp[5 + k] = sqrt(var) + 1e-9;
    }
}

/* ------------------------------------------------------------------- MT19937 */

static void mt_init_genrand(so_mt* r, uint32_t s) {
    r->mt[0] = s;
    for (int i = 1; i < 624; i++)
        r->mt[i] = 1812433253u * (r->mt[i - 1] ^ (r->mt[i - 1] >> 30)) + (uint32_t)i;
    r->mti = 624;
}

void so_mt_seed(so_mt* r, uint64_t seed) {
    /* engine/rng.hpp:27-52: init_by_array over the 32-bit words of the seed,
     * least significant first (one zero word for seed 0). */
    uint32_t key[2];
    int klen = 0;
    if (seed == 0) key[klen++] = 0;
    while (seed) {
        key[klen++] = (uint32_t)(seed & 0xffffffffu);
        seed >>= 32;
    }
    mt_init_genrand(r, 19650218u);
    int i = 1, j = 0;
    for (int k = (624 > klen ? 624 : klen); k; k--) {
        r->mt[i] = (r->mt[i] ^ ((r->mt[i - 1] ^ (r->mt[i - 1] >> 30)) * 1664525u)) + key[j] + (uint32_t)j;
        i++;
        j++;
        if (i >= 624) {
            r->mt[0] = r->mt[623];
            i = 1;
        }
        if (j >= klen) j = 0;
    }
    for (int k = 623; k; k--) {
        r->mt[i] = (r->mt[i] ^ ((r->mt[i - 1] ^ (r->mt[i - 1] >> 30)) * 1566083941u)) - (uint32_t)i;
        i++;
        if (i >= 624) {
            r->mt[0] = r->mt[623];
            i = 1;
        }
    }
    r->mt[0] = 0x80000000u;
    r->mti = 624;
    r->has_gauss = 0;
    r->gauss_next = 0.0;
}

uint32_t so_mt_genrand(so_mt* r) {
    /* engine/rng.hpp:54-75 */
    if (r->mti >= 624) {
        for (int k = 0; k < 624; k++) {
            uint32_t y = (r->mt[k] & 0x80000000u) | (r->mt[(k + 1) % 624] & 0x7fffffffu);
            r->mt[k] = r->mt[(k + 397) % 624] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
        }
        r->mti = 0;
    }
    uint32_t y = r->mt[r->mti++];
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return y;
}

double so_mt_random(so_mt* r) {
    /* engine/rng.hpp:78-81 */
    uint32_t a = so_mt_genrand(r) >> 5, b = so_mt_genrand(r) >> 6;
    return (a * 67108864.0 + b) * (1.0 / 9007199254740992.0);
}

double so_mt_gauss(so_mt* r, double mu, double sigma) {
    /* engine/rng.hpp:135-147 */
    double z;
    if (r->has_gauss) {
        z = r->gauss_next;
        r->has_gauss = 0;
    } else {
        double x2pi = so_mt_random(r) * (2.0 * 3.14159265358979323846);
        double g2rad = sqrt(-2.0 * log(1.0 - so_mt_random(r)));
        z = cos(x2pi) * g2rad;
        r->gauss_next = sin(x2pi) * g2rad;
        r->has_gauss = 1;
    }
    return mu + z * sigma;
}

void so_gen_durations(int n, const double* durations, double sigma, int S, long long base_seed,
                      double* out) {
    /* engine/sim_host.hpp:43-58 */
    so_mt r;
    for (int s = 0; s < S; s++) {
        so_mt_seed(&r, (uint64_t)(base_seed + s));
        for (int i = 0; i < n; i++) {
            double e = durations[i];
            double v = 0.0;
            if (e > 0.0) {
                v = so_mt_gauss(&r, e, sigma * e);
                if (!(v > 0.0)) v = 0.0;
            }
            out[(size_t)s * n + i] = v;
        }
    }
}

/* ------------------------------------------------------------ batch driver */

typedef struct {
    const so_simdata* sd;
    const double* zp;
    const int32_t *ops, *args, *offsets, *lengths;
    int P, T, group_size, mask_group;
    const double* sampled;
    const int64_t* masks;
    double* out;
    int p0, p1;
    so_counts cnt;
} so_job;

static void* so_job_run(void* arg) {
    so_job* J = (so_job*)arg;
    unsigned char vis[SO_MAX_N], scr[SO_MAX_N];
    for (int p = J->p0; p < J->p1; p++) {
        so_run R;
        memset(&R, 0, sizeof R);
        R.s = J->sd;
        R.zp = J->zp;
        R.mask = J->masks + (size_t)(p / J->mask_group) * SO_N_TERMS;
        R.ops = J->ops + J->offsets[p];
        R.args = J->args + 2 * (size_t)J->offsets[p];
        R.len = J->lengths[p];
        R.vis = vis;
        R.scr = scr;
        int g = p / J->group_size;
        for (int s = 0; s < J->T; s++) {
            const double* smp = J->sampled + ((size_t)g * J->T + s) * J->sd->n;
            J->out[(size_t)p * J->T + s] = sim_one_run(&R, smp);
        }
        J->cnt.decisions += R.cnt.decisions;
        J->cnt.candidates += R.cnt.candidates;
        J->cnt.tokens += R.cnt.tokens;
    }
    return NULL;
}

void so_eval_pairs(const so_simdata* sd, const double* zp, const int32_t* ops, const int32_t* args,
                   const int32_t* offsets, const int32_t* lengths, int P,
                   const double* grouped_sampled, int T, int group_size, const int64_t* masks,
                   int mask_group, double* out, int nthreads, so_counts* counts) {
    if (nthreads < 1) nthreads = 1;
    if (nthreads > P) nthreads = P > 0 ? P : 1;
    so_job* jobs = (so_job*)calloc((size_t)nthreads, sizeof(so_job));
    pthread_t* th = (pthread_t*)calloc((size_t)nthreads, sizeof(pthread_t));
    for (int t = 0; t < nthreads; t++) {
        so_job* J = &jobs[t];
        J->sd = sd;
        J->zp = zp;
        J->ops = ops;
        J->args = args;
        J->offsets = offsets;
        J->lengths = lengths;
        J->P = P;
        J->T = T;
        J->group_size = group_size;
        J->mask_group = mask_group;
        J->sampled = grouped_sampled;
        J->masks = masks;
        J->out = out;
        J->p0 = (int)((long long)P * t / nthreads);
        J->p1 = (int)((long long)P * (t + 1) / nthreads);
    }
    for (int t = 1; t < nthreads; t++) pthread_create(&th[t], NULL, so_job_run, &jobs[t]);
    so_job_run(&jobs[0]);
    for (int t = 1; t < nthreads; t++) pthread_join(th[t], NULL);
    if (counts) {
        memset(counts, 0, sizeof *counts);
        for (int t = 0; t < nthreads; t++) {
            counts->decisions += jobs[t].cnt.decisions;
            counts->candidates += jobs[t].cnt.candidates;
            counts->tokens += jobs[t].cnt.tokens;
        }
    }
    free(jobs);
    free(th);
}
