// sidr_factory.hpp -- C++20 drop-in for the reference's FactoryContext
// (augustompm/solver-informed-dispatching-rules, engine/factory.cuh:124-217),
// implemented over the C-ABI of include/sidr.h.
//
// The reference keeps its own data structures; only the evaluator changes.
// FactoryContextT is duck-typed on the caller's SimData (fields n, m, tmax,
// scores, durations, open_t, close_t, dist, dist_to_depot as std::vector<double>,
// engine/sim_host.hpp:12-40) and PackedTrees (ops, args, offsets, lengths as
// std::vector<int32_t>, engine/factory.cuh:20-24).  In engine/factory.cuh a
// maintainer replaces the struct FactoryContext with
//
//     #include "sidr_factory.hpp"
//     using FactoryContext = sidr::FactoryContextT<SimData, PackedTrees>;
//
// and links libsidr_b200.so; gp_engine.cu, timing.cu, ga.cu, gen_trace.cu,
// choice.cu, redeploy.cu and verify_cuda.cu then compile unchanged (and, with
// no kernel left in the header, as plain C++).  tests/test_dropin.py builds the
// reference's own verify_cuda.cu and gp_engine.cu this way and runs
// verify_cuda's gate through the library.
//
// Method names, argument order and meaning, the `threads` argument (accepted
// and ignored: the launch geometry is the library's) and the output layout
// out[p*N + s] are the reference's.  Errors: like the reference's CUDA_CHECK
// (engine/factory.cuh:16-18) a failure prints the message to stderr and exits
// with status 2; define SIDR_FACTORY_THROW before including to get a
// std::runtime_error instead.
#pragma once
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <vector>

#include "sidr.h"

namespace sidr {

inline void factory_fail(sidr_status s, const char* where) {
    std::string msg = std::string("sidr error (") + sidr_status_string(s) + ") in " + where + ": " +
                      sidr_last_error();
#ifdef SIDR_FACTORY_THROW
    throw std::runtime_error(msg);
#else
    std::fprintf(stderr, "%s\n", msg.c_str());
    std::exit(2);
#endif
}

template <class SimDataT>
sidr_instance_desc describe(const SimDataT& sd) {
    sidr_instance_desc d{};
    d.n = sd.n;
    d.m = sd.m;
    d.tmax = sd.tmax;
    d.scores = sd.scores.data();
    d.durations = sd.durations.data();
    d.open_t = sd.open_t.data();
    d.close_t = sd.close_t.data();
    d.dist = sd.dist.data();
    d.dist_to_depot = sd.dist_to_depot.data();
    return d;
}

template <class PackedTreesT>
sidr_rules_desc describe_rules(const PackedTreesT& pk) {
    sidr_rules_desc r{};
    r.ops = pk.ops.data();
    r.args = pk.args.data();
    r.offsets = pk.offsets.data();
    r.lengths = pk.lengths.data();
    r.P = (int32_t)pk.offsets.size();
    r.n_nodes = (int64_t)pk.ops.size();
    return r;
}

// zp_of (engine/sim_host.hpp:96-105) through the library's host computation.
template <class SimDataT>
std::vector<double> zp_of_sidr(const SimDataT& sd) {
    sidr_instance_desc d = describe(sd);
    std::vector<double> zp(10);
    sidr_status s = sidr_zstats(&d, zp.data());
    if (s != SIDR_OK) factory_fail(s, "zp_of");
    return zp;
}

template <class SimDataT, class PackedTreesT>
struct FactoryContextT {
    const SimDataT& sd;
    std::vector<double> zp_host;
    sidr_ctx* ctx = nullptr;

    FactoryContextT(const SimDataT& sd_, const std::vector<double>& zp, int device = 0)
        : sd(sd_), zp_host(zp) {
        if (zp.size() != 10) factory_fail(SIDR_ERR_INVALID, "FactoryContext: zp must hold 10 values");
        sidr_instance_desc d = describe(sd);
        sidr_status s = sidr_ctx_create(&d, zp.data(), device, &ctx);
        if (s != SIDR_OK) factory_fail(s, "FactoryContext");
    }
    ~FactoryContextT() { sidr_ctx_destroy(ctx); }
    FactoryContextT(const FactoryContextT&) = delete;
    FactoryContextT& operator=(const FactoryContextT&) = delete;

    // out[p*N+s]; all_sampled = N scenarios x n durations.
    std::vector<double> evaluate(const PackedTreesT& pk, const std::vector<double>& all_sampled,
                                 int N, const std::vector<int64_t>& term_mask,
                                 int threads = 128) {
        (void)threads;
        check_mask(term_mask, 1);
        check_sampled(all_sampled, (size_t)N * sd.n);
        sidr_rules_desc r = describe_rules(pk);
        std::vector<double> out((size_t)r.P * N);
        sidr_status s = sidr_evaluate(ctx, &r, all_sampled.data(), N, term_mask.data(), out.data());
        if (s != SIDR_OK) factory_fail(s, "evaluate");
        return out;
    }

    // grouped_sampled = G groups x T scenarios x n; tree p -> group p/group_size.
    std::vector<double> evaluate_grouped(const PackedTreesT& pk,
                                         const std::vector<double>& grouped_sampled, int G, int T,
                                         int group_size, const std::vector<int64_t>& term_mask,
                                         int threads = 128) {
        (void)threads;
        check_mask(term_mask, 1);
        const int Gv = groups_in(grouped_sampled, T);
        (void)G;  // the reference ignores G too; the buffer size decides
        sidr_rules_desc r = describe_rules(pk);
        std::vector<double> out((size_t)r.P * T);
        sidr_status s = sidr_evaluate_grouped(ctx, &r, grouped_sampled.data(), Gv, T, group_size,
                                              term_mask.data(), out.data());
        if (s != SIDR_OK) factory_fail(s, "evaluate_grouped");
        return out;
    }

    // masks holds one 61-flag row per block of mask_group trees.
    std::vector<double> evaluate_grouped_masks(const PackedTreesT& pk,
                                               const std::vector<double>& grouped_sampled, int T,
                                               int group_size, int mask_group,
                                               const std::vector<int64_t>& masks,
                                               int threads = 128) {
        (void)threads;
        sidr_rules_desc r = describe_rules(pk);
        if (mask_group < 1) factory_fail(SIDR_ERR_INVALID, "evaluate_grouped_masks: mask_group < 1");
        check_mask(masks, r.P > 0 ? (size_t)((r.P - 1) / mask_group + 1) : 0);
        const int Gv = groups_in(grouped_sampled, T);
        std::vector<double> out((size_t)r.P * T);
        sidr_status s = sidr_evaluate_grouped_masks(ctx, &r, grouped_sampled.data(), Gv, T,
                                                    group_size, mask_group, masks.data(),
                                                    out.data());
        if (s != SIDR_OK) factory_fail(s, "evaluate_grouped_masks");
        return out;
    }

  private:
    int groups_in(const std::vector<double>& v, int T) const {
        if (T <= 0 || sd.n <= 0) return 0;
        return (int)(v.size() / ((size_t)T * sd.n));
    }
    static void check_mask(const std::vector<int64_t>& m, size_t rows) {
        if (m.size() < rows * (size_t)SIDR_N_TERMS)
            factory_fail(SIDR_ERR_INVALID, "term mask shorter than 61 flags per row");
    }
    static void check_sampled(const std::vector<double>& v, size_t need) {
        if (v.size() < need) factory_fail(SIDR_ERR_INVALID, "scenario buffer shorter than N*n");
    }
};

}  // namespace sidr
