// ref_gpu_shim.cu -- extern "C" entry point over the reference's own GPU
// evaluator (augustompm/solver-informed-dispatching-rules,
// engine/factory.cuh: FactoryContext::evaluate_grouped_masks), compiled in
// place from the reference tree into oracle/_ref/libsidr_ref_gpu.so by
// oracle/Makefile with the reference Makefile's own nvcc flags (-O2, nvcc's
// default multiply-add contraction).  TEST INFRASTRUCTURE ONLY: it shows how
// the reference's GPU build differs from its CPU simulator on inputs where the
// campaign artefacts (made with that build) and the CPU simulator part ways.
//
// The reference kernel has no bounds checks (per-thread buffers of MAX_N
// customers and a MAX_STACK-deep stack), so every input is checked here
// before a launch: n <= MAX_N, well-formed post-order rules whose stack stays
// within MAX_STACK, slots < N_TERMS, scenario groups in range.
#include <algorithm>
#include <cstdint>
#include <vector>

#include "factory.cuh"

namespace {

bool rule_ok(const int32_t* ops, const int32_t* args, int L) {
    if (L < 1) return false;
    int sp = 0;
    for (int k = 0; k < L; k++) {
        const int o = ops[k];
        if (o == -1) {
            if (args[2 * k] < 0 || args[2 * k] >= N_TERMS) return false;
            sp++;
        } else if (o == -2) {
            sp++;
        } else if (o >= 0 && o <= 6) {
            if (sp < 2) return false;
            sp--;
        } else {
            return false;
        }
        if (sp > MAX_STACK) return false;
    }
    return sp == 1;
}

}  // namespace

extern "C" {

// out[P*T] = FactoryContext(sd, zp).evaluate_grouped_masks(...); returns 0,
// or -1 when an input is outside the kernel's bounds (nothing launched).
int ref_gpu_evaluate_grouped_masks(int n, int m, double tmax, const double* scores,
                                   const double* durations, const double* open_t,
                                   const double* close_t, const double* dist, const double* d2d,
                                   const double* zp, const int32_t* ops, const int32_t* args,
                                   const int32_t* offsets, const int32_t* lengths, int P,
                                   const double* grouped, int G, int T, int group_size,
                                   int mask_group, const int64_t* masks, double* out) {
    if (n < 1 || n > MAX_N || P < 1 || G < 1 || T < 1 || group_size < 1 || mask_group < 1)
        return -1;
    if ((P - 1) / group_size >= G) return -1;
    for (int p = 0; p < P; p++)
        if (offsets[p] < 0 || !rule_ok(ops + offsets[p], args + 2 * (size_t)offsets[p], lengths[p]))
            return -1;
    SimData sd;
    sd.n = n;
    sd.m = m;
    sd.ld = n + 1;
    sd.tmax = tmax;
    sd.scores.assign(scores, scores + n);
    sd.durations.assign(durations, durations + n);
    sd.open_t.assign(open_t, open_t + n);
    sd.close_t.assign(close_t, close_t + n);
    sd.dist.assign(dist, dist + (size_t)(n + 1) * (n + 1));
    sd.dist_to_depot.assign(d2d, d2d + n);
    PackedTrees pk;
    size_t nodes = 0;
    for (int p = 0; p < P; p++) nodes = std::max(nodes, (size_t)offsets[p] + lengths[p]);
    pk.ops.assign(ops, ops + nodes);
    pk.args.assign(args, args + 2 * nodes);
    pk.offsets.assign(offsets, offsets + P);
    pk.lengths.assign(lengths, lengths + P);
    const int n_masks = (P - 1) / mask_group + 1;
    std::vector<int64_t> mk(masks, masks + (size_t)n_masks * N_TERMS);
    std::vector<double> smp(grouped, grouped + (size_t)G * T * n);
    FactoryContext ctx(sd, std::vector<double>(zp, zp + 10));
    std::vector<double> r = ctx.evaluate_grouped_masks(pk, smp, T, group_size, mask_group, mk);
    std::copy(r.begin(), r.end(), out);
    return 0;
}

}  // extern "C"
