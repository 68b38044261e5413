// sidr_capi.cu -- the C-ABI of the evaluator (include/sidr.h).
//
// Contexts own the device copy of one instance and its lookup tables
// (FactoryContext's one-time upload, engine/factory.cuh:129-137).  Batches own
// one set of rules, scenarios and masks in HBM.  The reference-shaped
// evaluate* calls reuse grow-only device buffers held by the context instead of
// allocating and freeing per call (engine/factory.cuh:144-164 mallocs and frees
// seven buffers per call).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <mutex>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/sidr.h"
#include "../../include/sidr_surrogate.h"
#include "sidr_device.hpp"
#include "sidr_host.hpp"
#include "sidr_kernel.cuh"

using namespace sidr;

namespace {

thread_local std::string g_err;
thread_local long long g_h2d = 0, g_d2h = 0;
std::atomic<long long> g_launches{0};

// Op-model cost of one fused-scan neighbour for a rule's need set: the
// feasibility tests it shares plus each family's payload (counting only).
int scan_ops_of(uint32_t need) {
    int c = 0;
    if (need & (kNeedNSFused | kNeedRegret)) c += kOpsTest;
    if (need & kNeedNS) c += 2;
    if (need & kNeedMaxN) c += 2;
    if (need & kNeedReach2) c += 2;
    if (need & kNeedNSTW) c += 8;
    if (need & kNeedRegret) c += 1;
    if (need & kNeedRob) c += kOpsTest + 1;
    if (need & kNeedNSRob) c += 2;
    if (need & kNeedReach2Rob) c += 2;
    if (need & kNeedAfterC) c += kOpsTest;
    if (need & (kNeedStruct | kNeedPBust)) c += 6;
    if (need & kNeedReachK) c += 2;
    return c;
}

sidr_status fail(sidr_status s, const std::string& msg) {
    g_err = msg;
    return s;
}

#define SIDR_CUDA(call)                                                                      \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess)                                                               \
            return fail(SIDR_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// Grow-only device buffer.
struct DevBuf {
    void* p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t bytes) {
        if (bytes <= cap) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        size_t want = std::max<size_t>(bytes, 256);
        cudaError_t e = cudaMalloc(&p, want);
        if (e == cudaSuccess) cap = want;
        return e;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
};

// Rules compiled for one launch.
struct HostPrograms {
    std::vector<uint32_t> prog;
    std::vector<double> consts;
    std::vector<uint8_t> slots;
    std::vector<RuleMeta> meta;
    int rows = 1, prog_cap = 1, const_cap = 1;
    bool rmod = false;  // some rule has rmod instructions: the launch needs the RMOD kernel
};

}  // namespace

void sidr::set_last_error(const std::string& msg) { g_err = msg; }

struct sidr_ctx {
    int device = 0;
    int sm_count = 0;
    size_t smem_optin = 0;
    HostInstance h;
    DevInst inst{};
    std::vector<void*> owned;  // instance arrays and tables
    cudaStream_t stream = nullptr;
    int shape = 0;  // block shape of the reference-shaped evaluate* calls (sidr_ctx_set_shape)
    // grow-only scratch of the reference-shaped evaluate* calls
    DevBuf prog, consts, slots, meta, sampled, out, counter, stats, error;
};

struct sidr_batch {
    sidr_ctx* ctx = nullptr;
    DevBatch b{};
    int P = 0, T = 0, G = 0, group_size = 1;
    bool counting = false;
    bool rmod = false;  // the batch's rules use rmod
    int grid = 0, block = 0;  // the launch of shape 0 (also the counting launch's)
    size_t smem = 0;
    int shape = 0;                               // eval_kernel_fn's shape for sidr_batch_run
    int grid_s[SIDR_BATCH_SHAPES] = {}, block_s[SIDR_BATCH_SHAPES] = {};  // the launch of each shape
    size_t smem_s[SIDR_BATCH_SHAPES] = {};
    DevBuf prog, consts, slots, meta, sampled, out, counter, stats, error, fit;
    bool ran = false;
};

namespace {

sidr_status check_rules(const sidr_rules_desc* r) {
    if (!r) return fail(SIDR_ERR_INVALID, "rules descriptor is null");
    if (r->P < 0) return fail(SIDR_ERR_INVALID, "P < 0");
    if (r->P > 0 && (!r->ops || !r->args || !r->offsets || !r->lengths))
        return fail(SIDR_ERR_INVALID, "null rule array");
    for (int p = 0; p < r->P; p++) {
        const long long o = r->offsets[p], L = r->lengths[p];
        if (o < 0 || L < 1 || o + L > r->n_nodes)
            return fail(SIDR_ERR_INVALID, "rule " + std::to_string(p) + ": offset/length outside ops");
    }
    return SIDR_OK;
}

// Compile every rule under its mask row: row p/mask_group, or row_of[p] when
// given (multi-instance batches, where it is also the rule's instance).
sidr_status compile_all(const sidr_rules_desc* r, const int64_t* masks, int mask_group,
                        HostPrograms& hp, const int32_t* row_of = nullptr, bool all_active_rows = false) {
    hp = HostPrograms();
    hp.meta.resize(r->P);
    // compile every rule (independently, on the host's cores for large sets) ...
    std::vector<CompiledRule> crs(r->P);
    std::vector<std::string> errs(r->P);
    auto compile_range = [&](int lo, int hi) {
        for (int p = lo; p < hi; p++) {
            const int row = row_of ? row_of[p] : p / mask_group;
            const int64_t* M = masks + (size_t)row * kTerms;
            errs[p] = compile_rule(r->ops + r->offsets[p], r->args + 2 * (size_t)r->offsets[p],
                                   r->lengths[p], M, crs[p], all_active_rows);
        }
    };
    const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
    const int nt = r->P >= 2048 ? std::min(hw, 16) : 1;
    if (nt == 1) {
        compile_range(0, r->P);
    } else {
        std::vector<std::thread> ts;
        const int per = (r->P + nt - 1) / nt;
        for (int t = 0; t < nt; t++)
            ts.emplace_back(compile_range, std::min(r->P, t * per), std::min(r->P, (t + 1) * per));
        for (auto& t : ts) t.join();
    }
    // ... then lay them out in rule order
    for (int p = 0; p < r->P; p++) {
        const std::string& e = errs[p];
        if (!e.empty()) {
            const sidr_status s = (e.find("MAX_") != std::string::npos) ? SIDR_ERR_TOO_LARGE
                                                                        : SIDR_ERR_RULE;
            return fail(s, "rule " + std::to_string(p) + ": " + e);
        }
        const CompiledRule& cr = crs[p];
        RuleMeta& m = hp.meta[p];
        m.prog_off = (int32_t)hp.prog.size();
        m.const_off = (int32_t)hp.consts.size();
        m.slot_off = (int32_t)hp.slots.size();
        m.n_ins = (int16_t)cr.prog.size();
        m.n_const = (int16_t)cr.consts.size();
        m.K = (int16_t)cr.K;
        m.D = (int16_t)cr.D;
        m.res = (int16_t)cr.res;
        m.reach_k = (int8_t)cr.reach_k;
        m.scan_ops = (uint16_t)scan_ops_of(cr.need);
        m.inst = (int16_t)(row_of ? row_of[p] : 0);
        m.need = cr.need;
        m.explore = cr.explore;
        hp.prog.insert(hp.prog.end(), cr.prog.begin(), cr.prog.end());
        hp.consts.insert(hp.consts.end(), cr.consts.begin(), cr.consts.end());
        hp.slots.insert(hp.slots.end(), cr.slots.begin(), cr.slots.end());
        hp.rows = std::max(hp.rows, cr.K + cr.D);
        hp.rmod = hp.rmod || (cr.need & kNeedRmod) != 0;
        hp.prog_cap = std::max(hp.prog_cap, (int)cr.prog.size());
        hp.const_cap = std::max(hp.const_cap, (int)cr.consts.size());
    }
    if (hp.prog.empty()) hp.prog.push_back(0);
    if (hp.consts.empty()) hp.consts.push_back(0.0);
    if (hp.slots.empty()) hp.slots.push_back(0);
    return SIDR_OK;
}

sidr_status check_grouping(const sidr_rules_desc* r, const double* sampled, int G, int T,
                           int group_size, int mask_group, const int64_t* masks) {
    if (T < 0 || G < 0) return fail(SIDR_ERR_INVALID, "negative scenario count");
    if (group_size < 1 || mask_group < 1) return fail(SIDR_ERR_INVALID, "group sizes must be >= 1");
    if (r->P > 0 && T > 0) {
        if ((long long)(r->P - 1) / group_size >= G)
            return fail(SIDR_ERR_INVALID, "rules address scenario groups beyond G");
        if (!sampled) return fail(SIDR_ERR_INVALID, "scenario buffer is null");
    }
    if (r->P > 0 && !masks) return fail(SIDR_ERR_INVALID, "mask buffer is null");
    return SIDR_OK;
}

sidr_status check_finite(const double* v, size_t count) {
    for (size_t k = 0; k < count; k++)
        if (!std::isfinite(v[k]))
            return fail(SIDR_ERR_NONFINITE, "non-finite sampled duration at index " + std::to_string(k));
    return SIDR_OK;
}

template <class T>
cudaError_t upload(DevBuf& buf, const std::vector<T>& v, cudaStream_t st) {
    cudaError_t e = buf.ensure(v.size() * sizeof(T));
    if (e != cudaSuccess) return e;
    return cudaMemcpyAsync(buf.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st);
}

const char* kernel_error_text(int code) {
    switch (code) {
    case kErrRuleRecord: return "a rule record exceeds the launch's shared-memory slice";
    case kErrRuleIndex: return "a work item names a rule outside the batch";
    case kErrInstance: return "a rule names an instance outside the batch";
    }
    return "unknown kernel error code";
}

// Reads the kernel error word once the stream's work is done (this syncs the
// stream); SIDR_ERR_KERNEL when a launch raised it.
sidr_status read_error_word(const int* dev_word, cudaStream_t st) {
    int h = 0;
    SIDR_CUDA(cudaMemcpyAsync(&h, dev_word, sizeof(int), cudaMemcpyDeviceToHost, st));
    SIDR_CUDA(cudaStreamSynchronize(st));
    if (h) return fail(SIDR_ERR_KERNEL, std::string("evaluator kernel: ") + kernel_error_text(h));
    return SIDR_OK;
}

// The single-instance kernel for a launch: counting instantiation or not, with
// or without the rmod code (only batches that use rmod pay for it), and the
// block shape: {resident blocks per SM the registers are budgeted for, lanes
// per pair} (the counting instantiation exists for shape 0 only).
constexpr int kBatchShapes[SIDR_BATCH_SHAPES][2] = {
    {SIDR_MIN_BLOCKS, 32}, {kMoreBlocks, 32}, {SIDR_MIN_BLOCKS, 16}, {kMoreBlocks, 16}};
const void* eval_kernel_fn(bool counting, bool rmod, int shape = 0) {
    if (counting)
        return rmod ? (const void*)eval_kernel<true, true, SIDR_MIN_BLOCKS>
                    : (const void*)eval_kernel<true, false, SIDR_MIN_BLOCKS>;
    switch (shape) {
    case 1:
        return rmod ? (const void*)eval_kernel<false, true, kMoreBlocks>
                    : (const void*)eval_kernel<false, false, kMoreBlocks>;
    case 2:
        return rmod ? (const void*)eval_kernel<false, true, SIDR_MIN_BLOCKS, 16>
                    : (const void*)eval_kernel<false, false, SIDR_MIN_BLOCKS, 16>;
    case 3:
        return rmod ? (const void*)eval_kernel<false, true, kMoreBlocks, 16>
                    : (const void*)eval_kernel<false, false, kMoreBlocks, 16>;
    default:
        return rmod ? (const void*)eval_kernel<false, true, SIDR_MIN_BLOCKS>
                    : (const void*)eval_kernel<false, false, SIDR_MIN_BLOCKS>;
    }
}

// Launch geometry for a program set: warps per block bounded by the shared
// memory each warp's pair groups take; one persistent grid over all SMs.
sidr_status plan_launch(sidr_ctx* c, const HostPrograms& hp, long long items, bool counting,
                        int& grid, int& block, size_t& smem, int shape = 0) {
    const int lpp = counting ? 32 : kBatchShapes[shape][1];
    const int gpw = 32 / lpp;  // pairs per warp
    const size_t slice = warp_slice_bytes(hp.rows, hp.const_cap, hp.prog_cap, lpp) * gpw;
    if (slice > c->smem_optin)
        return fail(SIDR_ERR_TOO_LARGE, "rule programs need more shared memory than one block has");
    int wpb = (int)std::min<size_t>(SIDR_WARPS_PER_BLOCK, c->smem_optin / slice);
    if (wpb < 1) wpb = 1;
    block = 32 * wpb;
    smem = slice * wpb;
    const void* fn = eval_kernel_fn(counting, hp.rmod, shape);
    SIDR_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    SIDR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, block, smem));
    if (per_sm < 1) per_sm = 1;
    const long long per_block = (long long)wpb * gpw;
    long long want = (items + per_block - 1) / per_block;
    grid = (int)std::max<long long>(1, std::min<long long>(want, (long long)c->sm_count * per_sm));
    return SIDR_OK;
}

sidr_status launch(sidr_ctx* c, const DevBatch& b, bool counting, bool rmod, int grid, int block,
                   size_t smem, cudaStream_t st, int shape = 0) {
    SIDR_CUDA(cudaMemsetAsync(b.counter, 0, sizeof(unsigned long long), st));
    if (b.error) SIDR_CUDA(cudaMemsetAsync(b.error, 0, sizeof(int), st));
    if (counting && b.stats) SIDR_CUDA(cudaMemsetAsync(b.stats, 0, kStats * sizeof(unsigned long long), st));
    if ((long long)b.P * b.T == 0) return SIDR_OK;
    DevInst inst = c->inst;
    DevBatch bb = b;
    void* args[] = {&inst, &bb};
    SIDR_CUDA(cudaLaunchKernel(eval_kernel_fn(counting, rmod, counting ? 0 : shape), dim3(grid),
                               dim3(block), args, smem, st));
    g_launches.fetch_add(1);
    return SIDR_OK;
}

// FP64 pipe probe: 8 independent add/multiply chains per thread.
__global__ void fp64_probe_kernel(double* sink, int iters, double a, double b) {
    double x[8];
#pragma unroll
    for (int k = 0; k < 8; k++) x[k] = a + threadIdx.x * 1e-9 + k;
    for (int it = 0; it < iters; it++) {
#pragma unroll
        for (int k = 0; k < 8; k++) x[k] = __fma_rn(x[k], b, a);  // one DFMA per chain
    }
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 8; k++) s += x[k];
    if (s == 1234.5) sink[threadIdx.x] = s;
}

__global__ void fitness_kernel(const double* out, int P, int T, double* fit) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P) return;
    double acc = 0.0;
    for (int s = 0; s < T; s++) acc += out[(size_t)p * T + s];
    fit[p] = acc / T;
}

// An NVTX range for the scope: shows the library's calls on a profiler's
// timeline (no cost beyond a branch when no tool is attached).
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
};

// Shared body of the three reference-shaped evaluate calls.
sidr_status evaluate_common(sidr_ctx* c, const sidr_rules_desc* r, const double* sampled, int G,
                            int T, int group_size, int mask_group, const int64_t* masks,
                            double* out) {
    NvtxRange range("sidr_evaluate");
    if (!c) return fail(SIDR_ERR_INVALID, "context is null");
    g_h2d = g_d2h = 0;
    sidr_status s = check_rules(r);
    if (s) return s;
    s = check_grouping(r, sampled, G, T, group_size, mask_group, masks);
    if (s) return s;
    if (r->P > 0 && T > 0 && !out) return fail(SIDR_ERR_INVALID, "output buffer is null");
    const int P = r->P;
    if ((long long)P * T == 0) return SIDR_OK;
    const int groups_used = (P - 1) / group_size + 1;
    const size_t n_smp = (size_t)groups_used * T * c->h.n;
    s = check_finite(sampled, n_smp);
    if (s) return s;
    HostPrograms hp;
    s = compile_all(r, masks, mask_group, hp);
    if (s) return s;
    g_h2d = (long long)(hp.prog.size() * 4 + hp.consts.size() * 8 + hp.slots.size() +
                        hp.meta.size() * sizeof(RuleMeta) + n_smp * 8);
    g_d2h = (long long)P * T * 8;
    DeviceGuard device_guard;
    SIDR_CUDA(cudaSetDevice(c->device));
    cudaStream_t st = c->stream;
    SIDR_CUDA(upload(c->prog, hp.prog, st));
    SIDR_CUDA(upload(c->consts, hp.consts, st));
    SIDR_CUDA(upload(c->slots, hp.slots, st));
    SIDR_CUDA(upload(c->meta, hp.meta, st));
    SIDR_CUDA(c->sampled.ensure(n_smp * sizeof(double)));
    SIDR_CUDA(cudaMemcpyAsync(c->sampled.p, sampled, n_smp * sizeof(double), cudaMemcpyHostToDevice, st));
    SIDR_CUDA(c->out.ensure((size_t)P * T * sizeof(double)));
    SIDR_CUDA(c->counter.ensure(sizeof(unsigned long long)));
    SIDR_CUDA(c->error.ensure(sizeof(int)));
    SIDR_CUDA(cudaMemsetAsync(c->error.p, 0, sizeof(int), st));
    DevBatch b{};
    b.P = P;
    b.T = T;
    b.group_size = group_size;
    b.n = c->h.n;
    b.prog = (const uint32_t*)c->prog.p;
    b.consts = (const double*)c->consts.p;
    b.slots = (const uint8_t*)c->slots.p;
    b.meta = (const RuleMeta*)c->meta.p;
    b.sampled = (const double*)c->sampled.p;
    b.out = (double*)c->out.p;
    b.counter = (unsigned long long*)c->counter.p;
    b.stats = nullptr;
    b.error = (int*)c->error.p;
    b.rows = hp.rows;
    b.prog_cap = hp.prog_cap;
    b.const_cap = hp.const_cap;
    int grid, block;
    size_t smem;
    s = plan_launch(c, hp, (long long)P * T, false, grid, block, smem, c->shape);
    if (s) return s;
    s = launch(c, b, false, hp.rmod, grid, block, smem, st, c->shape);
    if (s) return s;
    SIDR_CUDA(cudaMemcpyAsync(out, c->out.p, (size_t)P * T * sizeof(double), cudaMemcpyDeviceToHost, st));
    return read_error_word(b.error, st);
}

}  // namespace

extern "C" {

const char* sidr_last_error(void) { return g_err.c_str(); }

const char* sidr_status_string(sidr_status s) {
    switch (s) {
    case SIDR_OK: return "ok";
    case SIDR_ERR_INVALID: return "invalid argument";
    case SIDR_ERR_RULE: return "malformed rule";
    case SIDR_ERR_TOO_LARGE: return "size limit exceeded";
    case SIDR_ERR_CUDA: return "CUDA error";
    case SIDR_ERR_NO_DEVICE: return "no CUDA device";
    case SIDR_ERR_KERNEL: return "kernel fault";
    case SIDR_ERR_NONFINITE: return "non-finite input";
    }
    return "unknown status";
}

int sidr_version(void) { return 100; }

int64_t sidr_kernel_launches(void) { return g_launches.load(); }

sidr_status sidr_last_transfer_bytes(int64_t* h2d, int64_t* d2h) {
    if (h2d) *h2d = g_h2d;
    if (d2h) *d2h = g_d2h;
    return SIDR_OK;
}

sidr_status sidr_fp64_peak(int device, int reps, double* ops_per_s) {
    if (!ops_per_s) return fail(SIDR_ERR_INVALID, "null argument");
    DeviceGuard device_guard;
    SIDR_CUDA(cudaSetDevice(device));
    int sms = 0;
    SIDR_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    double* sink = nullptr;
    SIDR_CUDA(cudaMalloc(&sink, 1024 * sizeof(double)));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int iters = 4096, threads = 512, blocks = sms * 4;
    float best = 1e30f;
    for (int r = 0; r < (reps < 1 ? 1 : reps) + 1; r++) {
        cudaEventRecord(e0);
        fp64_probe_kernel<<<blocks, threads>>>(sink, iters, 1.0000001, 0.9999999);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (r > 0 && ms < best) best = ms;  // first run is warm-up
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    SIDR_CUDA(cudaGetLastError());
    // each fused multiply-add is one instruction of the FP64 pipe = one op here
    const double ops = (double)blocks * threads * iters * 8.0;
    *ops_per_s = ops / (best * 1e-3);
    return SIDR_OK;
}

sidr_status sidr_capture_situations(sidr_ctx* c, const sidr_rules_desc* r, const double* sampled,
                                    int32_t S, const int64_t* mask, int32_t max_decisions,
                                    int32_t max_cand, double* terms, int32_t* cust, int32_t* info) {
    if (!c || !r || !mask || !sampled || !terms || !info) return fail(SIDR_ERR_INVALID, "null argument");
    if (r->P != 1) return fail(SIDR_ERR_INVALID, "capture takes exactly one rule");
    if (S < 1 || max_decisions < 1 || max_cand < 1) return fail(SIDR_ERR_INVALID, "S, max_decisions, max_cand >= 1");
    sidr_status s = check_rules(r);
    if (s) return s;
    const size_t n_smp = (size_t)S * c->h.n;
    if ((s = check_finite(sampled, n_smp))) return s;
    HostPrograms hp;
    if ((s = compile_all(r, mask, 1, hp, nullptr, true))) return s;
    const int K = hp.meta[0].K;
    std::vector<int> slot_of(hp.slots.begin(), hp.slots.begin() + K);  // row -> slot
    DeviceGuard device_guard;
    SIDR_CUDA(cudaSetDevice(c->device));
    cudaStream_t st = c->stream;
    SIDR_CUDA(upload(c->prog, hp.prog, st));
    SIDR_CUDA(upload(c->consts, hp.consts, st));
    SIDR_CUDA(upload(c->slots, hp.slots, st));
    SIDR_CUDA(upload(c->meta, hp.meta, st));
    SIDR_CUDA(c->sampled.ensure(n_smp * sizeof(double)));
    SIDR_CUDA(cudaMemcpyAsync(c->sampled.p, sampled, n_smp * sizeof(double), cudaMemcpyHostToDevice, st));
    SIDR_CUDA(c->out.ensure((size_t)S * sizeof(double)));
    SIDR_CUDA(c->counter.ensure(sizeof(unsigned long long)));
    SIDR_CUDA(c->error.ensure(sizeof(int)));
    SIDR_CUDA(cudaMemsetAsync(c->error.p, 0, sizeof(int), st));
    const size_t slots_n = (size_t)S * max_decisions, cand_n = slots_n * max_cand;
    double* d_rows = nullptr;
    int32_t *d_cust = nullptr, *d_info = nullptr;
    cudaError_t e = cudaMalloc(&d_rows, cand_n * K * sizeof(double));
    if (!e) e = cudaMalloc(&d_cust, cand_n * sizeof(int32_t));
    if (!e) e = cudaMalloc(&d_info, slots_n * 2 * sizeof(int32_t));
    if (!e) e = cudaMemsetAsync(d_info, 0, slots_n * 2 * sizeof(int32_t), st);
    if (!e) e = cudaMemsetAsync(c->counter.p, 0, sizeof(unsigned long long), st);
    DevBatch b{};
    b.P = 1;
    b.T = S;
    b.group_size = 1;
    b.n = c->h.n;
    b.prog = (const uint32_t*)c->prog.p;
    b.consts = (const double*)c->consts.p;
    b.slots = (const uint8_t*)c->slots.p;
    b.meta = (const RuleMeta*)c->meta.p;
    b.sampled = (const double*)c->sampled.p;
    b.out = (double*)c->out.p;
    b.counter = (unsigned long long*)c->counter.p;
    b.error = (int*)c->error.p;
    b.rows = hp.rows;
    b.prog_cap = hp.prog_cap;
    b.const_cap = hp.const_cap;
    CaptureBuf cb{d_rows, d_cust, d_info, max_decisions, max_cand, K};
    const size_t slice = warp_slice_bytes(hp.rows, hp.const_cap, hp.prog_cap);
    const int wpb = SIDR_WARPS_PER_BLOCK;
    const size_t smem = slice * wpb;
    if (!e && smem > c->smem_optin) e = cudaErrorInvalidValue;
    if (!e) e = cudaFuncSetAttribute(capture_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (!e) {
        const int grid = std::max(1, std::min((S + wpb - 1) / wpb, c->sm_count * 2));
        capture_kernel<<<grid, 32 * wpb, smem, st>>>(c->inst, b, cb);
        e = cudaGetLastError();
        g_launches++;
    }
    std::vector<double> rows;
    std::vector<int32_t> cu;
    if (!e) {
        rows.resize(cand_n * K);
        cu.resize(cand_n);
        e = cudaMemcpyAsync(rows.data(), d_rows, rows.size() * sizeof(double), cudaMemcpyDeviceToHost, st);
    }
    if (!e) e = cudaMemcpyAsync(cu.data(), d_cust, cu.size() * sizeof(int32_t), cudaMemcpyDeviceToHost, st);
    if (!e) e = cudaMemcpyAsync(info, d_info, slots_n * 2 * sizeof(int32_t), cudaMemcpyDeviceToHost, st);
    if (!e) e = cudaStreamSynchronize(st);
    cudaFree(d_rows);
    cudaFree(d_cust);
    cudaFree(d_info);
    if (e) return fail(SIDR_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(e));
    if ((s = read_error_word(b.error, st))) return s;
    // rows -> 61-slot tables: captured slots, C1..C5 where active, zero elsewhere
    static const double kC[5] = {0.1, 0.2, 0.3, 0.4, 0.5};
    for (size_t q = 0; q < cand_n; q++) {
        double* t = terms + q * kTerms;
        for (int k = 0; k < kTerms; k++) t[k] = 0.0;
        for (int k = 36; k <= 40; k++)
            if (slot_active(k, mask)) t[k] = kC[k - 36];
        for (int k = 0; k < K; k++) t[slot_of[k]] = rows[q * K + k];
    }
    if (cust) std::memcpy(cust, cu.data(), cu.size() * sizeof(int32_t));
    return SIDR_OK;
}

__global__ void libm_kernel(int fn, const double* x, long long n, double* out) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const double v = x[i];
        out[i] = fn == 0 ? libm::erf_(v) : fn == 1 ? libm::erfc_(v) : libm::exp_(v);
    }
}

sidr_status sidr_libm_eval(int32_t fn, const double* x, int64_t n, int device, double* out) {
    if (fn < 0 || fn > 2 || n < 0 || (n > 0 && (!x || !out))) return fail(SIDR_ERR_INVALID, "bad argument");
    if (n == 0) return SIDR_OK;
    DeviceGuard device_guard;
    SIDR_CUDA(cudaSetDevice(device));
    double *dx = nullptr, *dout = nullptr;
    SIDR_CUDA(cudaMalloc(&dx, (size_t)n * sizeof(double)));
    cudaError_t e = cudaMalloc(&dout, (size_t)n * sizeof(double));
    if (e == cudaSuccess) e = cudaMemcpy(dx, x, (size_t)n * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        libm_kernel<<<(int)std::min<long long>((n + 255) / 256, 4096), 256>>>(fn, dx, n, dout);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(out, dout, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(dx);
    cudaFree(dout);
    if (e != cudaSuccess) return fail(SIDR_ERR_CUDA, std::string("libm eval: ") + cudaGetErrorString(e));
    return SIDR_OK;
}

__global__ void libm_pow_kernel(const double* x, const double* y, long long n, double* out) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        out[i] = libm::pow_(x[i], y[i]);
}

sidr_status sidr_libm_pow(const double* x, const double* y, int64_t n, int device, double* out) {
    if (n < 0 || (n > 0 && (!x || !y || !out))) return fail(SIDR_ERR_INVALID, "bad argument");
    if (n == 0) return SIDR_OK;
    DeviceGuard device_guard;
    SIDR_CUDA(cudaSetDevice(device));
    double* d = nullptr;  // x, y, out
    SIDR_CUDA(cudaMalloc(&d, 3 * (size_t)n * sizeof(double)));
    cudaError_t e = cudaMemcpy(d, x, (size_t)n * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d + n, y, (size_t)n * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        libm_pow_kernel<<<(int)std::min<long long>((n + 255) / 256, 4096), 256>>>(d, d + n, n, d + 2 * n);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(out, d + 2 * n, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return fail(SIDR_ERR_CUDA, std::string("libm pow: ") + cudaGetErrorString(e));
    return SIDR_OK;
}

sidr_status sidr_rules_check(const sidr_rules_desc* r, const int64_t* masks, int32_t mask_group,
                             int32_t* max_rows) {
    sidr_status s = check_rules(r);
    if (s) return s;
    if (mask_group < 1) return fail(SIDR_ERR_INVALID, "mask_group must be >= 1");
    if (r->P > 0 && !masks) return fail(SIDR_ERR_INVALID, "mask buffer is null");
    HostPrograms hp;
    if (r->P > 0) {
        s = compile_all(r, masks, mask_group, hp);
        if (s) return s;
    }
    if (max_rows) *max_rows = hp.rows;
    return SIDR_OK;
}

sidr_status sidr_zstats(const sidr_instance_desc* d, double zp[10]) {
    if (!d || !zp) return fail(SIDR_ERR_INVALID, "null argument");
    HostInstance h;
    std::string e = build_instance(d->n, d->m, d->tmax, d->scores, d->durations, d->open_t,
                                   d->close_t, d->dist, d->dist_to_depot, h, false);
    if (!e.empty()) return fail(e.find("finite") != std::string::npos ? SIDR_ERR_NONFINITE
                                : (d->n > kMaxN ? SIDR_ERR_TOO_LARGE : SIDR_ERR_INVALID), e);
    host_zstats(h, zp);
    return SIDR_OK;
}

sidr_status sidr_atrisk_table_check(const sidr_instance_desc* d, int32_t seed, int64_t* checked,
                                    int64_t* mismatches) {
    if (!d || !checked || !mismatches) return fail(SIDR_ERR_INVALID, "null argument");
    HostInstance h;
    std::string e = build_instance(d->n, d->m, d->tmax, d->scores, d->durations, d->open_t,
                                   d->close_t, d->dist, d->dist_to_depot, h, true);
    if (!e.empty()) return fail(SIDR_ERR_INVALID, e);
    long long c = 0, b = 0;
    atrisk_table_check(h, seed, c, b);
    *checked = c;
    *mismatches = b;
    return SIDR_OK;
}

sidr_status sidr_ctx_create(const sidr_instance_desc* d, const double zp[10], int device,
                            sidr_ctx** out) {
    if (!out) return fail(SIDR_ERR_INVALID, "out is null");
    *out = nullptr;
    if (!d || !zp) return fail(SIDR_ERR_INVALID, "null argument");
    for (int k = 0; k < 10; k++)
        if (std::isnan(zp[k])) return fail(SIDR_ERR_NONFINITE, "zp holds NaN");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
        cudaGetLastError();
        return fail(SIDR_ERR_NO_DEVICE, "no CUDA device");
    }
    if (device < 0 || device >= ndev) return fail(SIDR_ERR_INVALID, "device index out of range");
    sidr_ctx* c = new sidr_ctx();
    std::string e = build_instance(d->n, d->m, d->tmax, d->scores, d->durations, d->open_t,
                                   d->close_t, d->dist, d->dist_to_depot, c->h, true);
    if (!e.empty()) {
        delete c;
        return fail(e.find("finite") != std::string::npos ? SIDR_ERR_NONFINITE
                    : (d->n > kMaxN ? SIDR_ERR_TOO_LARGE : SIDR_ERR_INVALID), e);
    }
    c->device = device;
    auto bail = [&](cudaError_t err, const char* what) {
        sidr_ctx_destroy(c);
        return fail(SIDR_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(err));
    };
    DeviceGuard device_guard;
    cudaError_t err = cudaSetDevice(device);
    if (err != cudaSuccess) return bail(err, "cudaSetDevice");
    int v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device);
    c->sm_count = v;
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    c->smem_optin = (size_t)v;
    err = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (err != cudaSuccess) return bail(err, "cudaStreamCreate");
    auto put = [&](const void* src, size_t bytes, const void** dst) -> cudaError_t {
        void* p = nullptr;
        cudaError_t e2 = cudaMalloc(&p, std::max<size_t>(bytes, 8));
        if (e2 != cudaSuccess) return e2;
        c->owned.push_back(p);
        *dst = p;
        return cudaMemcpy(p, src, bytes, cudaMemcpyHostToDevice);
    };
    const HostInstance& h = c->h;
    DevInst& I = c->inst;
    I.n = h.n;
    I.m = h.m;
    I.ld = h.n + 1;
    I.nw = h.nw;
    I.tmax = h.tmax;
    I.ns = h.ns;
    struct Item { const void* src; size_t bytes; const void** dst; };
    const Item items[] = {
        {h.scores.data(), (size_t)h.n * 8, (const void**)&I.scores},
        {h.durations.data(), (size_t)h.n * 8, (const void**)&I.durations},
        {h.open_t.data(), (size_t)h.n * 8, (const void**)&I.open_t},
        {h.close_t.data(), (size_t)h.n * 8, (const void**)&I.close_t},
        {h.d2d.data(), (size_t)h.n * 8, (const void**)&I.d2d},
        {h.dist.data(), h.dist.size() * 8, (const void**)&I.dist},
        {h.F.data(), h.F.size() * 8, (const void**)&I.F},
        {h.G.data(), h.G.size() * 8, (const void**)&I.G},
        {h.R.data(), h.R.size() * 8, (const void**)&I.R},
        {h.P1.data(), h.P1.size() * 8, (const void**)&I.P1},
        {h.P0.data(), h.P0.size() * 8, (const void**)&I.P0},
        {h.zlt.data(), h.zlt.size() * 4, (const void**)&I.zlt},
        {h.zle.data(), h.zle.size() * 4, (const void**)&I.zle},
        {h.FR.data(), h.FR.size() * 8, (const void**)&I.FR},
        {h.GD.data(), h.GD.size() * 8, (const void**)&I.GD},
        {h.DP.data(), h.DP.size() * 8, (const void**)&I.DP},
        {h.CU.data(), h.CU.size() * 8, (const void**)&I.CU},
        {h.TK.data(), h.TK.size() * 8, (const void**)&I.TK},
        {h.TC.data(), h.TC.size(), (const void**)&I.TC},
        {h.ord.data(), h.ord.size() * 2, (const void**)&I.ord},
        {h.sF.data(), h.sF.size() * 8, (const void**)&I.sF},
        {h.sG.data(), h.sG.size() * 8, (const void**)&I.sG},
        {h.bF.data(), h.bF.size() * 8, (const void**)&I.bF},
        {h.bG.data(), h.bG.size() * 8, (const void**)&I.bG},
        {h.cnt_pos.data(), h.cnt_pos.size() * 4, (const void**)&I.cnt_pos},
        {h.cnt_gm1.data(), h.cnt_gm1.size() * 4, (const void**)&I.cnt_gm1},
        {zp, 80, (const void**)&I.zp},
    };
    for (const Item& it : items) {
        err = put(it.src, it.bytes, it.dst);
        if (err != cudaSuccess) return bail(err, "instance upload");
    }
    *out = c;
    return SIDR_OK;
}

void sidr_ctx_destroy(sidr_ctx* c) {
    if (!c) return;
    DeviceGuard device_guard;
    cudaSetDevice(c->device);
    for (void* p : c->owned) cudaFree(p);
    for (DevBuf* b : {&c->prog, &c->consts, &c->slots, &c->meta, &c->sampled, &c->out, &c->counter,
                      &c->stats, &c->error})
        b->release();
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

sidr_status sidr_evaluate(sidr_ctx* c, const sidr_rules_desc* r, const double* sampled, int32_t N,
                          const int64_t* term_mask, double* out) {
    const int P = r ? r->P : 0;
    return evaluate_common(c, r, sampled, 1, N, P > 0 ? P : 1, P > 0 ? P : 1, term_mask, out);
}

sidr_status sidr_evaluate_grouped(sidr_ctx* c, const sidr_rules_desc* r,
                                  const double* grouped_sampled, int32_t G, int32_t T,
                                  int32_t group_size, const int64_t* term_mask, double* out) {
    const int P = r ? r->P : 0;
    return evaluate_common(c, r, grouped_sampled, G, T, group_size, P > 0 ? P : 1, term_mask, out);
}

sidr_status sidr_evaluate_grouped_masks(sidr_ctx* c, const sidr_rules_desc* r,
                                        const double* grouped_sampled, int32_t G, int32_t T,
                                        int32_t group_size, int32_t mask_group,
                                        const int64_t* masks, double* out) {
    return evaluate_common(c, r, grouped_sampled, G, T, group_size, mask_group, masks, out);
}

sidr_status sidr_batch_create(sidr_ctx* c, const sidr_rules_desc* r, const double* sampled,
                              int32_t G, int32_t T, int32_t group_size, int32_t mask_group,
                              const int64_t* masks, sidr_batch** out) {
    if (!out) return fail(SIDR_ERR_INVALID, "out is null");
    *out = nullptr;
    if (!c) return fail(SIDR_ERR_INVALID, "context is null");
    sidr_status s = check_rules(r);
    if (s) return s;
    s = check_grouping(r, sampled, G, T, group_size, mask_group, masks);
    if (s) return s;
    const int P = r->P;
    const int groups_used = P > 0 ? (P - 1) / group_size + 1 : 0;
    const size_t n_smp = (size_t)groups_used * T * c->h.n;
    if (P > 0 && T > 0) {
        s = check_finite(sampled, n_smp);
        if (s) return s;
    }
    HostPrograms hp;
    if (P > 0) {
        s = compile_all(r, masks, mask_group, hp);
        if (s) return s;
    } else {
        hp.prog.push_back(0);
        hp.consts.push_back(0.0);
        hp.slots.push_back(0);
    }
    DeviceGuard device_guard;
    SIDR_CUDA(cudaSetDevice(c->device));
    sidr_batch* bt = new sidr_batch();
    bt->ctx = c;
    bt->P = P;
    bt->T = T;
    bt->G = G;
    bt->group_size = group_size;
    bt->rmod = hp.rmod;
    auto bail = [&](cudaError_t err, const char* what) {
        sidr_batch_destroy(bt);
        return fail(SIDR_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(err));
    };
    cudaStream_t st = c->stream;
    cudaError_t err;
    if ((err = upload(bt->prog, hp.prog, st)) != cudaSuccess) return bail(err, "upload programs");
    if ((err = upload(bt->consts, hp.consts, st)) != cudaSuccess) return bail(err, "upload constants");
    if ((err = upload(bt->slots, hp.slots, st)) != cudaSuccess) return bail(err, "upload slots");
    if (!hp.meta.empty() && (err = upload(bt->meta, hp.meta, st)) != cudaSuccess)
        return bail(err, "upload rule table");
    if ((err = bt->sampled.ensure(std::max<size_t>(n_smp, 1) * sizeof(double))) != cudaSuccess)
        return bail(err, "alloc scenarios");
    if (n_smp && (err = cudaMemcpyAsync(bt->sampled.p, sampled, n_smp * sizeof(double),
                                        cudaMemcpyHostToDevice, st)) != cudaSuccess)
        return bail(err, "upload scenarios");
    if ((err = bt->out.ensure(std::max<size_t>((size_t)P * T, 1) * sizeof(double))) != cudaSuccess)
        return bail(err, "alloc output");
    if ((err = bt->fit.ensure(std::max<size_t>((size_t)P, 1) * sizeof(double))) != cudaSuccess)
        return bail(err, "alloc fitness");
    if ((err = bt->counter.ensure(sizeof(unsigned long long))) != cudaSuccess) return bail(err, "alloc counter");
    if ((err = bt->stats.ensure(kStats * sizeof(unsigned long long))) != cudaSuccess) return bail(err, "alloc stats");
    if ((err = bt->error.ensure(sizeof(int))) != cudaSuccess) return bail(err, "alloc error word");
    if ((err = cudaMemsetAsync(bt->error.p, 0, sizeof(int), st)) != cudaSuccess) return bail(err, "memset");
    if ((err = cudaStreamSynchronize(st)) != cudaSuccess) return bail(err, "sync");
    DevBatch& b = bt->b;
    b.P = P;
    b.T = T;
    b.group_size = group_size;
    b.n = c->h.n;
    b.prog = (const uint32_t*)bt->prog.p;
    b.consts = (const double*)bt->consts.p;
    b.slots = (const uint8_t*)bt->slots.p;
    b.meta = (const RuleMeta*)bt->meta.p;
    b.sampled = (const double*)bt->sampled.p;
    b.out = (double*)bt->out.p;
    b.counter = (unsigned long long*)bt->counter.p;
    b.stats = (unsigned long long*)bt->stats.p;
    b.error = (int*)bt->error.p;
    b.rows = hp.rows;
    b.prog_cap = hp.prog_cap;
    b.const_cap = hp.const_cap;
    s = plan_launch(c, hp, (long long)P * T, false, bt->grid, bt->block, bt->smem);
    for (int sh = 1; sh < SIDR_BATCH_SHAPES && !s; sh++)
        s = plan_launch(c, hp, (long long)P * T, false, bt->grid_s[sh], bt->block_s[sh], bt->smem_s[sh], sh);
    if (s) {
        sidr_batch_destroy(bt);
        return s;
    }
    bt->grid_s[0] = bt->grid;
    bt->block_s[0] = bt->block;
    bt->smem_s[0] = bt->smem;
    int g2, b2;
    size_t s2;
    s = plan_launch(c, hp, (long long)P * T, true, g2, b2, s2);
    if (s) {
        sidr_batch_destroy(bt);
        return s;
    }
    *out = bt;
    return SIDR_OK;
}

sidr_status sidr_batch_set_counting(sidr_batch* b, int enable) {
    if (!b) return fail(SIDR_ERR_INVALID, "batch is null");
    b->counting = enable != 0;
    return SIDR_OK;
}

sidr_status sidr_batch_run(sidr_batch* bt, void* stream) {
    NvtxRange range("sidr_batch_run");
    if (!bt) return fail(SIDR_ERR_INVALID, "batch is null");
    DeviceGuard device_guard;
    SIDR_CUDA(cudaSetDevice(bt->ctx->device));
    cudaStream_t st = (cudaStream_t)stream;  // 0 = the legacy default stream
    const int sh = bt->counting ? 0 : bt->shape;
    sidr_status s = launch(bt->ctx, bt->b, bt->counting, bt->rmod, bt->grid_s[sh], bt->block_s[sh],
                           bt->smem_s[sh], st, sh);
    if (s) return s;
    if (bt->P > 0) {
        fitness_kernel<<<(bt->P + 127) / 128, 128, 0, st>>>(bt->b.out, bt->P, bt->T,
                                                            (double*)bt->fit.p);
        SIDR_CUDA(cudaGetLastError());
        g_launches.fetch_add(1);
    }
    bt->ran = true;
    return SIDR_OK;
}

sidr_status sidr_ctx_set_shape(sidr_ctx* c, int32_t shape) {
    if (!c) return fail(SIDR_ERR_INVALID, "context is null");
    if (shape < 0 || shape >= SIDR_BATCH_SHAPES) return fail(SIDR_ERR_INVALID, "shape out of range");
    c->shape = shape;
    return SIDR_OK;
}

sidr_status sidr_batch_set_shape(sidr_batch* bt, int32_t shape) {
    if (!bt) return fail(SIDR_ERR_INVALID, "batch is null");
    if (shape < 0 || shape >= SIDR_BATCH_SHAPES) return fail(SIDR_ERR_INVALID, "shape out of range");
    bt->shape = shape;
    return SIDR_OK;
}

sidr_status sidr_batch_autotune_sampled(sidr_batch* bt, int32_t reps, int32_t stride, int32_t* chosen,
                                        float* ms) {
    if (!bt || stride < 1) return fail(SIDR_ERR_INVALID, "null batch or stride < 1");
    DeviceGuard device_guard;
    SIDR_CUDA(cudaSetDevice(bt->ctx->device));
    if ((long long)bt->P * bt->T == 0) {
        if (chosen) *chosen = bt->shape;
        return SIDR_OK;
    }
    // every stride-th rule: the sample keeps the batch's mix of rule costs
    std::vector<int32_t> sample;
    for (int p = 0; p < bt->P; p += stride) sample.push_back(p);
    int32_t* d_order = nullptr;
    SIDR_CUDA(cudaMalloc(&d_order, sample.size() * sizeof(int32_t)));
    cudaStream_t st = bt->ctx->stream;
    cudaError_t e = cudaMemcpyAsync(d_order, sample.data(), sample.size() * sizeof(int32_t),
                                    cudaMemcpyHostToDevice, st);
    DevBatch b = bt->b;
    b.order = d_order;
    b.P_items = (int)sample.size();
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (!e) e = cudaEventCreate(&e0);
    if (!e) e = cudaEventCreate(&e1);
    float best = 1e30f;
    int best_sh = 0;
    sidr_status s = SIDR_OK;
    for (int sh = 0; sh < SIDR_BATCH_SHAPES && !e && !s; sh++) {
        float t_best = 1e30f;
        for (int k = 0; k < (reps < 1 ? 1 : reps) + 1 && !e && !s; k++) {  // the first run warms up
            e = cudaEventRecord(e0, st);
            if (!e) s = launch(bt->ctx, b, false, bt->rmod, bt->grid_s[sh], bt->block_s[sh], bt->smem_s[sh], st, sh);
            if (!e && !s) e = cudaEventRecord(e1, st);
            if (!e && !s) e = cudaEventSynchronize(e1);
            float t = 0.f;
            if (!e && !s) e = cudaEventElapsedTime(&t, e0, e1);
            if (k > 0 && t < t_best) t_best = t;
        }
        if (ms) ms[sh] = t_best;
        if (t_best < best) {
            best = t_best;
            best_sh = sh;
        }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaStreamSynchronize(st);
    cudaFree(d_order);
    if (s) return s;
    if (e) return fail(SIDR_ERR_CUDA, std::string("batch autotune: ") + cudaGetErrorString(e));
    if ((s = read_error_word(b.error, st))) return s;
    bt->shape = best_sh;
    if (chosen) *chosen = best_sh;
    return SIDR_OK;
}

sidr_status sidr_batch_read(sidr_batch* bt, double* out) {
    if (!bt) return fail(SIDR_ERR_INVALID, "batch is null");
    if ((size_t)bt->P * bt->T == 0) return SIDR_OK;
    if (!out) return fail(SIDR_ERR_INVALID, "output buffer is null");
    DeviceGuard device_guard;
    SIDR_CUDA(cudaSetDevice(bt->ctx->device));
    SIDR_CUDA(cudaDeviceSynchronize());
    SIDR_CUDA(cudaMemcpy(out, bt->out.p, (size_t)bt->P * bt->T * sizeof(double), cudaMemcpyDeviceToHost));
    return read_error_word(bt->b.error, 0);
}

sidr_status sidr_batch_fitness(sidr_batch* bt, double* fitness) {
    if (!bt) return fail(SIDR_ERR_INVALID, "batch is null");
    if (bt->P == 0) return SIDR_OK;
    if (!fitness) return fail(SIDR_ERR_INVALID, "fitness buffer is null");
    DeviceGuard device_guard;
    SIDR_CUDA(cudaSetDevice(bt->ctx->device));
    SIDR_CUDA(cudaDeviceSynchronize());
    SIDR_CUDA(cudaMemcpy(fitness, bt->fit.p, (size_t)bt->P * sizeof(double), cudaMemcpyDeviceToHost));
    return read_error_word(bt->b.error, 0);
}

sidr_status sidr_batch_guard_check(sidr_batch* bt) {
    if (!bt) return fail(SIDR_ERR_INVALID, "batch is null");
    if ((long long)bt->P * bt->T == 0) return fail(SIDR_ERR_INVALID, "empty batch");
    DeviceGuard device_guard;
    SIDR_CUDA(cudaSetDevice(bt->ctx->device));
    DevBatch b = bt->b;
    b.prog_cap = 0;  // slices with room for no instruction and the minimum of rows
    b.rows = 0;
    cudaStream_t st = bt->ctx->stream;
    sidr_status s = launch(bt->ctx, b, false, bt->rmod, bt->grid, bt->block, bt->smem, st);
    if (s) return s;
    return read_error_word(b.error, st);
}

const double* sidr_batch_device_out(const sidr_batch* bt) { return bt ? (const double*)bt->out.p : nullptr; }

sidr_status sidr_batch_counts(sidr_batch* bt, sidr_counts* out) {
    if (!bt || !out) return fail(SIDR_ERR_INVALID, "null argument");
    unsigned long long v[kStats] = {};
    DeviceGuard device_guard;
    SIDR_CUDA(cudaSetDevice(bt->ctx->device));
    SIDR_CUDA(cudaDeviceSynchronize());
    SIDR_CUDA(cudaMemcpy(v, bt->stats.p, sizeof v, cudaMemcpyDeviceToHost));
    out->decisions = (int64_t)v[0];
    out->candidates = (int64_t)v[1];
    out->scan_iters = (int64_t)v[2];
    out->heavy_iters = (int64_t)v[3];
    out->hop_iters = (int64_t)v[4];
    out->fp64_ops = (int64_t)v[5];
    return SIDR_OK;
}

void sidr_batch_destroy(sidr_batch* bt) {
    if (!bt) return;
    DeviceGuard device_guard;
    cudaSetDevice(bt->ctx->device);
    cudaDeviceSynchronize();
    for (DevBuf* b : {&bt->prog, &bt->consts, &bt->slots, &bt->meta, &bt->sampled, &bt->out,
                      &bt->counter, &bt->stats, &bt->error, &bt->fit})
        b->release();
    delete bt;
}

}  // extern "C"

#ifdef SIDR_SECTION_CLOCKS
// Profiling builds only: read (and clear) the per-section cycle totals.
extern "C" int sidr_section_cycles_take(unsigned long long* out16) {
    if (cudaMemcpyFromSymbol(out16, sidr::sidr_section_cycles, 16 * sizeof(unsigned long long)) !=
        cudaSuccess)
        return 1;
    static const unsigned long long zero[16] = {};
    return cudaMemcpyToSymbol(sidr::sidr_section_cycles, zero, sizeof zero) == cudaSuccess ? 0 : 1;
}
#endif

// ----------------------------------------------------------------------------
// Evaluation without device allocation (sidr_evaluate_static).
//
// For callers that cannot call cudaMalloc -- their device memory belongs to
// another allocator, or they must not pay cudaMalloc/cudaFree's implicit device
// synchronisation per call.  Everything the evaluator keeps on the device for
// one call lives in this file-scope array, which every GPU that loads the
// library holds until the process exits.  In host code the name
// sidr_static_scratch is only a host-side stand-in, not a device address: the
// address comes from cudaGetSymbolAddress, looked up once per device with that
// device current, and is passed to the kernel inside DevInst/DevBatch.  The
// address is kept for the life of the process, so a cudaDeviceReset between
// calls is not supported.  The copies, the launch and the wait run on a
// non-blocking stream the library creates once per device, so a call does not
// synchronise with work the caller has queued on the legacy default stream.

namespace {

static __device__ __align__(256) unsigned char sidr_static_scratch[SIDR_STATIC_SCRATCH_BYTES];

std::mutex g_static_lock;                 // serialises every use of the array
unsigned char* g_static_ptr[256] = {};    // device address per device index
cudaStream_t g_static_stream[256] = {};   // the library's own non-blocking stream per device

// Byte layout of one call inside the array.
struct StaticLayout {
    size_t off = 0;
    size_t take(size_t bytes) {
        const size_t at = off;
        off = align_up(off + (bytes ? bytes : 1), 256);
        return at;
    }
};

}  // namespace

extern "C" sidr_status sidr_evaluate_static(const sidr_instance_desc* d, const double zp[10],
                                            const sidr_rules_desc* r, const double* sampled,
                                            int32_t G, int32_t T, int32_t group_size,
                                            int32_t mask_group, const int64_t* masks,
                                            int32_t device, double* out) {
    g_h2d = g_d2h = 0;
    if (!d || !zp) return fail(SIDR_ERR_INVALID, "null argument");
    if (d->n > SIDR_STATIC_MAX_N)
        return fail(SIDR_ERR_TOO_LARGE, "sidr_evaluate_static: n = " + std::to_string(d->n) +
                                            " exceeds SIDR_STATIC_MAX_N = " +
                                            std::to_string(SIDR_STATIC_MAX_N));
    sidr_status s = check_rules(r);
    if (s) return s;
    s = check_grouping(r, sampled, G, T, group_size, mask_group, masks);
    if (s) return s;
    if (r->P > 0 && T > 0 && !out) return fail(SIDR_ERR_INVALID, "output buffer is null");
    for (int k = 0; k < 10; k++)
        if (std::isnan(zp[k])) return fail(SIDR_ERR_NONFINITE, "zp holds NaN");
    const int P = r->P;
    if ((long long)P * T == 0) return SIDR_OK;
    HostInstance h;
    std::string e = build_instance(d->n, d->m, d->tmax, d->scores, d->durations, d->open_t,
                                   d->close_t, d->dist, d->dist_to_depot, h, true);
    if (!e.empty())
        return fail(e.find("finite") != std::string::npos ? SIDR_ERR_NONFINITE : SIDR_ERR_INVALID, e);
    const size_t n_smp = (size_t)((P - 1) / group_size + 1) * T * h.n;
    s = check_finite(sampled, n_smp);
    if (s) return s;
    HostPrograms hp;
    s = compile_all(r, masks, mask_group, hp);
    if (s) return s;

    // Place every device-side array of this call in the scratch.
    struct Piece { const void* src; size_t bytes; const void** dst; size_t at; };
    DevInst I{};
    DevBatch b{};
    std::vector<Piece> up = {
        {h.scores.data(), (size_t)h.n * 8, (const void**)&I.scores, 0},
        {h.durations.data(), (size_t)h.n * 8, (const void**)&I.durations, 0},
        {h.open_t.data(), (size_t)h.n * 8, (const void**)&I.open_t, 0},
        {h.close_t.data(), (size_t)h.n * 8, (const void**)&I.close_t, 0},
        {h.d2d.data(), (size_t)h.n * 8, (const void**)&I.d2d, 0},
        {h.dist.data(), h.dist.size() * 8, (const void**)&I.dist, 0},
        {h.F.data(), h.F.size() * 8, (const void**)&I.F, 0},
        {h.G.data(), h.G.size() * 8, (const void**)&I.G, 0},
        {h.R.data(), h.R.size() * 8, (const void**)&I.R, 0},
        {h.P1.data(), h.P1.size() * 8, (const void**)&I.P1, 0},
        {h.P0.data(), h.P0.size() * 8, (const void**)&I.P0, 0},
        {h.zlt.data(), h.zlt.size() * 4, (const void**)&I.zlt, 0},
        {h.zle.data(), h.zle.size() * 4, (const void**)&I.zle, 0},
        {h.FR.data(), h.FR.size() * 8, (const void**)&I.FR, 0},
        {h.GD.data(), h.GD.size() * 8, (const void**)&I.GD, 0},
        {h.DP.data(), h.DP.size() * 8, (const void**)&I.DP, 0},
        {h.CU.data(), h.CU.size() * 8, (const void**)&I.CU, 0},
        {h.TK.data(), h.TK.size() * 8, (const void**)&I.TK, 0},
        {h.TC.data(), h.TC.size(), (const void**)&I.TC, 0},
        {h.ord.data(), h.ord.size() * 2, (const void**)&I.ord, 0},
        {h.sF.data(), h.sF.size() * 8, (const void**)&I.sF, 0},
        {h.sG.data(), h.sG.size() * 8, (const void**)&I.sG, 0},
        {h.bF.data(), h.bF.size() * 8, (const void**)&I.bF, 0},
        {h.bG.data(), h.bG.size() * 8, (const void**)&I.bG, 0},
        {h.cnt_pos.data(), h.cnt_pos.size() * 4, (const void**)&I.cnt_pos, 0},
        {h.cnt_gm1.data(), h.cnt_gm1.size() * 4, (const void**)&I.cnt_gm1, 0},
        {zp, 80, (const void**)&I.zp, 0},
        {hp.prog.data(), hp.prog.size() * 4, (const void**)&b.prog, 0},
        {hp.consts.data(), hp.consts.size() * 8, (const void**)&b.consts, 0},
        {hp.slots.data(), hp.slots.size(), (const void**)&b.slots, 0},
        {hp.meta.data(), hp.meta.size() * sizeof(RuleMeta), (const void**)&b.meta, 0},
        {sampled, n_smp * 8, (const void**)&b.sampled, 0},
    };
    StaticLayout L;
    for (Piece& p : up) p.at = L.take(p.bytes);
    const size_t at_out = L.take((size_t)P * T * 8);
    const size_t at_counter = L.take(sizeof(unsigned long long));
    const size_t at_error = L.take(sizeof(int));
    if (L.off > (size_t)SIDR_STATIC_SCRATCH_BYTES)
        return fail(SIDR_ERR_TOO_LARGE, "sidr_evaluate_static: this call needs " +
                                            std::to_string(L.off) + " bytes of device scratch, "
                                            "more than SIDR_STATIC_SCRATCH_BYTES = " +
                                            std::to_string((size_t)SIDR_STATIC_SCRATCH_BYTES));

    std::lock_guard<std::mutex> guard(g_static_lock);
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
        cudaGetLastError();
        return fail(SIDR_ERR_NO_DEVICE, "no CUDA device");
    }
    if (device < 0 || device >= ndev || device >= 256)
        return fail(SIDR_ERR_INVALID, "device index out of range");
    DeviceGuard device_guard;
    SIDR_CUDA(cudaSetDevice(device));
    if (!g_static_ptr[device]) {  // once per device, with that device current
        void* ptr = nullptr;
        SIDR_CUDA(cudaGetSymbolAddress(&ptr, sidr_static_scratch));
        g_static_ptr[device] = static_cast<unsigned char*>(ptr);
    }
    if (!g_static_stream[device])  // a non-blocking stream: no implicit sync with the legacy stream
        SIDR_CUDA(cudaStreamCreateWithFlags(&g_static_stream[device], cudaStreamNonBlocking));
    unsigned char* base = g_static_ptr[device];
    cudaStream_t st = g_static_stream[device];
    for (const Piece& p : up) {
        *p.dst = base + p.at;
        SIDR_CUDA(cudaMemcpyAsync(base + p.at, p.src, p.bytes, cudaMemcpyHostToDevice, st));
    }
    I.n = h.n;
    I.m = h.m;
    I.ld = h.n + 1;
    I.nw = h.nw;
    I.tmax = h.tmax;
    I.ns = h.ns;
    b.P = P;
    b.T = T;
    b.group_size = group_size;
    b.n = h.n;
    b.out = reinterpret_cast<double*>(base + at_out);
    b.counter = reinterpret_cast<unsigned long long*>(base + at_counter);
    b.stats = nullptr;
    b.error = reinterpret_cast<int*>(base + at_error);
    b.rows = hp.rows;
    b.prog_cap = hp.prog_cap;
    b.const_cap = hp.const_cap;

    // Launch geometry from the device's own attributes (no context here).
    sidr_ctx geo;
    geo.device = device;
    int v = 0;
    SIDR_CUDA(cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device));
    geo.sm_count = v;
    SIDR_CUDA(cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
    geo.smem_optin = (size_t)v;
    geo.inst = I;
    int grid, block;
    size_t smem;
    s = plan_launch(&geo, hp, (long long)P * T, false, grid, block, smem);
    if (s) return s;
    s = launch(&geo, b, false, hp.rmod, grid, block, smem, st);
    if (s) return s;
    SIDR_CUDA(cudaMemcpyAsync(out, base + at_out, (size_t)P * T * 8, cudaMemcpyDeviceToHost, st));
    s = read_error_word(b.error, st);  // waits for the call's work; launch() cleared the word
    if (s) return s;
    g_h2d = 0;
    for (const Piece& p : up) g_h2d += (long long)p.bytes;
    g_d2h = (long long)P * T * 8;
    return SIDR_OK;
}

// ----------------------------------------------------------------------------
// Multi-instance batches (sidr_multi_*).

#include <array>
#include <map>

namespace {

// The compiled block shapes of eval_multi_kernel: {warps per block, min
// blocks per SM, lanes per pair}.
constexpr int kShapes[SIDR_MULTI_SHAPES][3] = {{4, 3, 32}, {8, 2, 32}, {2, 6, 32}, {4, 3, 16}, {4, 3, 8}};
const void* multi_kernel(int shape, bool rmod) {
    switch (shape) {
    case 0: return rmod ? (const void*)eval_multi_kernel<4, 3, true> : (const void*)eval_multi_kernel<4, 3, false>;
    case 1: return rmod ? (const void*)eval_multi_kernel<8, 2, true> : (const void*)eval_multi_kernel<8, 2, false>;
    case 2: return rmod ? (const void*)eval_multi_kernel<2, 6, true> : (const void*)eval_multi_kernel<2, 6, false>;
    case 3:
        return rmod ? (const void*)eval_multi_kernel<4, 3, true, 16> : (const void*)eval_multi_kernel<4, 3, false, 16>;
    default:
        return rmod ? (const void*)eval_multi_kernel<4, 3, true, 8> : (const void*)eval_multi_kernel<4, 3, false, 8>;
    }
}

// Size class of an instance of n customers (each class runs in a launch of
// its own, with its own block shape).
int size_class(int n) { return n <= 32 ? 0 : n <= 64 ? 1 : n <= 128 ? 2 : 3; }

using ClassShapes = std::array<int, SIDR_SIZE_CLASSES>;
std::mutex g_tune_lock;
std::map<std::string, ClassShapes> g_tune_cache;  // batch layout -> chosen block shape per size class

}  // namespace

struct sidr_multi {
    int device = 0, K = 0, P = 0, T = 0, sm_count = 0;
    size_t smem_optin = 0;
    std::vector<void*> owned;
    DevBatch b{};
    ClassShapes shape{};                         // block shape of each size class's launch
    int cls_first[SIDR_SIZE_CLASSES] = {};       // the class's first rule in the work order
    int cls_items[SIDR_SIZE_CLASSES] = {};       // its number of rules
    int block[SIDR_MULTI_SHAPES] = {};
    int full_grid[SIDR_MULTI_SHAPES] = {};       // resident blocks of each shape on all SMs
    size_t smem[SIDR_MULTI_SHAPES] = {};
    std::string key;
    std::vector<int32_t> order;  // the work order (host copy): class by class, longest first in each
    bool rmod = false;           // some rule uses rmod: the RMOD kernels
    cudaStream_t gstream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
};

namespace {

void multi_free(sidr_multi* m) {
    if (!m) return;
    DeviceGuard device_guard;
    cudaSetDevice(m->device);
    cudaDeviceSynchronize();
    if (m->gexec) cudaGraphExecDestroy(m->gexec);
    if (m->graph) cudaGraphDestroy(m->graph);
    if (m->gstream) cudaStreamDestroy(m->gstream);
    for (void* p : m->owned) cudaFree(p);
    delete m;
}

cudaError_t put_dev(sidr_multi* m, const void* src, size_t bytes, const void** dst) {
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, bytes ? bytes : 8);
    if (e != cudaSuccess) return e;
    m->owned.push_back(p);
    *dst = p;
    if (!src || !bytes) return cudaSuccess;  // allocation only
    return cudaMemcpy(p, src, bytes, cudaMemcpyHostToDevice);
}

// One launch of block shape `shape` over n_rules rules of the work order
// (device array `order`), all T scenarios each; the persistent grid is cut to
// the items there are.
sidr_status launch_part(sidr_multi* m, int shape, const int32_t* order, int n_rules, cudaStream_t st) {
    if (n_rules <= 0 || m->T <= 0) return SIDR_OK;
    DevBatch b = m->b;
    b.order = order;
    b.P_items = n_rules;
    const long long per_block = (long long)kShapes[shape][0] * (32 / kShapes[shape][2]);
    const long long items = (long long)n_rules * m->T;
    const int grid = (int)std::max<long long>(
        1, std::min<long long>((items + per_block - 1) / per_block, m->full_grid[shape]));
    SIDR_CUDA(cudaMemsetAsync(m->b.counter, 0, sizeof(unsigned long long), st));
    void* args[] = {&b};
    SIDR_CUDA(cudaLaunchKernel(multi_kernel(shape, m->rmod), dim3(grid), dim3(m->block[shape]), args,
                               m->smem[shape], st));
    g_launches.fetch_add(1);
    return SIDR_OK;
}

// The whole batch: one launch per non-empty size class, each with its shape,
// one after another on st; the error word is cleared once before them.
sidr_status multi_launch(sidr_multi* m, const ClassShapes& shapes, cudaStream_t st) {
    SIDR_CUDA(cudaMemsetAsync(m->b.error, 0, sizeof(int), st));
    for (int c = SIDR_SIZE_CLASSES - 1; c >= 0; c--) {
        const sidr_status s = launch_part(m, shapes[c], m->b.order + m->cls_first[c], m->cls_items[c], st);
        if (s) return s;
    }
    return SIDR_OK;
}

int class_launches(const sidr_multi* m) {
    int k = 0;
    for (int c = 0; c < SIDR_SIZE_CLASSES; c++) k += m->cls_items[c] > 0 && m->T > 0;
    return k;
}

ClassShapes all_classes(int shape) {
    ClassShapes a;
    a.fill(shape);
    return a;
}

}  // namespace

extern "C" {

sidr_status sidr_multi_create(const sidr_instance_desc* insts, const double* zps, int32_t K,
                              const sidr_rules_desc* r, const int32_t* rule_instance,
                              const double* sampled, int64_t n_sampled,
                              const int64_t* sampled_offsets, int32_t T, const int64_t* masks,
                              int32_t device, sidr_multi** out) {
    if (!out) return fail(SIDR_ERR_INVALID, "out is null");
    *out = nullptr;
    if (!insts || !zps || K < 1 || K > 32767 || !rule_instance || !sampled_offsets || !masks)
        return fail(SIDR_ERR_INVALID, "null argument or K out of 1..32767");
    sidr_status s = check_rules(r);
    if (s) return s;
    if (T < 0) return fail(SIDR_ERR_INVALID, "T < 0");
    for (int p = 0; p < r->P; p++)
        if (rule_instance[p] < 0 || rule_instance[p] >= K)
            return fail(SIDR_ERR_INVALID, "rule " + std::to_string(p) + ": instance out of range");
    std::vector<HostInstance> hs(K);
    for (int k = 0; k < K; k++) {
        const sidr_instance_desc& d = insts[k];
        std::string e = build_instance(d.n, d.m, d.tmax, d.scores, d.durations, d.open_t,
                                       d.close_t, d.dist, d.dist_to_depot, hs[k], true);
        if (!e.empty())
            return fail(e.find("finite") != std::string::npos ? SIDR_ERR_NONFINITE
                        : (d.n > kMaxN ? SIDR_ERR_TOO_LARGE : SIDR_ERR_INVALID),
                        "instance " + std::to_string(k) + ": " + e);
        const int64_t need = sampled_offsets[k] + (int64_t)T * d.n;
        if (sampled_offsets[k] < 0 || need > n_sampled)
            return fail(SIDR_ERR_INVALID, "instance " + std::to_string(k) + ": scenario block outside the buffer");
        s = check_finite(sampled + sampled_offsets[k], (size_t)T * d.n);
        if (s) return s;
    }
    HostPrograms hp;
    if (r->P > 0) {
        s = compile_all(r, masks, 1, hp, rule_instance);
        if (s) return s;
    } else {
        hp.prog.push_back(0);
        hp.consts.push_back(0.0);
        hp.slots.push_back(0);
    }
    // Longest-estimated-first order: n^2 x the neighbour work of the rule's
    // families, plus the program.
    std::vector<int32_t> order(r->P);
    std::vector<double> est(r->P);
    for (int p = 0; p < r->P; p++) {
        const RuleMeta& mm = hp.meta[p];
        const double nk = hs[mm.inst].n;
        const double fam = 8.0 + scan_ops_of(mm.need) + ((mm.need & kNeedAtRisk) ? kOpsAtRisk : 0) +
                           8.0 * mm.reach_k;
        est[p] = nk * nk * fam + nk * mm.n_ins;
        order[p] = p;
    }
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return est[a] > est[b]; });
    // then grouped by the size class of the rule's instance, largest class
    // first: each class is one launch of its own block shape
    int cls_first[SIDR_SIZE_CLASSES] = {}, cls_items[SIDR_SIZE_CLASSES] = {};
    {
        std::vector<int32_t> by_class;
        by_class.reserve(order.size());
        for (int c = SIDR_SIZE_CLASSES - 1; c >= 0; c--) {
            cls_first[c] = (int)by_class.size();
            for (int32_t p : order)
                if (size_class(hs[hp.meta[p].inst].n) == c) by_class.push_back(p);
            cls_items[c] = (int)by_class.size() - cls_first[c];
        }
        order.swap(by_class);
    }

    DeviceGuard device_guard;
    SIDR_CUDA(cudaSetDevice(device));
    sidr_multi* m = new sidr_multi();
    m->device = device;
    m->K = K;
    m->rmod = hp.rmod;
    m->P = r->P;
    m->T = T;
    auto bail = [&](cudaError_t err, const char* what) {
        multi_free(m);
        return fail(SIDR_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(err));
    };
    int v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device);
    m->sm_count = v;
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    m->smem_optin = (size_t)v;
    std::vector<DevInst> dinst(K);
    for (int k = 0; k < K; k++) {
        const HostInstance& h = hs[k];
        DevInst& I = dinst[k];
        I.n = h.n;
        I.m = h.m;
        I.ld = h.n + 1;
        I.nw = h.nw;
        I.tmax = h.tmax;
        I.ns = h.ns;
        struct Item { const void* src; size_t bytes; const void** dst; };
        const Item items[] = {
            {h.scores.data(), (size_t)h.n * 8, (const void**)&I.scores},
            {h.durations.data(), (size_t)h.n * 8, (const void**)&I.durations},
            {h.open_t.data(), (size_t)h.n * 8, (const void**)&I.open_t},
            {h.close_t.data(), (size_t)h.n * 8, (const void**)&I.close_t},
            {h.d2d.data(), (size_t)h.n * 8, (const void**)&I.d2d},
            {h.dist.data(), h.dist.size() * 8, (const void**)&I.dist},
            {h.F.data(), h.F.size() * 8, (const void**)&I.F},
            {h.G.data(), h.G.size() * 8, (const void**)&I.G},
            {h.R.data(), h.R.size() * 8, (const void**)&I.R},
            {h.P1.data(), h.P1.size() * 8, (const void**)&I.P1},
            {h.P0.data(), h.P0.size() * 8, (const void**)&I.P0},
            {h.zlt.data(), h.zlt.size() * 4, (const void**)&I.zlt},
            {h.zle.data(), h.zle.size() * 4, (const void**)&I.zle},
            {h.FR.data(), h.FR.size() * 8, (const void**)&I.FR},
            {h.GD.data(), h.GD.size() * 8, (const void**)&I.GD},
            {h.DP.data(), h.DP.size() * 8, (const void**)&I.DP},
            {h.CU.data(), h.CU.size() * 8, (const void**)&I.CU},
            {h.TK.data(), h.TK.size() * 8, (const void**)&I.TK},
        {h.TC.data(), h.TC.size(), (const void**)&I.TC},
            {h.ord.data(), h.ord.size() * 2, (const void**)&I.ord},
            {h.sF.data(), h.sF.size() * 8, (const void**)&I.sF},
            {h.sG.data(), h.sG.size() * 8, (const void**)&I.sG},
            {h.bF.data(), h.bF.size() * 8, (const void**)&I.bF},
            {h.bG.data(), h.bG.size() * 8, (const void**)&I.bG},
            {h.cnt_pos.data(), h.cnt_pos.size() * 4, (const void**)&I.cnt_pos},
            {h.cnt_gm1.data(), h.cnt_gm1.size() * 4, (const void**)&I.cnt_gm1},
            {zps + 10 * (size_t)k, 80, (const void**)&I.zp},
        };
        for (const Item& it : items) {
            cudaError_t e = put_dev(m, it.src, it.bytes, it.dst);
            if (e != cudaSuccess) return bail(e, "instance upload");
        }
    }
    DevBatch& b = m->b;
    const size_t out_n = std::max<size_t>((size_t)r->P * T, 1);
    cudaError_t e;
    if ((e = put_dev(m, dinst.data(), dinst.size() * sizeof(DevInst), (const void**)&b.insts)) ||
        (e = put_dev(m, hp.prog.data(), hp.prog.size() * 4, (const void**)&b.prog)) ||
        (e = put_dev(m, hp.consts.data(), hp.consts.size() * 8, (const void**)&b.consts)) ||
        (e = put_dev(m, hp.slots.data(), hp.slots.size(), (const void**)&b.slots)) ||
        (e = put_dev(m, hp.meta.data(), hp.meta.size() * sizeof(RuleMeta), (const void**)&b.meta)) ||
        (e = put_dev(m, sampled, (size_t)n_sampled * 8, (const void**)&b.sampled)) ||
        (e = put_dev(m, sampled_offsets, (size_t)K * 8, (const void**)&b.smp_off)) ||
        (e = put_dev(m, order.data(), order.size() * 4, (const void**)&b.order)) ||
        (e = put_dev(m, nullptr, out_n * 8, (const void**)&b.out)) ||
        (e = put_dev(m, nullptr, 8, (const void**)&b.counter)) ||
        (e = put_dev(m, nullptr, 8, (const void**)&b.error)) ||
        (e = cudaMemset((void*)b.error, 0, sizeof(int))))
        return bail(e, "batch upload");
    b.n_inst = K;
    m->order = order;
    for (int c = 0; c < SIDR_SIZE_CLASSES; c++) {
        m->cls_first[c] = cls_first[c];
        m->cls_items[c] = cls_items[c];
    }
    b.P = r->P;
    b.T = T;
    b.group_size = r->P > 0 ? r->P : 1;
    b.n = 0;
    b.stats = nullptr;
    b.rows = hp.rows;
    b.prog_cap = hp.prog_cap;
    b.const_cap = hp.const_cap;
    int nmax = 0;
    for (int k = 0; k < K; k++) nmax = std::max(nmax, hs[k].n);
    char kb[256];
    std::snprintf(kb, sizeof kb, "K%d P%d T%d rows%d prog%d sm%d nmax%d rmod%d|", K, r->P, T, hp.rows,
                  hp.prog_cap, m->sm_count, nmax, (int)hp.rmod);
    m->key = kb;
    for (int k = 0; k < K; k++) m->key += std::to_string(hs[k].n) + ",";
    for (int sh = 0; sh < SIDR_MULTI_SHAPES; sh++) {
        const int wpb = kShapes[sh][0], lpp = kShapes[sh][2];
        m->block[sh] = 32 * wpb;
        m->smem[sh] = warp_slice_bytes(hp.rows, hp.const_cap, hp.prog_cap, lpp) * (32 / lpp) * wpb;
        if (m->smem[sh] > m->smem_optin) {
            multi_free(m);
            return fail(SIDR_ERR_TOO_LARGE, "rule programs need more shared memory than one block has");
        }
        if ((e = cudaFuncSetAttribute(multi_kernel(sh, m->rmod), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)m->smem[sh])) != cudaSuccess)
            return bail(e, "cudaFuncSetAttribute");
        int per_sm = 0;
        if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, multi_kernel(sh, m->rmod), m->block[sh],
                                                               m->smem[sh])) != cudaSuccess)
            return bail(e, "occupancy");
        m->full_grid[sh] = m->sm_count * std::max(per_sm, 1);
    }
    {
        std::lock_guard<std::mutex> g(g_tune_lock);
        auto it = g_tune_cache.find(m->key);
        if (it != g_tune_cache.end()) m->shape = it->second;
    }
    *out = m;
    return SIDR_OK;
}

sidr_status sidr_multi_set_shape(sidr_multi* m, int32_t shape) {
    if (!m || shape < 0 || shape >= SIDR_MULTI_SHAPES) return fail(SIDR_ERR_INVALID, "bad shape");
    if (m->gexec) return fail(SIDR_ERR_INVALID, "the batch's launch is already captured");
    m->shape = all_classes(shape);
    return SIDR_OK;
}

sidr_status sidr_multi_set_class_shape(sidr_multi* m, int32_t cls, int32_t shape) {
    if (!m || cls < 0 || cls >= SIDR_SIZE_CLASSES || shape < 0 || shape >= SIDR_MULTI_SHAPES)
        return fail(SIDR_ERR_INVALID, "bad class or shape");
    if (m->gexec) return fail(SIDR_ERR_INVALID, "the batch's launch is already captured");
    m->shape[cls] = shape;
    return SIDR_OK;
}

sidr_status sidr_multi_shapes(sidr_multi* m, int32_t* shapes, int32_t* class_rules) {
    if (!m) return fail(SIDR_ERR_INVALID, "null batch");
    for (int c = 0; c < SIDR_SIZE_CLASSES; c++) {
        if (shapes) shapes[c] = m->shape[c];
        if (class_rules) class_rules[c] = m->cls_items[c];
    }
    return SIDR_OK;
}

}  // extern "C"

namespace {

// Best of reps timed runs (after one warm-up run) of launch(); 0 or an error.
template <class F>
sidr_status time_best(int reps, cudaStream_t st, F launch, float& t_best) {
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t e = cudaEventCreate(&e0);
    if (!e) e = cudaEventCreate(&e1);
    sidr_status s = SIDR_OK;
    t_best = 1e30f;
    for (int k = 0; k < (reps < 1 ? 1 : reps) + 1 && !e && !s; k++) {
        e = cudaEventRecord(e0, st);
        if (!e) s = launch();
        if (!e && !s) e = cudaEventRecord(e1, st);
        if (!e && !s) e = cudaEventSynchronize(e1);
        float t = 0.f;
        if (!e && !s) e = cudaEventElapsedTime(&t, e0, e1);
        if (!e && !s && k > 0 && t < t_best) t_best = t;
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (s) return s;
    if (e) return fail(SIDR_ERR_CUDA, std::string("autotune: ") + cudaGetErrorString(e));
    return SIDR_OK;
}

void remember(sidr_multi* m) {
    std::lock_guard<std::mutex> g(g_tune_lock);
    g_tune_cache[m->key] = m->shape;
}

}  // namespace

extern "C" {

sidr_status sidr_multi_autotune(sidr_multi* m, int32_t reps, int32_t* chosen, float* ms) {
    if (!m) return fail(SIDR_ERR_INVALID, "null batch");
    if (m->gexec) return fail(SIDR_ERR_INVALID, "the batch's launch is already captured");
    DeviceGuard device_guard;
    SIDR_CUDA(cudaSetDevice(m->device));
    if ((long long)m->P * m->T == 0) {
        if (chosen) *chosen = m->shape[0];
        return SIDR_OK;
    }
    float best = 1e30f;
    int best_sh = 0;
    for (int sh = 0; sh < SIDR_MULTI_SHAPES; sh++) {
        float t = 0.f;
        const sidr_status s = time_best(reps, 0, [&] { return multi_launch(m, all_classes(sh), 0); }, t);
        if (s) return s;
        if (ms) ms[sh] = t;
        if (t < best) {
            best = t;
            best_sh = sh;
        }
    }
    sidr_status s = read_error_word(m->b.error, 0);
    if (s) return s;
    m->shape = all_classes(best_sh);
    remember(m);
    if (chosen) *chosen = best_sh;
    return SIDR_OK;
}

sidr_status sidr_multi_autotune_sampled(sidr_multi* m, int32_t reps, int32_t stride, int32_t* chosen,
                                        float* ms) {
    if (!m || stride < 1) return fail(SIDR_ERR_INVALID, "null batch or stride < 1");
    if (m->gexec) return fail(SIDR_ERR_INVALID, "the batch's launch is already captured");
    DeviceGuard device_guard;
    SIDR_CUDA(cudaSetDevice(m->device));
    if ((long long)m->P * m->T == 0) {
        if (chosen) *chosen = m->shape[0];
        return SIDR_OK;
    }
    // every stride-th rule of the work order: the sample keeps the batch's mix
    // of instance sizes and rule costs; each shape runs it in one launch
    std::vector<int32_t> sample;
    for (size_t i = 0; i < m->order.size(); i += (size_t)stride) sample.push_back(m->order[i]);
    int32_t* d_order = nullptr;
    SIDR_CUDA(cudaMalloc(&d_order, sample.size() * sizeof(int32_t)));
    cudaError_t e = cudaMemcpy(d_order, sample.data(), sample.size() * sizeof(int32_t), cudaMemcpyHostToDevice);
    float best = 1e30f;
    int best_sh = 0;
    sidr_status s = e ? fail(SIDR_ERR_CUDA, std::string("sampled autotune: ") + cudaGetErrorString(e)) : SIDR_OK;
    for (int sh = 0; sh < SIDR_MULTI_SHAPES && !s; sh++) {
        float t = 0.f;
        s = time_best(reps, 0, [&] { return launch_part(m, sh, d_order, (int)sample.size(), 0); }, t);
        if (s) break;
        if (ms) ms[sh] = t;
        if (t < best) {
            best = t;
            best_sh = sh;
        }
    }
    cudaFree(d_order);
    if (s) return s;
    if ((s = read_error_word(m->b.error, 0))) return s;
    m->shape = all_classes(best_sh);
    remember(m);
    if (chosen) *chosen = best_sh;
    return SIDR_OK;
}

sidr_status sidr_multi_autotune_classes(sidr_multi* m, int32_t reps, int32_t stride, int32_t* chosen,
                                        float* ms) {
    if (!m || stride < 1) return fail(SIDR_ERR_INVALID, "null batch or stride < 1");
    if (m->gexec) return fail(SIDR_ERR_INVALID, "the batch's launch is already captured");
    DeviceGuard device_guard;
    SIDR_CUDA(cudaSetDevice(m->device));
    // every stride-th rule of each class's part of the work order, in one array
    std::vector<int32_t> sample;
    int first[SIDR_SIZE_CLASSES] = {}, count[SIDR_SIZE_CLASSES] = {};
    for (int c = 0; c < SIDR_SIZE_CLASSES; c++) {
        first[c] = (int)sample.size();
        for (int i = 0; i < m->cls_items[c]; i += stride) sample.push_back(m->order[m->cls_first[c] + i]);
        count[c] = (int)sample.size() - first[c];
    }
    if (ms)
        for (int k = 0; k < SIDR_SIZE_CLASSES * SIDR_MULTI_SHAPES; k++) ms[k] = -1.f;
    if (sample.empty() || m->T == 0) {
        for (int c = 0; c < SIDR_SIZE_CLASSES; c++)
            if (chosen) chosen[c] = m->cls_items[c] ? m->shape[c] : -1;
        return SIDR_OK;
    }
    int32_t* d_order = nullptr;
    SIDR_CUDA(cudaMalloc(&d_order, sample.size() * sizeof(int32_t)));
    cudaError_t e = cudaMemcpy(d_order, sample.data(), sample.size() * sizeof(int32_t), cudaMemcpyHostToDevice);
    sidr_status s = e ? fail(SIDR_ERR_CUDA, std::string("class autotune: ") + cudaGetErrorString(e)) : SIDR_OK;
    ClassShapes pick = m->shape;
    for (int c = 0; c < SIDR_SIZE_CLASSES && !s; c++) {
        if (!count[c]) continue;
        float best = 1e30f;
        for (int sh = 0; sh < SIDR_MULTI_SHAPES && !s; sh++) {
            float t = 0.f;
            s = time_best(reps, 0, [&] { return launch_part(m, sh, d_order + first[c], count[c], 0); }, t);
            if (s) break;
            if (ms) ms[c * SIDR_MULTI_SHAPES + sh] = t;
            if (t < best) {
                best = t;
                pick[c] = sh;
            }
        }
    }
    cudaFree(d_order);
    if (s) return s;
    if ((s = read_error_word(m->b.error, 0))) return s;
    m->shape = pick;
    remember(m);
    for (int c = 0; c < SIDR_SIZE_CLASSES; c++)
        if (chosen) chosen[c] = m->cls_items[c] ? m->shape[c] : -1;
    return SIDR_OK;
}

sidr_status sidr_multi_capture(sidr_multi* m) {
    if (!m) return fail(SIDR_ERR_INVALID, "null batch");
    if (m->gexec) return SIDR_OK;
    DeviceGuard device_guard;
    SIDR_CUDA(cudaSetDevice(m->device));
    if (!m->gstream) SIDR_CUDA(cudaStreamCreateWithFlags(&m->gstream, cudaStreamNonBlocking));
    SIDR_CUDA(cudaStreamBeginCapture(m->gstream, cudaStreamCaptureModeThreadLocal));
    sidr_status s = SIDR_OK;
    if ((long long)m->P * m->T > 0) s = multi_launch(m, m->shape, m->gstream);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(m->gstream, &g);
    if (s) {
        if (g) cudaGraphDestroy(g);
        return s;
    }
    if (e != cudaSuccess) return fail(SIDR_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(e));
    m->graph = g;
    SIDR_CUDA(cudaGraphInstantiate(&m->gexec, m->graph, 0));
    return SIDR_OK;
}

sidr_status sidr_multi_run(sidr_multi* m, void* stream) {
    NvtxRange range("sidr_multi_run");
    if (!m) return fail(SIDR_ERR_INVALID, "null batch");
    DeviceGuard device_guard;
    SIDR_CUDA(cudaSetDevice(m->device));
    cudaStream_t st = (cudaStream_t)stream;
    if (m->gexec) {
        SIDR_CUDA(cudaGraphLaunch(m->gexec, st));
        g_launches.fetch_add(class_launches(m));
        return SIDR_OK;
    }
    if ((long long)m->P * m->T == 0) return SIDR_OK;
    return multi_launch(m, m->shape, st);
}

sidr_status sidr_multi_read(sidr_multi* m, double* out) {
    if (!m) return fail(SIDR_ERR_INVALID, "null batch");
    if ((long long)m->P * m->T == 0) return SIDR_OK;
    if (!out) return fail(SIDR_ERR_INVALID, "output buffer is null");
    DeviceGuard device_guard;
    SIDR_CUDA(cudaSetDevice(m->device));
    SIDR_CUDA(cudaDeviceSynchronize());
    SIDR_CUDA(cudaMemcpy(out, m->b.out, (size_t)m->P * m->T * 8, cudaMemcpyDeviceToHost));
    return read_error_word(m->b.error, 0);
}

void sidr_multi_destroy(sidr_multi* m) { multi_free(m); }

}  // extern "C"
