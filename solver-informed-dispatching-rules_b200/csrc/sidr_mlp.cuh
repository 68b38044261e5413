// sidr_mlp.cuh -- the surrogate's tensor-core GEMM for sm_100a.
//
// C[M x N] = A[M x K] * B[N x K]^T with BF16 operands stored K-major (K
// contiguous; row strides lda / ldb elements, multiples of 8 so that every row
// starts on 16 bytes) and FP32 accumulation in tensor memory (TMEM).  One CTA of
// four warps computes a 128 x 64 tile:
//   * warp 0, one lane: the producer.  K is walked in chunks of 64 elements (128
//     bytes: one 128-byte swizzle span); each chunk's A (128 x 64) and B (64 x
//     64) tiles are fetched by TMA (cp.async.bulk.tensor, no multicast) into a
//     ring of kStages shared-memory stages, each stage guarded by a "full"
//     mbarrier (TMA transaction bytes) and an "empty" one (MMA completion);
//     rows and K beyond the tensor's extent arrive as zeros;
//   * warp 1, one lane: the MMA issuer.  Per chunk, four tcgen05.mma (kind::f16,
//     M = 128, N = 64, K = 16) read the stage through 128-byte-swizzle K-major
//     matrix descriptors; tcgen05.commit releases the stage when they finish,
//     and a last commit signals the accumulator;
//   * all four warps: the epilogue reads the accumulator with tcgen05.ld (warp w
//     owns TMEM lanes 32w .. 32w+31) and applies one of: plain store, bias +
//     ReLU with a BF16 copy, or a store into the partial-sum slice of its K
//     range (split-K over blockIdx.z; split_sum_kernel adds the slices in slice
//     order, so the result does not depend on the order CTAs finish in).
// Every mbarrier wait is bounded: a wait that runs out sets the error flag, the
// producer then waits (bounded) for the copies it has in flight, the TMEM is
// freed and the kernel returns.  The tensor maps cover this GPU's memory only.
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace sidr {
namespace mlp {

enum Epilogue : int {
    kStoreF32 = 0,    // C[m*ldc + n] = acc
    kBiasRelu = 1,    // z = acc + bias[n]; Hb[m*ldh + n] = bf16(max(z, 0))
    kSplitF32 = 2,    // C[z*split_stride + m*ldc + n] = acc, z = blockIdx.z
};

struct GemmArgs {
    const __nv_bfloat16* A;
    long long lda;       // A(m, k) = A[m*lda + k]
    const __nv_bfloat16* B;
    long long ldb;       // B(n, k) = B[n*ldb + k]
    int M, N, K;
    int k_split;         // K range of one blockIdx.z (multiple of kChunkK)
    int epilogue;
    float* C;
    int ldc;
    long long split_stride;  // floats between the partial-sum slices (kSplitF32)
    const float* bias;
    __nv_bfloat16* Hb;
    int ldh;
    int* error;          // set to 1 when an mbarrier wait runs out
    uint32_t wait_limit; // polls of an mbarrier before a wait gives up (0: kWaitLimit)
    int withhold;        // failure-detection check: issue no MMA and no commit, so
                         // the waits for them run out (no copy is left in flight)
};

constexpr int kTileM = 128;
constexpr int kTileN = 64;
constexpr int kChunkK = 64;           // one 128-byte swizzle span of BF16
constexpr int kStages = 4;
constexpr uint32_t kTileABytes = kTileM * kChunkK * 2;  // 16 KB
constexpr uint32_t kTileBBytes = kTileN * kChunkK * 2;  // 8 KB
constexpr size_t kGemmSmem = (size_t)kStages * (kTileABytes + kTileBBytes) + 1024;  // + alignment slack
constexpr uint32_t kWaitLimit = 1u << 26;
constexpr uint32_t kTmemCols = 64;

// The kind::f16 instruction descriptor: F32 accumulator (bits 4-5 = 1), BF16
// A and B (bits 7-9, 10-12 = 1), both K-major (bits 15, 16 = 0), N >> 3 at bit
// 17, M >> 4 at bit 24.
__host__ __device__ constexpr uint32_t instr_desc_bf16(int m, int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) |
           ((uint32_t)(m >> 4) << 24);
}

// Shared-memory matrix descriptor of a K-major tile written by TMA with the
// 128-byte swizzle: start address >> 4 (bits 0-13), leading byte offset 16
// bytes (unused by a swizzled K-major operand; bits 16-29), stride byte offset
// 1024 (eight 128-byte rows between 8-row groups; bits 32-45), version 1 (bit
// 46), layout type 2 = 128-byte swizzle (bits 61-63).  The tile base is
// 1024-byte aligned; the MMA's K = 16 step is a 32-byte advance of the start.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t addr) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3fffu);
    d |= (uint64_t)(16u >> 4) << 16;
    d |= (uint64_t)(1024u >> 4) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)2 << 61;
    return d;
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// Polls the mbarrier until the phase of the given parity has completed, at
// most `limit` times; false when the wait ran out.
__device__ __forceinline__ bool wait_phase(uint32_t bar, uint32_t parity, uint32_t limit) {
    for (uint32_t spins = 0;; spins++) {
        uint32_t done = 0;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
        if (spins >= limit) return false;
    }
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

__global__ void __launch_bounds__(128) umma_gemm_kernel(const __grid_constant__ CUtensorMap map_a,
                                                        const __grid_constant__ CUtensorMap map_b,
                                                        GemmArgs g) {
    extern __shared__ unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t full_bar[kStages], empty_bar[kStages], accum_bar;
    __shared__ uint32_t tmem_base;
    __shared__ volatile int failed;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * kTileM, n0 = blockIdx.y * kTileN;
    const int k_begin = blockIdx.z * g.k_split;
    const int k_end = min(g.K, k_begin + g.k_split);
    const int chunks = k_end > k_begin ? (k_end - k_begin + kChunkK - 1) / kChunkK : 0;
    const uint32_t base = (smem_addr(smem_raw) + 1023u) & ~1023u;
    const uint32_t limit = g.wait_limit ? g.wait_limit : kWaitLimit;
    auto stage_a = [&](int s) { return base + (uint32_t)s * kTileABytes; };
    auto stage_b = [&](int s) { return base + (uint32_t)kStages * kTileABytes + (uint32_t)s * kTileBBytes; };

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_base)),
                     "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 32) {
        for (int s = 0; s < kStages; s++) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&full_bar[s])));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&empty_bar[s])));
        }
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&accum_bar)));
        asm volatile("fence.mbarrier_init.release.cluster;");
        failed = 0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmem_base;

    int issued = 0;  // producer: chunks whose copies were started
    if (warp == 0 && lane == 0) {
        for (int it = 0; it < chunks; it++) {
            const int s = it % kStages;
            if (it >= kStages && !wait_phase(smem_addr(&empty_bar[s]), ((it / kStages) - 1) & 1, limit)) {
                failed = 1;
                break;
            }
            if (failed) break;
            const uint32_t fb = smem_addr(&full_bar[s]);
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(fb),
                         "r"(kTileABytes + kTileBBytes)
                         : "memory");
            const int k0 = k_begin + it * kChunkK;  // a multiple of 64 elements: 128-byte aligned
            tma_load_2d(stage_a(s), &map_a, k0, m0, fb);
            tma_load_2d(stage_b(s), &map_b, k0, n0, fb);
            issued = it + 1;
        }
    } else if (warp == 1 && lane == 0) {
        constexpr uint32_t idesc = instr_desc_bf16(kTileM, kTileN);
        for (int it = 0; it < chunks; it++) {
            const int s = it % kStages;
            if (!wait_phase(smem_addr(&full_bar[s]), (it / kStages) & 1, limit)) {
                failed = 1;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;");
            if (g.withhold) continue;
#pragma unroll
            for (int ks = 0; ks < kChunkK / 16; ks++) {
                const uint64_t da = sw128_desc(stage_a(s) + 32u * ks);
                const uint64_t db = sw128_desc(stage_b(s) + 32u * ks);
                const uint32_t accumulate = (it > 0 || ks > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
                    "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_addr(&empty_bar[s]))
                         : "memory");
        }
        if (!g.withhold && !failed && chunks > 0)
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_addr(&accum_bar))
                         : "memory");
    }
    __syncwarp();

    // the accumulator is complete when the last commit arrives
    bool have = chunks > 0;
    if (have && !wait_phase(smem_addr(&accum_bar), 0, limit)) {
        failed = 1;
        have = false;
    }
    asm volatile("tcgen05.fence::after_thread_sync;");
    __syncthreads();
    if (have && !failed) {
        const int m = m0 + warp * 32 + lane;
        for (int c0 = 0; c0 < kTileN; c0 += 16) {
            uint32_t v[16];
            const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
                "%11, %12, %13, %14, %15}, [%16];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                  "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]),
                  "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
                : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (m < g.M) {
#pragma unroll
                for (int j = 0; j < 16; j++) {
                    const int n = n0 + c0 + j;
                    if (n >= g.N) continue;
                    const float acc = __uint_as_float(v[j]);
                    if (g.epilogue == kStoreF32) {
                        g.C[(long long)m * g.ldc + n] = acc;
                    } else if (g.epilogue == kSplitF32) {
                        g.C[(long long)blockIdx.z * g.split_stride + (long long)m * g.ldc + n] = acc;
                    } else {
                        const float z = acc + g.bias[n];
                        g.Hb[(long long)m * g.ldh + n] = __float2bfloat16(z > 0.0f ? z : 0.0f);
                    }
                }
            }
        }
    }
    if (failed && warp == 0 && lane == 0) {
        // a wait ran out: let the copies this CTA started land before its shared memory goes
        for (int it = issued > kStages ? issued - kStages : 0; it < issued; it++)
            wait_phase(smem_addr(&full_bar[it % kStages]), (it / kStages) & 1, limit);
        atomicExch(g.error, 1);
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
    }
}

// dst[c*ldd + r] = src[r*lds + c] for r < rows, c < cols: an operand stored
// with M (or N) contiguous turned K-major for the GEMM's tensor maps.
__global__ void transpose_bf16_kernel(const __nv_bfloat16* src, int rows, int cols, long long lds,
                                      __nv_bfloat16* dst, long long ldd) {
    __shared__ __nv_bfloat16 tile[32][33];
    const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int r = r0 + i, c = c0 + threadIdx.x;
        if (r < rows && c < cols) tile[i][threadIdx.x] = src[(long long)r * lds + c];
    }
    __syncthreads();
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int c = c0 + i, r = r0 + threadIdx.x;
        if (r < rows && c < cols) dst[(long long)c * ldd + r] = tile[threadIdx.x][i];
    }
}

// out[i] = parts[i] + parts[count + i] + ... over `splits` slices, added in
// slice order.
__global__ void split_sum_kernel(const float* parts, int splits, long long count, float* out) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
         i += (long long)gridDim.x * blockDim.x) {
        float acc = parts[i];
        for (int z = 1; z < splits; z++) acc += parts[(long long)z * count + i];
        out[i] = acc;
    }
}

}  // namespace mlp
}  // namespace sidr
