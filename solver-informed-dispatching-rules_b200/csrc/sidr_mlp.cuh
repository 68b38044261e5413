// sidr_mlp.cuh -- the surrogate's tensor-core GEMM for sm_100a.
//
// C[M x N] = A[M x K] * B[N x K]^T with BF16 operands and FP32 accumulation in
// tensor memory (TMEM), issued with tcgen05.mma (kind::f16, one CTA, M = 128).
// Operands are read from global memory with arbitrary element strides (so a
// transposed operand needs no copy), staged by the CTA's 128 threads into
// shared memory in the no-swizzle K-major core-matrix layout the matrix
// descriptors describe (8 rows x 16 bytes per core matrix), one K chunk of 32
// at a time; one elected thread issues the MMAs and commits them to an
// mbarrier that the CTA waits on (bounded).  The epilogue reads the
// accumulator back with tcgen05.ld (32 lanes x 32 bits per warp) and applies
// one of: plain store, bias + ReLU with a BF16 copy, or a store into the
// partial-sum slice of its K range (split-K over blockIdx.z for the weight
// gradients; the slices are then added in slice order by split_sum_kernel, so
// the result does not depend on the order in which CTAs finish).
#pragma once
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
    long long sam, sak;  // A(m, k) = A[m*sam + k*sak]
    const __nv_bfloat16* B;
    long long sbn, sbk;  // B(n, k) = B[n*sbn + k*sbk]
    int M, N, K;
    int k_split;         // K range of one blockIdx.z (multiple of 32)
    int epilogue;
    float* C;
    int ldc;
    long long split_stride;  // floats between the partial-sum slices (kSplitF32)
    const float* bias;
    __nv_bfloat16* Hb;
    int ldh;
    int* error;          // set to 1 when an MMA wait runs out
    uint32_t wait_limit; // polls of the mbarrier before a wait gives up (0: kWaitLimit)
    int withhold;        // failure-detection check: issue no MMA and no commit, so
                         // every wait runs out (nothing is left in flight)
};

constexpr int kTileM = 128;
constexpr int kChunkK = 32;           // two MMAs of K = 16
constexpr uint32_t kWaitLimit = 1u << 26;

// The kind::f16 instruction descriptor: F32 accumulator, BF16 A and B, both
// K-major, N >> 3 at bit 17, M >> 4 at bit 24.
__host__ __device__ constexpr uint32_t instr_desc_bf16(int m, int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) |
           ((uint32_t)(m >> 4) << 24);
}

// Shared-memory matrix descriptor, no swizzle: start address, leading byte
// offset (between the two 8-element K halves of one MMA), stride byte offset
// (between 8-row groups), all in 16-byte units; version 1 at bit 46.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3fffu);
    d |= (uint64_t)((lbo >> 4) & 0x3fffu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3fffu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// Byte offset of element (row, k) of a [rows x kChunkK] tile in the core-matrix
// layout: 8-row groups every 512 bytes (SBO), 8-element K blocks every 128
// bytes (LBO), 16 bytes per row inside a core matrix.
__device__ __forceinline__ uint32_t tile_offset(int row, int k) {
    return (uint32_t)((row >> 3) * 512 + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}
constexpr uint32_t kLbo = 128, kSbo = 512;

template <int BN>
__global__ void __launch_bounds__(128) umma_gemm_kernel(GemmArgs g) {
    static_assert(BN % 16 == 0 && BN >= 16 && BN <= 256, "N tile");
    constexpr int kCols = BN <= 32 ? 32 : BN <= 64 ? 64 : BN <= 128 ? 128 : 256;  // TMEM columns
    __shared__ __align__(1024) unsigned char sA[kTileM * kChunkK * 2];
    __shared__ __align__(1024) unsigned char sB[BN * kChunkK * 2];
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_base;
    __shared__ int failed;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * kTileM, n0 = blockIdx.y * BN;
    const int k_begin = blockIdx.z * g.k_split;
    const int k_end = min(g.K, k_begin + g.k_split);

    if (warp == 0) {
        const uint32_t dst = (uint32_t)__cvta_generic_to_shared(&tmem_base);
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst),
                     "r"((uint32_t)kCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        failed = 0;
        const uint32_t bar = (uint32_t)__cvta_generic_to_shared(&mbar);
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmem_base;
    const uint32_t bar = (uint32_t)__cvta_generic_to_shared(&mbar);
    const uint32_t a_base = (uint32_t)__cvta_generic_to_shared(sA);
    const uint32_t b_base = (uint32_t)__cvta_generic_to_shared(sB);
    constexpr uint32_t idesc = instr_desc_bf16(kTileM, BN);

    uint32_t phase = 0;
    bool first = true;
    for (int k0 = k_begin; k0 < k_end; k0 += kChunkK) {
        // stage A (128 x 32) and B (BN x 32); out-of-range elements are zero
        for (int e = tid; e < kTileM * kChunkK; e += 128) {
            const int r = e / kChunkK, k = e % kChunkK;
            const int m = m0 + r, kk = k0 + k;
            __nv_bfloat16 v = __float2bfloat16(0.0f);
            if (m < g.M && kk < k_end) v = g.A[(long long)m * g.sam + (long long)kk * g.sak];
            *reinterpret_cast<__nv_bfloat16*>(sA + tile_offset(r, k)) = v;
        }
        for (int e = tid; e < BN * kChunkK; e += 128) {
            const int r = e / kChunkK, k = e % kChunkK;
            const int n = n0 + r, kk = k0 + k;
            __nv_bfloat16 v = __float2bfloat16(0.0f);
            if (n < g.N && kk < k_end) v = g.B[(long long)n * g.sbn + (long long)kk * g.sbk];
            *reinterpret_cast<__nv_bfloat16*>(sB + tile_offset(r, k)) = v;
        }
        // generic-proxy shared-memory writes become visible to the MMA's async proxy
        asm volatile("fence.proxy.async.shared::cta;");
        __syncthreads();
        if (tid == 0 && !g.withhold) {
            asm volatile("tcgen05.fence::after_thread_sync;");
#pragma unroll
            for (int ks = 0; ks < kChunkK / 16; ks++) {
                const uint64_t da = smem_desc(a_base + ks * 2 * kLbo, kLbo, kSbo);
                const uint64_t db = smem_desc(b_base + ks * 2 * kLbo, kLbo, kSbo);
                const uint32_t accumulate = (first && ks == 0) ? 0u : 1u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
                    "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                         : "memory");
        }
        // every thread waits for the MMAs (they read the staged tiles)
        const uint32_t limit = g.wait_limit ? g.wait_limit : kWaitLimit;
        uint32_t done = 0, spins = 0;
        while (!done) {
            asm volatile(
                "{\n\t.reg .pred p;\n\t"
                "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                "selp.u32 %0, 1, 0, p;\n\t}\n"
                : "=r"(done)
                : "r"(bar), "r"(phase));
            if (!done && ++spins > limit) {
                failed = 1;
                break;
            }
        }
        phase ^= 1u;
        first = false;
        asm volatile("tcgen05.fence::after_thread_sync;");
        __syncthreads();
        if (failed) break;
    }

    if (!failed && !first) {
        // epilogue: warp w owns TMEM lanes (rows) 32w .. 32w+31
        const int m = m0 + warp * 32 + lane;
        for (int c0 = 0; c0 < BN; c0 += 16) {
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
    if (failed && tid == 0) atomicExch(g.error, 1);
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"((uint32_t)kCols));
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
