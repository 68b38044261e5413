// sidr_surrogate.cu -- the surrogate fitness model of the surrogate-assisted
// GP (include/sidr_surrogate.h): a 40 -> 256 -> 256 -> 1 ReLU MLP with BF16
// weights and activations and FP32 accumulation, trained on the device with
// Adam.  Its five GEMMs per training step (two forward, the backward pass's
// input gradient and two weight gradients) run on the TMA-fed tcgen05 kernel
// of sidr_mlp.cuh, the backward ones on K-major copies made by a transpose
// kernel; the 256 -> 1 layer, the ReLU masks, the bias gradients, the
// loss and Adam are small element-wise kernels.  Also here: the phenotype
// kernel (each rule's priority ranking on fixed decision situations) and the
// diagnostic GEMM entry point.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <random>
#include <string>
#include <vector>

#include "../../include/sidr_surrogate.h"
#include "sidr_device.hpp"
#include "sidr_host.hpp"
#include "sidr_libm.cuh"
#include "sidr_mlp.cuh"

using namespace sidr;
using namespace sidr::mlp;

namespace {

constexpr int kIn = SIDR_MLP_INPUTS;   // 40
constexpr int kInPad = 48;             // K of the first layer (multiple of 16)
constexpr int kHid = SIDR_MLP_HIDDEN;  // 256

sidr_status fail_s(sidr_status s, const std::string& m) {
    set_last_error(m);
    return s;
}

#define SIDR_SCHECK(call)                                                                      \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                 \
            return fail_s(SIDR_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// ----------------------------------------------------------------- kernels

__global__ void to_bf16_kernel(const float* x, __nv_bfloat16* y, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        y[i] = __float2bfloat16(x[i]);
}

// rows x kIn floats -> rows x kInPad bf16 (zero padding)
__global__ void pad_inputs_kernel(const float* x, __nv_bfloat16* xb, int rows) {
    const long long n = (long long)rows * kInPad;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(i / kInPad), c = (int)(i % kInPad);
        xb[i] = __float2bfloat16(c < kIn ? x[(long long)r * kIn + c] : 0.0f);
    }
}

// y[b] = sum_n H2[b][n] * w3[n] + b3 (n ascending, FP32)
__global__ void head_forward_kernel(const __nv_bfloat16* h2, const float* w3, const float* b3, float* y,
                                    int rows) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= rows) return;
    float acc = 0.0f;
    for (int n = 0; n < kHid; n++) acc += __bfloat162float(h2[(long long)b * kHid + n]) * w3[n];
    y[b] = acc + b3[0];
}

// loss = mean (y - t)^2 ; dy = 2 (y - t) / rows
__global__ void loss_kernel(const float* y, const float* t, float* dy, float* loss, int rows) {
    __shared__ float part[256];
    float acc = 0.0f;
    for (int b = threadIdx.x; b < rows; b += blockDim.x) {
        const float d = y[b] - t[b];
        dy[b] = 2.0f * d / rows;
        acc += d * d;
    }
    part[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) part[threadIdx.x] += part[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) loss[0] = part[0] / rows;
}

// dw3[n] = sum_b H2[b][n] dy[b]; db3 = sum_b dy[b]  (one thread per n; thread kHid does db3)
__global__ void head_backward_kernel(const __nv_bfloat16* h2, const float* dy, float* dw3, float* db3,
                                     int rows) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n > kHid) return;
    float acc = 0.0f;
    if (n == kHid) {
        for (int b = 0; b < rows; b++) acc += dy[b];
        db3[0] = acc;
        return;
    }
    for (int b = 0; b < rows; b++) acc += __bfloat162float(h2[(long long)b * kHid + n]) * dy[b];
    dw3[n] = acc;
}

// dZ2[b][n] = dy[b] * w3[n] where H2 > 0 (else 0), stored BF16
__global__ void head_delta_kernel(const __nv_bfloat16* h2, const float* dy, const float* w3,
                                  float* dz, __nv_bfloat16* dzb, int rows) {
    const long long n_all = (long long)rows * kHid;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n_all;
         i += (long long)gridDim.x * blockDim.x) {
        const int b = (int)(i / kHid), n = (int)(i % kHid);
        const float v = __bfloat162float(h2[i]) > 0.0f ? dy[b] * w3[n] : 0.0f;
        dz[i] = v;
        dzb[i] = __float2bfloat16(v);
    }
}

// dZ1 = dH1 where H1 > 0 (else 0), FP32 and BF16
__global__ void relu_back_kernel(const float* dh, const __nv_bfloat16* h, float* dz, __nv_bfloat16* dzb,
                                 long long n_all) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n_all;
         i += (long long)gridDim.x * blockDim.x) {
        const float v = __bfloat162float(h[i]) > 0.0f ? dh[i] : 0.0f;
        dz[i] = v;
        dzb[i] = __float2bfloat16(v);
    }
}

// db[n] = sum_b dz[b][n] (b ascending)
__global__ void col_sum_kernel(const float* dz, float* db, int rows, int cols) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= cols) return;
    float acc = 0.0f;
    for (int b = 0; b < rows; b++) acc += dz[(long long)b * cols + n];
    db[n] = acc;
}

__global__ void adam_kernel(float* p, const float* g, float* m, float* v, long long n, float lr, float b1,
                            float b2, float eps, float c1, float c2) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

__global__ void gather_rows_kernel(const float* src, const float* tsrc, const int* idx, float* dst,
                                   float* tdst, int rows, int cols) {
    const long long n = (long long)rows * cols;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(i / cols), c = (int)(i % cols);
        dst[i] = src[(long long)idx[r] * cols + c];
        if (c == 0) tdst[r] = tsrc[idx[r]];
    }
}

// eval_tree (engine/sim_core.hpp:11-41) over one 61-slot terminal table.
__device__ double eval_rule(const int32_t* ops, const int32_t* args, int len, const double* t) {
    double st[32];
    int sp = 0;
    for (int k = 0; k < len; k++) {
        const int o = ops[k];
        if (o == -1) {
            st[sp++] = t[args[2 * k]];
        } else if (o == -2) {
            st[sp++] = args[2 * k] / 1000.0;
        } else {
            const double b = st[sp - 1], a = st[sp - 2];
            sp -= 2;
            double r;
            if (o == 0) r = a + b;
            else if (o == 1) r = a - b;
            else if (o == 2) r = a * b;
            else if (o == 3) r = fabs(b) < 1e-10 ? 1.0 : a / b;
            else if (o == 4) r = a < b ? a : b;
            else if (o == 5) r = a > b ? a : b;
            else {
                const double base = a > 0.0 ? a : 0.0;
                const double e = b < 0.0 ? 0.0 : (b > 1.0 ? 1.0 : b);
                r = libm::pow_(base, 1.0 + e);
            }
            st[sp++] = r;
        }
    }
    const double v = st[0];
    return v != v ? -1e300 : v;
}

// One thread per (rule, situation): the position of the situation's
// reference choice in the rule's ranking of the candidates (strict >, lower
// position first on ties), scaled to [0, 1].
__global__ void phenotype_kernel(const int32_t* ops, const int32_t* args, const int32_t* off,
                                 const int32_t* len, int P, const double* terms, const int32_t* ncand,
                                 const int32_t* ref, int n_sit, int max_cand, float* feat, int n_feat) {
    const long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (id >= (long long)P * n_sit) return;
    const int p = (int)(id / n_sit), j = (int)(id % n_sit);
    const int nc = ncand[j], r = ref[j];
    const int32_t* o = ops + off[p];
    const int32_t* a = args + 2 * (size_t)off[p];
    const double* base = terms + (size_t)j * max_cand * 61;
    const double pr = eval_rule(o, a, len[p], base + (size_t)r * 61);
    int pos = 0;
    for (int c = 0; c < nc; c++) {
        if (c == r) continue;
        const double pc = eval_rule(o, a, len[p], base + (size_t)c * 61);
        if (pc > pr || (pc == pr && c < r)) pos++;
    }
    feat[(size_t)p * n_feat + j] = nc > 1 ? (float)pos / (float)(nc - 1) : 0.0f;
}

int grid_for(long long n, int threads = 256) {
    return (int)std::max<long long>(1, std::min<long long>((n + threads - 1) / threads, 148 * 8));
}

// ------------------------------------------------------------- GEMM launch

// cuTensorMapEncodeTiled, reached through the runtime's driver entry point
// (the library links no driver library).
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled() {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiledFn)p;
        else
            cudaGetLastError();
    });
    return fn;
}

// The tensor map of a K-major BF16 operand [rows][K] with row stride ld
// elements: boxes of kChunkK x box_rows with the 128-byte swizzle, zeros
// outside the extent.
sidr_status operand_map(CUtensorMap* map, const __nv_bfloat16* p, int rows, int K, long long ld, int box_rows) {
    if (((uintptr_t)p & 15u) != 0 || (ld * 2) % 16 != 0)
        return fail_s(SIDR_ERR_INVALID, "GEMM operand: base or row stride not a multiple of 16 bytes");
    EncodeTiledFn enc = encode_tiled();
    if (!enc) return fail_s(SIDR_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
    const cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
    const cuuint32_t box[2] = {(cuuint32_t)kChunkK, (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<__nv_bfloat16*>(p), dims, strides,
                           box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail_s(SIDR_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
    return SIDR_OK;
}

bool smem_attr_set[256] = {};  // per device: the kernel's dynamic shared-memory limit raised
std::mutex smem_attr_lock;

// Launches C = A B^T (both K-major).  With splits > 1 the K range is cut into
// slices of a multiple of kChunkK; epilogue kSplitF32 then writes slice z at
// C + z*split_stride and *slices receives the number of slices launched.
sidr_status launch_gemm(const GemmArgs& g0, int splits, cudaStream_t st, int* slices = nullptr) {
    GemmArgs g = g0;
    if (slices) *slices = 0;
    if (g.M <= 0 || g.N <= 0 || g.K <= 0) return SIDR_OK;
    if (splits < 1) splits = 1;
    int ks = (g.K + splits - 1) / splits;
    ks = (ks + kChunkK - 1) / kChunkK * kChunkK;
    g.k_split = ks;
    const int gz = (g.K + ks - 1) / ks;  // every slice holds at least one chunk
    if (slices) *slices = gz;
    CUtensorMap ma, mb;
    sidr_status s = operand_map(&ma, g.A, g.M, g.K, g.lda, kTileM);
    if (s) return s;
    if ((s = operand_map(&mb, g.B, g.N, g.K, g.ldb, kTileN))) return s;
    {
        int dev = 0;
        SIDR_SCHECK(cudaGetDevice(&dev));
        std::lock_guard<std::mutex> lk(smem_attr_lock);
        if (dev < 0 || dev >= 256) return fail_s(SIDR_ERR_INVALID, "device index out of range");
        if (!smem_attr_set[dev]) {
            SIDR_SCHECK(cudaFuncSetAttribute(umma_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)kGemmSmem));
            smem_attr_set[dev] = true;
        }
    }
    dim3 grid((g.M + kTileM - 1) / kTileM, (g.N + kTileN - 1) / kTileN, gz);
    umma_gemm_kernel<<<grid, 128, kGemmSmem, st>>>(ma, mb, g);
    SIDR_SCHECK(cudaGetLastError());
    return SIDR_OK;
}

// dst [cols][ldd] = src [rows][lds] transposed (an M- or N-contiguous operand
// turned K-major); ldd is a multiple of 8 elements.
sidr_status transpose(const __nv_bfloat16* src, int rows, int cols, long long lds, __nv_bfloat16* dst,
                      long long ldd, cudaStream_t st) {
    dim3 grid((cols + 31) / 32, (rows + 31) / 32);
    transpose_bf16_kernel<<<grid, dim3(32, 8), 0, st>>>(src, rows, cols, lds, dst, ldd);
    SIDR_SCHECK(cudaGetLastError());
    return SIDR_OK;
}

long long pad8(long long x) { return (x + 7) / 8 * 8; }

// A split-K GEMM whose M x ldc result is the sum of its slices in slice order
// (deterministic): the slices go to `parts` (room for kMaxSplits slices),
// then split_sum_kernel adds them into C.
constexpr int kMaxSplits = 16;
sidr_status gemm_split_sum(GemmArgs g, int splits, float* parts, float* C, cudaStream_t st) {
    const long long count = (long long)g.M * g.ldc;
    g.epilogue = kSplitF32;
    g.C = parts;
    g.split_stride = count;
    int gz = 0;
    sidr_status s = launch_gemm(g, std::min(splits, kMaxSplits), st, &gz);
    if (s || gz == 0) return s;
    split_sum_kernel<<<(int)std::min<long long>((count + 255) / 256, 148 * 8), 256, 0, st>>>(parts, gz, count, C);
    SIDR_SCHECK(cudaGetLastError());
    return SIDR_OK;
}

// ------------------------------------------------------------------- model

struct Param {
    float* p = nullptr;
    float* g = nullptr;
    float* m = nullptr;
    float* v = nullptr;
    long long n = 0;
};

}  // namespace

struct sidr_mlp {
    int device = 0;
    cudaStream_t st = nullptr;
    Param W1, b1, W2, b2, w3, b3;  // W1 [kHid][kInPad], W2 [kHid][kHid]
    __nv_bfloat16 *W1b = nullptr, *W2b = nullptr;
    int cap = 0;  // rows of the activation buffers
    float *X = nullptr, *T = nullptr, *Xall = nullptr, *Tall = nullptr;
    int* idx = nullptr;
    int all_cap = 0;
    __nv_bfloat16 *Xb = nullptr, *H1b = nullptr, *H2b = nullptr, *dZ2b = nullptr, *dZ1b = nullptr;
    float *y = nullptr, *dy = nullptr, *dZ2 = nullptr, *dH1 = nullptr, *dZ1 = nullptr, *loss = nullptr;
    float* parts = nullptr;  // split-K partial sums of the weight gradients [kMaxSplits][kHid][kHid]
    // K-major copies of the operands the backward pass reads M- or N-contiguous
    __nv_bfloat16 *dZ2T = nullptr, *H1T = nullptr, *dZ1T = nullptr, *XbT = nullptr, *W2T = nullptr;
    long long ldT = 0;  // row stride of dZ2T/H1T/dZ1T/XbT: cap rounded up to 8
    int* err = nullptr;
    long long step = 0;
    std::vector<void*> owned;

    template <class T>
    cudaError_t alloc(T*& p, size_t n) {
        cudaError_t e = cudaMalloc(&p, n * sizeof(T));
        if (e == cudaSuccess) {
            owned.push_back(p);
            e = cudaMemset(p, 0, n * sizeof(T));
        }
        return e;
    }
    ~sidr_mlp() {
        for (void* p : owned) cudaFree(p);
        if (st) cudaStreamDestroy(st);
    }
};

namespace {

cudaError_t alloc_param(sidr_mlp* m, Param& p, long long n) {
    p.n = n;
    cudaError_t e;
    if ((e = m->alloc(p.p, n)) != cudaSuccess || (e = m->alloc(p.g, n)) != cudaSuccess ||
        (e = m->alloc(p.m, n)) != cudaSuccess || (e = m->alloc(p.v, n)) != cudaSuccess)
        return e;
    return cudaSuccess;
}

sidr_status ensure_rows(sidr_mlp* m, int rows) {
    if (rows <= m->cap) return SIDR_OK;
    const int cap = std::max(rows, 1024);
    cudaError_t e;
    if ((e = m->alloc(m->X, (size_t)cap * kIn)) || (e = m->alloc(m->T, cap)) ||
        (e = m->alloc(m->Xb, (size_t)cap * kInPad)) || (e = m->alloc(m->H1b, (size_t)cap * kHid)) ||
        (e = m->alloc(m->H2b, (size_t)cap * kHid)) || (e = m->alloc(m->dZ2b, (size_t)cap * kHid)) ||
        (e = m->alloc(m->dZ1b, (size_t)cap * kHid)) || (e = m->alloc(m->y, cap)) ||
        (e = m->alloc(m->dy, cap)) || (e = m->alloc(m->dZ2, (size_t)cap * kHid)) ||
        (e = m->alloc(m->dH1, (size_t)cap * kHid)) || (e = m->alloc(m->dZ1, (size_t)cap * kHid)) ||
        (e = m->alloc(m->dZ2T, (size_t)kHid * pad8(cap))) || (e = m->alloc(m->H1T, (size_t)kHid * pad8(cap))) ||
        (e = m->alloc(m->dZ1T, (size_t)kHid * pad8(cap))) || (e = m->alloc(m->XbT, (size_t)kInPad * pad8(cap))))
        return fail_s(SIDR_ERR_CUDA, std::string("surrogate buffers: ") + cudaGetErrorString(e));
    m->ldT = pad8(cap);
    m->cap = cap;  // (older, smaller buffers stay owned until the model is destroyed)
    return SIDR_OK;
}

void refresh_bf16(sidr_mlp* m) {
    to_bf16_kernel<<<grid_for(m->W1.n), 256, 0, m->st>>>(m->W1.p, m->W1b, m->W1.n);
    to_bf16_kernel<<<grid_for(m->W2.n), 256, 0, m->st>>>(m->W2.p, m->W2b, m->W2.n);
}

// forward pass over rows of m->X (already in m->X); fills Xb, H1b, H2b, y
sidr_status forward(sidr_mlp* m, int rows) {
    pad_inputs_kernel<<<grid_for((long long)rows * kInPad), 256, 0, m->st>>>(m->X, m->Xb, rows);
    GemmArgs g{};
    g.error = m->err;
    // H1 = relu(Xb W1^T + b1): M = rows, N = 256, K = 48
    g.A = m->Xb; g.lda = kInPad;
    g.B = m->W1b; g.ldb = kInPad;
    g.M = rows; g.N = kHid; g.K = kInPad;
    g.epilogue = kBiasRelu; g.bias = m->b1.p; g.Hb = m->H1b; g.ldh = kHid;
    sidr_status s = launch_gemm(g, 1, m->st);
    if (s) return s;
    // H2 = relu(H1 W2^T + b2): K = 256
    g.A = m->H1b; g.lda = kHid;
    g.B = m->W2b; g.ldb = kHid;
    g.K = kHid; g.bias = m->b2.p; g.Hb = m->H2b;
    if ((s = launch_gemm(g, 1, m->st))) return s;
    head_forward_kernel<<<(rows + 127) / 128, 128, 0, m->st>>>(m->H2b, m->w3.p, m->b3.p, m->y, rows);
    SIDR_SCHECK(cudaGetLastError());
    return SIDR_OK;
}

// loss and all gradients for the rows of m->X / m->T (forward included)
sidr_status backward(sidr_mlp* m, int rows) {
    sidr_status s = forward(m, rows);
    if (s) return s;
    cudaStream_t st = m->st;
    loss_kernel<<<1, 256, 0, st>>>(m->y, m->T, m->dy, m->loss, rows);
    head_backward_kernel<<<(kHid + 1 + 127) / 128, 128, 0, st>>>(m->H2b, m->dy, m->w3.g, m->b3.g, rows);
    head_delta_kernel<<<grid_for((long long)rows * kHid), 256, 0, st>>>(m->H2b, m->dy, m->w3.p, m->dZ2,
                                                                         m->dZ2b, rows);
    col_sum_kernel<<<(kHid + 127) / 128, 128, 0, st>>>(m->dZ2, m->b2.g, rows, kHid);
    const int splits = std::max(1, std::min(kMaxSplits, rows / 128));
    GemmArgs g{};
    g.error = m->err;
    // dW2[out][in] = sum_b dZ2[b][out] H1[b][in]: M = 256 (out), N = 256 (in), K = rows,
    // on K-major copies dZ2^T [out][b] and H1^T [in][b]
    if ((s = transpose(m->dZ2b, rows, kHid, kHid, m->dZ2T, m->ldT, st))) return s;
    if ((s = transpose(m->H1b, rows, kHid, kHid, m->H1T, m->ldT, st))) return s;
    g.A = m->dZ2T; g.lda = m->ldT;
    g.B = m->H1T; g.ldb = m->ldT;
    g.M = kHid; g.N = kHid; g.K = rows;
    g.ldc = kHid;
    if ((s = gemm_split_sum(g, splits, m->parts, m->W2.g, st))) return s;
    // dH1[b][in] = sum_out dZ2[b][out] W2[out][in]: M = rows, N = 256, K = 256, B = W2^T [in][out]
    if ((s = transpose(m->W2b, kHid, kHid, kHid, m->W2T, kHid, st))) return s;
    g.A = m->dZ2b; g.lda = kHid;
    g.B = m->W2T; g.ldb = kHid;
    g.M = rows; g.N = kHid; g.K = kHid;
    g.epilogue = kStoreF32; g.C = m->dH1; g.ldc = kHid;
    if ((s = launch_gemm(g, 1, st))) return s;
    relu_back_kernel<<<grid_for((long long)rows * kHid), 256, 0, st>>>(m->dH1, m->H1b, m->dZ1, m->dZ1b,
                                                                        (long long)rows * kHid);
    col_sum_kernel<<<(kHid + 127) / 128, 128, 0, st>>>(m->dZ1, m->b1.g, rows, kHid);
    // dW1[out][in] = sum_b dZ1[b][out] Xb[b][in]: M = 256, N = 48, K = rows, on dZ1^T and Xb^T
    if ((s = transpose(m->dZ1b, rows, kHid, kHid, m->dZ1T, m->ldT, st))) return s;
    if ((s = transpose(m->Xb, rows, kInPad, kInPad, m->XbT, m->ldT, st))) return s;
    g.A = m->dZ1T; g.lda = m->ldT;
    g.B = m->XbT; g.ldb = m->ldT;
    g.M = kHid; g.N = kInPad; g.K = rows;
    g.ldc = kInPad;
    if ((s = gemm_split_sum(g, splits, m->parts, m->W1.g, st))) return s;
    SIDR_SCHECK(cudaGetLastError());
    return SIDR_OK;
}

sidr_status adam_all(sidr_mlp* m, float lr) {
    m->step++;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float c1 = 1.0f - std::pow(b1, (float)m->step), c2 = 1.0f - std::pow(b2, (float)m->step);
    for (Param* p : {&m->W1, &m->b1, &m->W2, &m->b2, &m->w3, &m->b3})
        adam_kernel<<<grid_for(p->n), 256, 0, m->st>>>(p->p, p->g, p->m, p->v, p->n, lr, b1, b2, eps, c1, c2);
    refresh_bf16(m);
    SIDR_SCHECK(cudaGetLastError());
    return SIDR_OK;
}

sidr_status check_error(sidr_mlp* m) {
    int h = 0;
    SIDR_SCHECK(cudaMemcpyAsync(&h, m->err, sizeof(int), cudaMemcpyDeviceToHost, m->st));
    SIDR_SCHECK(cudaStreamSynchronize(m->st));
    if (h) return fail_s(SIDR_ERR_KERNEL, "a tensor-core MMA did not complete within its wait limit");
    return SIDR_OK;
}

Param* param_by_index(sidr_mlp* m, int i) {
    Param* ps[6] = {&m->W1, &m->b1, &m->W2, &m->b2, &m->w3, &m->b3};
    return (i >= 0 && i < 6) ? ps[i] : nullptr;
}

}  // namespace

extern "C" {

sidr_status sidr_gemm_bf16(const uint16_t* A, const uint16_t* B, int32_t M, int32_t N, int32_t K,
                           int32_t splits, int device, float* C) {
    if (!A || !B || !C || M < 1 || N < 1 || K < 1 || N > 256)
        return fail_s(SIDR_ERR_INVALID, "gemm: bad argument (1 <= N <= 256)");
    DeviceGuard device_guard;
    SIDR_SCHECK(cudaSetDevice(device));
    __nv_bfloat16 *dA = nullptr, *dB = nullptr;
    float* dC = nullptr;
    int* err = nullptr;
    const long long ld = pad8(K);  // rows padded to 16 bytes for the tensor maps
    cudaError_t e = cudaMalloc(&dA, (size_t)M * ld * 2);
    if (!e) e = cudaMalloc(&dB, (size_t)N * ld * 2);
    float* parts = nullptr;
    if (!e) e = cudaMalloc(&dC, (size_t)M * N * 4);
    if (!e && splits > 1) e = cudaMalloc(&parts, (size_t)kMaxSplits * M * N * 4);
    if (!e) e = cudaMalloc(&err, sizeof(int));
    if (!e) e = cudaMemcpy2D(dA, ld * 2, A, (size_t)K * 2, (size_t)K * 2, M, cudaMemcpyHostToDevice);
    if (!e) e = cudaMemcpy2D(dB, ld * 2, B, (size_t)K * 2, (size_t)K * 2, N, cudaMemcpyHostToDevice);
    if (!e) e = cudaMemset(dC, 0, (size_t)M * N * 4);
    if (!e) e = cudaMemset(err, 0, sizeof(int));
    sidr_status s = SIDR_OK;
    if (!e) {
        GemmArgs g{};
        g.A = dA; g.lda = ld;
        g.B = dB; g.ldb = ld;
        g.M = M; g.N = N; g.K = K;
        g.epilogue = kStoreF32;
        g.C = dC; g.ldc = N; g.error = err;
        s = splits > 1 ? gemm_split_sum(g, splits, parts, dC, 0) : launch_gemm(g, 1, 0);
        if (!s) e = cudaDeviceSynchronize();
    }
    int h = 0;
    if (!e && !s) e = cudaMemcpy(&h, err, sizeof(int), cudaMemcpyDeviceToHost);
    if (!e && !s) e = cudaMemcpy(C, dC, (size_t)M * N * 4, cudaMemcpyDeviceToHost);
    cudaFree(dA);
    cudaFree(dB);
    cudaFree(dC);
    cudaFree(parts);
    cudaFree(err);
    if (s) return s;
    if (e) return fail_s(SIDR_ERR_CUDA, std::string("gemm: ") + cudaGetErrorString(e));
    if (h) return fail_s(SIDR_ERR_KERNEL, "gemm: an MMA did not complete within its wait limit");
    return SIDR_OK;
}

sidr_status sidr_gemm_wait_check(int device, uint32_t wait_limit) {
    if (wait_limit < 1 || wait_limit > (1u << 20))
        return fail_s(SIDR_ERR_INVALID, "wait check: wait_limit out of 1..2^20");
    DeviceGuard device_guard;
    SIDR_SCHECK(cudaSetDevice(device));
    constexpr int M = 128, N = 48, K = 32;
    __nv_bfloat16 *dA = nullptr, *dB = nullptr;
    float* dC = nullptr;
    int* err = nullptr;
    cudaError_t e = cudaMalloc(&dA, (size_t)M * K * 2);
    if (!e) e = cudaMalloc(&dB, (size_t)N * K * 2);
    if (!e) e = cudaMalloc(&dC, (size_t)M * N * 4);
    if (!e) e = cudaMalloc(&err, sizeof(int));
    if (!e) e = cudaMemset(dA, 0, (size_t)M * K * 2);
    if (!e) e = cudaMemset(dB, 0, (size_t)N * K * 2);
    if (!e) e = cudaMemset(err, 0, sizeof(int));
    sidr_status s = SIDR_OK;
    if (!e) {
        GemmArgs g{};
        g.A = dA; g.lda = K;
        g.B = dB; g.ldb = K;
        g.M = M; g.N = N; g.K = K;
        g.epilogue = kStoreF32;
        g.C = dC; g.ldc = N; g.error = err;
        g.wait_limit = wait_limit;
        g.withhold = 1;
        s = launch_gemm(g, 1, 0);
        if (!s) e = cudaDeviceSynchronize();
    }
    int h = 0;
    if (!e && !s) e = cudaMemcpy(&h, err, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(dA);
    cudaFree(dB);
    cudaFree(dC);
    cudaFree(err);
    if (s) return s;
    if (e) return fail_s(SIDR_ERR_CUDA, std::string("wait check: ") + cudaGetErrorString(e));
    if (h) return fail_s(SIDR_ERR_KERNEL, "wait check: the MMA waits ran out and the kernel reported it");
    return SIDR_OK;
}

sidr_status sidr_phenotype(const sidr_rules_desc* r, const double* terms, const int32_t* ncand,
                           const int32_t* ref, int32_t n_sit, int32_t max_cand, int device,
                           float* features) {
    if (!r || !terms || !ncand || !ref || !features || n_sit < 1 || max_cand < 1)
        return fail_s(SIDR_ERR_INVALID, "bad argument");
    const int P = r->P, nf = n_sit + 8;
    for (int j = 0; j < n_sit; j++)
        if (ncand[j] < 1 || ncand[j] > max_cand || ref[j] < 0 || ref[j] >= ncand[j])
            return fail_s(SIDR_ERR_INVALID, "situation " + std::to_string(j) + ": bad candidate count or choice");
    // host: rule validity (the device interpreter trusts it) and token features
    for (int p = 0; p < P; p++) {
        const int32_t* o = r->ops + r->offsets[p];
        const int32_t* a = r->args + 2 * (size_t)r->offsets[p];
        const int L = r->lengths[p];
        if (L < 1 || L > 1024) return fail_s(SIDR_ERR_RULE, "rule " + std::to_string(p) + ": bad length");
        int sp = 0, depth_max = 0, leaves = 0, consts = 0, addsub = 0, muldiv = 0, other = 0;
        std::vector<int> dstack;
        bool seen[61] = {false};
        int distinct = 0;
        for (int k = 0; k < L; k++) {
            if (o[k] == -1 || o[k] == -2) {
                if (o[k] == -1) {
                    if (a[2 * k] < 0 || a[2 * k] >= 61) return fail_s(SIDR_ERR_RULE, "slot out of range");
                    if (!seen[a[2 * k]]) distinct++;
                    seen[a[2 * k]] = true;
                } else {
                    consts++;
                }
                leaves++;
                dstack.push_back(0);
                sp++;
            } else if (o[k] >= 0 && o[k] <= 6) {
                if (sp < 2) return fail_s(SIDR_ERR_RULE, "stack underflow");
                const int d1 = dstack.back();
                dstack.pop_back();
                const int d0 = dstack.back();
                dstack.pop_back();
                dstack.push_back(1 + std::max(d0, d1));
                depth_max = std::max(depth_max, dstack.back());
                sp--;
                if (o[k] <= 1) addsub++;
                else if (o[k] <= 3) muldiv++;
                else other++;
            } else {
                return fail_s(SIDR_ERR_RULE, "unknown opcode");
            }
            if (sp > 32) return fail_s(SIDR_ERR_RULE, "stack deeper than 32");
        }
        if (sp != 1) return fail_s(SIDR_ERR_RULE, "rule leaves more than one value");
        const int ops_n = std::max(1, addsub + muldiv + other);
        float* f = features + (size_t)p * nf + n_sit;
        f[0] = L / 255.0f;
        f[1] = depth_max / 16.0f;
        f[2] = leaves / 128.0f;
        f[3] = distinct / 32.0f;
        f[4] = consts / 32.0f;
        f[5] = (float)addsub / ops_n;
        f[6] = (float)muldiv / ops_n;
        f[7] = (float)other / ops_n;
    }
    if (P == 0) return SIDR_OK;
    DeviceGuard device_guard;
    SIDR_SCHECK(cudaSetDevice(device));
    const size_t nodes = (size_t)r->n_nodes;
    int32_t *d_ops = nullptr, *d_args = nullptr, *d_off = nullptr, *d_len = nullptr, *d_nc = nullptr,
            *d_ref = nullptr;
    double* d_terms = nullptr;
    float* d_feat = nullptr;
    const size_t tn = (size_t)n_sit * max_cand * 61;
    cudaError_t e = cudaMalloc(&d_ops, nodes * 4);
    if (!e) e = cudaMalloc(&d_args, nodes * 8);
    if (!e) e = cudaMalloc(&d_off, (size_t)P * 4);
    if (!e) e = cudaMalloc(&d_len, (size_t)P * 4);
    if (!e) e = cudaMalloc(&d_nc, (size_t)n_sit * 4);
    if (!e) e = cudaMalloc(&d_ref, (size_t)n_sit * 4);
    if (!e) e = cudaMalloc(&d_terms, tn * 8);
    if (!e) e = cudaMalloc(&d_feat, (size_t)P * nf * 4);
    if (!e) e = cudaMemcpy(d_ops, r->ops, nodes * 4, cudaMemcpyHostToDevice);
    if (!e) e = cudaMemcpy(d_args, r->args, nodes * 8, cudaMemcpyHostToDevice);
    if (!e) e = cudaMemcpy(d_off, r->offsets, (size_t)P * 4, cudaMemcpyHostToDevice);
    if (!e) e = cudaMemcpy(d_len, r->lengths, (size_t)P * 4, cudaMemcpyHostToDevice);
    if (!e) e = cudaMemcpy(d_nc, ncand, (size_t)n_sit * 4, cudaMemcpyHostToDevice);
    if (!e) e = cudaMemcpy(d_ref, ref, (size_t)n_sit * 4, cudaMemcpyHostToDevice);
    if (!e) e = cudaMemcpy(d_terms, terms, tn * 8, cudaMemcpyHostToDevice);
    if (!e) {
        const long long items = (long long)P * n_sit;
        phenotype_kernel<<<(int)((items + 127) / 128), 128>>>(d_ops, d_args, d_off, d_len, P, d_terms, d_nc,
                                                              d_ref, n_sit, max_cand, d_feat, nf);
        e = cudaGetLastError();
    }
    // the kernel wrote the ranking columns; the token columns come from the host
    std::vector<float> got;
    if (!e) {
        got.resize((size_t)P * nf);
        e = cudaMemcpy(got.data(), d_feat, got.size() * 4, cudaMemcpyDeviceToHost);
    }
    for (void* q : {(void*)d_ops, (void*)d_args, (void*)d_off, (void*)d_len, (void*)d_nc, (void*)d_ref,
                    (void*)d_terms, (void*)d_feat})
        cudaFree(q);
    if (e) return fail_s(SIDR_ERR_CUDA, std::string("phenotype: ") + cudaGetErrorString(e));
    for (int p = 0; p < P; p++)
        for (int j = 0; j < n_sit; j++) features[(size_t)p * nf + j] = got[(size_t)p * nf + j];
    return SIDR_OK;
}

sidr_status sidr_mlp_create(int device, uint64_t seed, sidr_mlp** out) {
    if (!out) return fail_s(SIDR_ERR_INVALID, "out is null");
    *out = nullptr;
    DeviceGuard device_guard;
    SIDR_SCHECK(cudaSetDevice(device));
    sidr_mlp* m = new sidr_mlp();
    m->device = device;
    cudaError_t e = cudaStreamCreateWithFlags(&m->st, cudaStreamNonBlocking);
    if (!e) e = alloc_param(m, m->W1, (long long)kHid * kInPad);
    if (!e) e = alloc_param(m, m->b1, kHid);
    if (!e) e = alloc_param(m, m->W2, (long long)kHid * kHid);
    if (!e) e = alloc_param(m, m->b2, kHid);
    if (!e) e = alloc_param(m, m->w3, kHid);
    if (!e) e = alloc_param(m, m->b3, 1);
    if (!e) e = m->alloc(m->W1b, (size_t)kHid * kInPad);
    if (!e) e = m->alloc(m->W2b, (size_t)kHid * kHid);
    if (!e) e = m->alloc(m->loss, 1);
    if (!e) e = m->alloc(m->err, 1);
    if (!e) e = m->alloc(m->parts, (size_t)kMaxSplits * kHid * kHid);
    if (!e) e = m->alloc(m->W2T, (size_t)kHid * kHid);
    if (e) {
        delete m;
        return fail_s(SIDR_ERR_CUDA, std::string("surrogate create: ") + cudaGetErrorString(e));
    }
    // He-uniform weights (bound sqrt(6 / fan_in)), zero biases; W1's padding columns stay zero
    std::mt19937_64 rng(seed);
    auto init = [&](Param& p, int rows, int cols, int fan_in, int used_cols) -> cudaError_t {
        std::vector<float> h((size_t)rows * cols, 0.0f);
        const float bound = std::sqrt(6.0f / fan_in);
        std::uniform_real_distribution<float> U(-bound, bound);
        for (int r = 0; r < rows; r++)
            for (int c = 0; c < used_cols; c++) h[(size_t)r * cols + c] = U(rng);
        return cudaMemcpy(p.p, h.data(), h.size() * 4, cudaMemcpyHostToDevice);
    };
    if (!e) e = init(m->W1, kHid, kInPad, kIn, kIn);
    if (!e) e = init(m->W2, kHid, kHid, kHid, kHid);
    if (!e) e = init(m->w3, 1, kHid, kHid, kHid);
    if (e) {
        delete m;
        return fail_s(SIDR_ERR_CUDA, std::string("surrogate init: ") + cudaGetErrorString(e));
    }
    refresh_bf16(m);
    if ((e = cudaStreamSynchronize(m->st))) {
        delete m;
        return fail_s(SIDR_ERR_CUDA, std::string("surrogate init: ") + cudaGetErrorString(e));
    }
    *out = m;
    return SIDR_OK;
}

void sidr_mlp_destroy(sidr_mlp* m) { delete m; }

sidr_status sidr_mlp_param(sidr_mlp* m, int32_t which, int32_t write, float* values, float* grads,
                           int64_t* count) {
    if (!m) return fail_s(SIDR_ERR_INVALID, "null model");
    Param* p = param_by_index(m, which);
    if (!p) return fail_s(SIDR_ERR_INVALID, "parameter index 0..5");
    if (count) *count = p->n;
    DeviceGuard device_guard;
    SIDR_SCHECK(cudaSetDevice(m->device));
    SIDR_SCHECK(cudaStreamSynchronize(m->st));
    if (values) {
        if (write) {
            SIDR_SCHECK(cudaMemcpy(p->p, values, p->n * 4, cudaMemcpyHostToDevice));
            refresh_bf16(m);
            SIDR_SCHECK(cudaStreamSynchronize(m->st));
        } else {
            SIDR_SCHECK(cudaMemcpy(values, p->p, p->n * 4, cudaMemcpyDeviceToHost));
        }
    }
    if (grads) SIDR_SCHECK(cudaMemcpy(grads, p->g, p->n * 4, cudaMemcpyDeviceToHost));
    return SIDR_OK;
}

sidr_status sidr_mlp_state(sidr_mlp* m, int32_t write, float* state, int64_t* count, int64_t* step) {
    if (!m) return fail_s(SIDR_ERR_INVALID, "null model");
    int64_t total = 0;
    for (int w = 0; w < 6; w++) total += 3 * param_by_index(m, w)->n;
    if (count) *count = total;
    if (!state) {
        if (step) *step = m->step;
        return SIDR_OK;
    }
    DeviceGuard device_guard;
    SIDR_SCHECK(cudaSetDevice(m->device));
    SIDR_SCHECK(cudaStreamSynchronize(m->st));
    float* at = state;
    for (int w = 0; w < 6; w++) {
        Param* p = param_by_index(m, w);
        for (float* dev : {p->p, p->m, p->v}) {
            if (write) SIDR_SCHECK(cudaMemcpy(dev, at, p->n * 4, cudaMemcpyHostToDevice));
            else SIDR_SCHECK(cudaMemcpy(at, dev, p->n * 4, cudaMemcpyDeviceToHost));
            at += p->n;
        }
    }
    if (write) {
        if (step) m->step = *step;
        refresh_bf16(m);
        SIDR_SCHECK(cudaStreamSynchronize(m->st));
    } else if (step) {
        *step = m->step;
    }
    return SIDR_OK;
}

sidr_status sidr_mlp_predict(sidr_mlp* m, const float* x, int32_t rows, float* y) {
    if (!m || (rows > 0 && (!x || !y)) || rows < 0) return fail_s(SIDR_ERR_INVALID, "bad argument");
    if (rows == 0) return SIDR_OK;
    DeviceGuard device_guard;
    SIDR_SCHECK(cudaSetDevice(m->device));
    sidr_status s = ensure_rows(m, rows);
    if (s) return s;
    SIDR_SCHECK(cudaMemcpyAsync(m->X, x, (size_t)rows * kIn * 4, cudaMemcpyHostToDevice, m->st));
    if ((s = forward(m, rows))) return s;
    SIDR_SCHECK(cudaMemcpyAsync(y, m->y, (size_t)rows * 4, cudaMemcpyDeviceToHost, m->st));
    return check_error(m);
}

sidr_status sidr_mlp_gradients(sidr_mlp* m, const float* x, const float* t, int32_t rows, float* loss) {
    if (!m || !x || !t || rows < 1) return fail_s(SIDR_ERR_INVALID, "bad argument");
    DeviceGuard device_guard;
    SIDR_SCHECK(cudaSetDevice(m->device));
    sidr_status s = ensure_rows(m, rows);
    if (s) return s;
    SIDR_SCHECK(cudaMemcpyAsync(m->X, x, (size_t)rows * kIn * 4, cudaMemcpyHostToDevice, m->st));
    SIDR_SCHECK(cudaMemcpyAsync(m->T, t, (size_t)rows * 4, cudaMemcpyHostToDevice, m->st));
    if ((s = backward(m, rows))) return s;
    if (loss) SIDR_SCHECK(cudaMemcpyAsync(loss, m->loss, 4, cudaMemcpyDeviceToHost, m->st));
    return check_error(m);
}

sidr_status sidr_mlp_train(sidr_mlp* m, const float* x, const float* t, int32_t n, int32_t steps,
                           int32_t batch, float lr, uint64_t seed, float* final_loss) {
    if (!m || !x || !t || n < 1 || steps < 0 || batch < 1)
        return fail_s(SIDR_ERR_INVALID, "bad argument");
    DeviceGuard device_guard;
    SIDR_SCHECK(cudaSetDevice(m->device));
    const int rows = std::min(batch, n);
    sidr_status s = ensure_rows(m, rows);
    if (s) return s;
    if (n > m->all_cap) {
        cudaError_t e;
        if ((e = m->alloc(m->Xall, (size_t)n * kIn)) || (e = m->alloc(m->Tall, n)) ||
            (e = m->alloc(m->idx, (size_t)std::max(n, 1024))))
            return fail_s(SIDR_ERR_CUDA, std::string("surrogate data: ") + cudaGetErrorString(e));
        m->all_cap = n;
    }
    SIDR_SCHECK(cudaMemcpyAsync(m->Xall, x, (size_t)n * kIn * 4, cudaMemcpyHostToDevice, m->st));
    SIDR_SCHECK(cudaMemcpyAsync(m->Tall, t, (size_t)n * 4, cudaMemcpyHostToDevice, m->st));
    // minibatches drawn without replacement from a shuffled order, reshuffled per pass
    std::mt19937_64 rng(seed);
    std::vector<int> order(n), pick(rows);
    for (int i = 0; i < n; i++) order[i] = i;
    std::shuffle(order.begin(), order.end(), rng);
    int at = 0;
    for (int k = 0; k < steps; k++) {
        for (int r = 0; r < rows; r++) {
            if (at == n) {
                std::shuffle(order.begin(), order.end(), rng);
                at = 0;
            }
            pick[r] = order[at++];
        }
        SIDR_SCHECK(cudaMemcpyAsync(m->idx, pick.data(), rows * 4, cudaMemcpyHostToDevice, m->st));
        gather_rows_kernel<<<grid_for((long long)rows * kIn), 256, 0, m->st>>>(m->Xall, m->Tall, m->idx,
                                                                               m->X, m->T, rows, kIn);
        if ((s = backward(m, rows))) return s;
        if ((s = adam_all(m, lr))) return s;
        // the pinned pick buffer is reused: wait before the host rewrites it
        SIDR_SCHECK(cudaStreamSynchronize(m->st));
    }
    if (final_loss) SIDR_SCHECK(cudaMemcpyAsync(final_loss, m->loss, 4, cudaMemcpyDeviceToHost, m->st));
    return check_error(m);
}

}  // extern "C"
