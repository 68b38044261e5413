// sidr_sample.cu -- scenario sampling on the GPU (gen_durations,
// engine/sim_host.hpp:50-58 with the generator of engine/rng.hpp:27-147),
// bit-identical to the host's sidr_gen_durations.
//
// One warp per scenario.  Scenario s seeds a fresh MT19937 with base_seed + s
// (init_by_array over the seed's 32-bit words, least significant first); the
// warp keeps the 624-word state in shared memory: lane 0 runs the seeding
// recurrence, which is sequential, and the warp refreshes the state (the
// "twist") in three phases whose reads all precede their writes.  Each
// Box-Muller pair takes four consecutive 32-bit outputs (two 53-bit draws),
// so a refresh of 624 words serves 156 pairs, which the lanes take in turn.
// Customers with a positive expected service time draw in index order, one
// Gaussian each (cos of a pair, then its sin); the others get 0 and draw
// nothing.  The pair's durations come from sidr_sample.cuh; a pair it cannot
// settle is recorded (scenario, pair, the two draws) and recomputed on the
// host with the C library after the kernel, then written over the device's
// guess.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "../../include/sidr.h"
#include "../../include/sidr_gp.h"
#include "sidr_device.hpp"
#include "sidr_host.hpp"
#include "sidr_sample.cuh"

namespace sidr {
namespace smp {
namespace {

constexpr int kN = kMtN;
constexpr int kPairsPerRefresh = kN / 4;  // four 32-bit outputs per pair
constexpr int kWarps = 8;                 // warps per block, a scenario each

struct FlagRec {
    int32_t s, p;
    double u1, u2;
};

struct SampleArgs {
    int n, S, npos, npairs, nzero;
    long long base_seed;
    const double* mu;      // [npos] expected service times of the drawing customers, in index order
    const double* sd;      // [npos] sigma * mu
    const int32_t* cust;   // [npos] their customer indices
    const int32_t* zeros;  // [nzero] customers that draw nothing
    double* out;           // [S][n]
    unsigned long long* nflag;
    FlagRec* flags;
    long long flag_cap;
};

// A state refresh by the whole warp: each phase computes its words from the
// current state, then stores them.
__device__ void refresh(uint32_t* mt, int lane) {
    uint32_t nv[8];
    const int lo[3] = {0, kMtN - kMtM, 2 * (kMtN - kMtM)};
    const int hi[3] = {kMtN - kMtM, 2 * (kMtN - kMtM), kMtN - 1};
#pragma unroll
    for (int ph = 0; ph < 3; ph++) {
#pragma unroll
        for (int t = 0; t < 8; t++) {
            const int kk = lo[ph] + lane + 32 * t;
            if (kk < hi[ph]) nv[t] = mt_refreshed(mt, kk);
        }
        __syncwarp();
#pragma unroll
        for (int t = 0; t < 8; t++) {
            const int kk = lo[ph] + lane + 32 * t;
            if (kk < hi[ph]) mt[kk] = nv[t];
        }
        __syncwarp();
    }
    if (lane == 0) mt[kMtN - 1] = mt_refreshed_last(mt);
    __syncwarp();
}

__global__ void __launch_bounds__(32 * kWarps) sample_kernel(const SampleArgs A) {
    __shared__ uint32_t state[kWarps][kN];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    uint32_t* mt = state[wib];
    const int warps = gridDim.x * kWarps;
    for (int s = blockIdx.x * kWarps + wib; s < A.S; s += warps) {
        double* row = A.out + (size_t)s * A.n;
        for (int z = lane; z < A.nzero; z += 32) row[A.zeros[z]] = 0.0;
        if (A.npairs == 0) continue;
        if (lane == 0) mt_seed(mt, (unsigned long long)(A.base_seed + s));
        __syncwarp();
        for (int blk = 0; blk * kPairsPerRefresh < A.npairs; blk++) {
            refresh(mt, lane);
            const int p0 = blk * kPairsPerRefresh;
            for (int pp = lane; pp < kPairsPerRefresh && p0 + pp < A.npairs; pp += 32) {
                const int p = p0 + pp;
                const double u1 = mt_draw(mt[4 * pp], mt[4 * pp + 1]);
                const double u2 = mt_draw(mt[4 * pp + 2], mt[4 * pp + 3]);
                const int g0 = 2 * p, g1 = 2 * p + 1;
                const bool has1 = g1 < A.npos;
                double d0, d1;
                const bool ok = gauss_pair_durations(u1, u2, A.mu[g0], A.sd[g0], has1, has1 ? A.mu[g1] : 0.0,
                                                     has1 ? A.sd[g1] : 0.0, d0, d1);
                row[A.cust[g0]] = d0;
                if (has1) row[A.cust[g1]] = d1;
                if (!ok) {
                    const unsigned long long at = atomicAdd(A.nflag, 1ull);
                    if ((long long)at < A.flag_cap) A.flags[at] = FlagRec{s, p, u1, u2};
                }
            }
            __syncwarp();  // the pairs' reads of this refresh are done
        }
    }
}

// The double-double log, sin and cos of draws u1, u2 with the candidates
// they name (diagnostic): {log hi, lo, second candidate, sin hi, lo, second,
// cos hi, lo, second} of 1 - u2 and u1 * 2 pi.
constexpr int kEvalWidth = 9;
SIDR_HD void dd_eval_one(double u1, double u2, double* o) {
    constexpr double kTwoPi = 2.0 * 3.14159265358979323846;
    const dd lg = log_dd(1.0 - u2);
    dd sn, cs;
    sincos_dd(u1 * kTwoPi, sn, cs);
    double c[2];
    candidates(lg, kGuardLog, c);
    o[0] = lg.hi;
    o[1] = lg.lo;
    o[2] = c[1];
    candidates(sn, kGuardTrig, c);
    o[3] = sn.hi;
    o[4] = sn.lo;
    o[5] = c[1];
    candidates(cs, kGuardTrig, c);
    o[6] = cs.hi;
    o[7] = cs.lo;
    o[8] = c[1];
}

__global__ void dd_eval_kernel(const double* u1, const double* u2, int k, double* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < k) dd_eval_one(u1[i], u2[i], out + kEvalWidth * (size_t)i);
}

__global__ void patch_kernel(double* out, const long long* idx, const double* val, int k) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < k) out[idx[i]] = val[i];
}

// The pair as the reference computes it, with this host's C library
// (engine/rng.hpp:135-147): x2pi from the first draw, g2rad from the second.
void host_pair(double u1, double u2, double mu0, double sd0, bool has1, double mu1, double sd1, double& d0,
               double& d1) {
    constexpr double kTwoPi = 2.0 * 3.14159265358979323846;
    const double x2pi = u1 * kTwoPi;
    const double g2rad = std::sqrt(-2.0 * std::log(1.0 - u2));
    const double z0 = std::cos(x2pi) * g2rad;
    const double z1 = std::sin(x2pi) * g2rad;
    const double v0 = mu0 + z0 * sd0;
    d0 = v0 > 0.0 ? v0 : 0.0;
    const double v1 = mu1 + z1 * sd1;
    d1 = has1 ? (v1 > 0.0 ? v1 : 0.0) : 0.0;
}

template <class T>
struct DevArr {
    T* p = nullptr;
    ~DevArr() {
        if (p) cudaFree(p);
    }
    cudaError_t alloc(size_t n) { return cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)); }
};

}  // namespace
}  // namespace smp
}  // namespace sidr

using namespace sidr::smp;

namespace {
sidr_status fail_s(sidr_status s, const std::string& m) {
    sidr::set_last_error(m);
    return s;
}
}  // namespace

extern "C" sidr_status sidr_gen_durations_device(int32_t device, int32_t n, const double* durations, double sigma,
                                                 int32_t S, int64_t base_seed, double* out, int32_t out_on_device,
                                                 sidr_sample_stats* stats) {
    if (n < 0 || S < 0 || (n > 0 && S > 0 && (!durations || !out)))
        return fail_s(SIDR_ERR_INVALID, "bad argument");
    if (!std::isfinite(sigma)) return fail_s(SIDR_ERR_NONFINITE, "sigma is not finite");
    if ((long long)S * n > (1ll << 40)) return fail_s(SIDR_ERR_TOO_LARGE, "S * n too large");
    std::vector<double> mu, sd;
    std::vector<int32_t> cust, zeros;
    for (int i = 0; i < n; i++) {
        const double e = durations[i];
        if (!std::isfinite(e)) return fail_s(SIDR_ERR_NONFINITE, "expected service time is not finite");
        if (e > 0.0) {  // zero-duration visits draw nothing
            mu.push_back(e);
            sd.push_back(sigma * e);
            cust.push_back(i);
        } else {
            zeros.push_back(i);
        }
    }
    const int npos = (int)mu.size(), npairs = (npos + 1) / 2;
    if (stats) {
        stats->pairs = (int64_t)S * npairs;
        stats->host_pairs = 0;
    }
    if ((long long)S * n == 0) return SIDR_OK;
    sidr::DeviceGuard device_guard;
    cudaError_t e = cudaSetDevice(device);
    DevArr<double> d_mu, d_sd, d_out;
    DevArr<int32_t> d_cust, d_zeros;
    DevArr<unsigned long long> d_nflag;
    DevArr<FlagRec> d_flags;
    // records of unsettled pairs: room for an eighth of the pairs (about 5 % are
    // unsettled); a block with more falls back to the host sampler as a whole
    const long long all_pairs = (long long)S * npairs;
    const long long cap = std::min(all_pairs, std::max(4096ll, all_pairs / 8));
    cudaStream_t st = nullptr;
    if (!e) e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (!e) e = d_mu.alloc(npos);
    if (!e) e = d_sd.alloc(npos);
    if (!e) e = d_cust.alloc(npos);
    if (!e) e = d_zeros.alloc(zeros.size());
    if (!e) e = d_nflag.alloc(1);
    if (!e) e = d_flags.alloc((size_t)cap);
    if (!e && !out_on_device) e = d_out.alloc((size_t)S * n);
    double* dst = out_on_device ? out : d_out.p;
    if (!e && npos) e = cudaMemcpyAsync(d_mu.p, mu.data(), npos * 8, cudaMemcpyHostToDevice, st);
    if (!e && npos) e = cudaMemcpyAsync(d_sd.p, sd.data(), npos * 8, cudaMemcpyHostToDevice, st);
    if (!e && npos) e = cudaMemcpyAsync(d_cust.p, cust.data(), npos * 4, cudaMemcpyHostToDevice, st);
    if (!e && !zeros.empty())
        e = cudaMemcpyAsync(d_zeros.p, zeros.data(), zeros.size() * 4, cudaMemcpyHostToDevice, st);
    if (!e) e = cudaMemsetAsync(d_nflag.p, 0, sizeof(unsigned long long), st);
    int sms = 148;
    if (!e) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (!e) {
        SampleArgs a{n, S, npos, npairs, (int)zeros.size(), (long long)base_seed, d_mu.p, d_sd.p, d_cust.p,
                     d_zeros.p, dst, d_nflag.p, d_flags.p, cap};
        const int grid = std::max(1, std::min((S + kWarps - 1) / kWarps, sms * 4));
        sample_kernel<<<grid, 32 * kWarps, 0, st>>>(a);
        e = cudaGetLastError();
    }
    unsigned long long nflag = 0;
    if (!e) e = cudaMemcpyAsync(&nflag, d_nflag.p, sizeof nflag, cudaMemcpyDeviceToHost, st);
    if (!e) e = cudaStreamSynchronize(st);
    if (!e && (long long)nflag > cap) {
        // more unsettled pairs than records: the host sampler gives the block
        std::vector<double> host;
        double* hout = out;
        if (out_on_device) {
            host.resize((size_t)S * n);
            hout = host.data();
        }
        const sidr_status hs = sidr_gen_durations(n, durations, sigma, S, base_seed, hout);
        if (hs != SIDR_OK) {
            cudaStreamDestroy(st);
            return hs;
        }
        if (out_on_device) e = cudaMemcpy(out, hout, (size_t)S * n * 8, cudaMemcpyHostToDevice);
        cudaStreamDestroy(st);
        if (e) return fail_s(SIDR_ERR_CUDA, std::string("sampling: ") + cudaGetErrorString(e));
        if (stats) stats->host_pairs = all_pairs;
        return SIDR_OK;
    }
    std::vector<FlagRec> fl;
    if (!e && nflag) {
        fl.resize((size_t)nflag);
        e = cudaMemcpyAsync(fl.data(), d_flags.p, fl.size() * sizeof(FlagRec), cudaMemcpyDeviceToHost, st);
        if (!e) e = cudaStreamSynchronize(st);
    }
    // the pairs the device left to the C library
    std::vector<long long> pidx;
    std::vector<double> pval;
    for (const FlagRec& f : fl) {
        const int g0 = 2 * f.p, g1 = 2 * f.p + 1;
        const bool has1 = g1 < npos;
        double d0, d1;
        host_pair(f.u1, f.u2, mu[g0], sd[g0], has1, has1 ? mu[g1] : 0.0, has1 ? sd[g1] : 0.0, d0, d1);
        pidx.push_back((long long)f.s * n + cust[g0]);
        pval.push_back(d0);
        if (has1) {
            pidx.push_back((long long)f.s * n + cust[g1]);
            pval.push_back(d1);
        }
    }
    if (!e && !out_on_device) {
        e = cudaMemcpyAsync(out, d_out.p, (size_t)S * n * 8, cudaMemcpyDeviceToHost, st);
        if (!e) e = cudaStreamSynchronize(st);
        if (!e)
            for (size_t k = 0; k < pidx.size(); k++) out[pidx[k]] = pval[k];
    } else if (!e && !pidx.empty()) {
        DevArr<long long> d_idx;
        DevArr<double> d_val;
        e = d_idx.alloc(pidx.size());
        if (!e) e = d_val.alloc(pval.size());
        if (!e) e = cudaMemcpyAsync(d_idx.p, pidx.data(), pidx.size() * 8, cudaMemcpyHostToDevice, st);
        if (!e) e = cudaMemcpyAsync(d_val.p, pval.data(), pval.size() * 8, cudaMemcpyHostToDevice, st);
        if (!e) {
            const int k = (int)pidx.size();
            patch_kernel<<<(k + 255) / 256, 256, 0, st>>>(out, d_idx.p, d_val.p, k);
            e = cudaGetLastError();
        }
        if (!e) e = cudaStreamSynchronize(st);
    }
    if (st) cudaStreamDestroy(st);
    if (e) return fail_s(SIDR_ERR_CUDA, std::string("sampling: ") + cudaGetErrorString(e));
    if (stats) stats->host_pairs = (int64_t)fl.size();
    return SIDR_OK;
}

extern "C" sidr_status sidr_sample_dd_eval(int32_t device, const double* u1, const double* u2, int32_t k,
                                           int32_t on_device, double* out) {
    if (k < 0 || (k > 0 && (!u1 || !u2 || !out))) return fail_s(SIDR_ERR_INVALID, "bad argument");
    if (k == 0) return SIDR_OK;
    if (!on_device) {
        for (int i = 0; i < k; i++) dd_eval_one(u1[i], u2[i], out + kEvalWidth * (size_t)i);
        return SIDR_OK;
    }
    sidr::DeviceGuard device_guard;
    cudaError_t e = cudaSetDevice(device);
    DevArr<double> a, b, o;
    if (!e) e = a.alloc(k);
    if (!e) e = b.alloc(k);
    if (!e) e = o.alloc(kEvalWidth * (size_t)k);
    if (!e) e = cudaMemcpy(a.p, u1, k * 8, cudaMemcpyHostToDevice);
    if (!e) e = cudaMemcpy(b.p, u2, k * 8, cudaMemcpyHostToDevice);
    if (!e) {
        dd_eval_kernel<<<(k + 127) / 128, 128>>>(a.p, b.p, k, o.p);
        e = cudaGetLastError();
    }
    if (!e) e = cudaMemcpy(out, o.p, kEvalWidth * (size_t)k * 8, cudaMemcpyDeviceToHost);
    if (e) return fail_s(SIDR_ERR_CUDA, std::string("sample dd eval: ") + cudaGetErrorString(e));
    return SIDR_OK;
}
