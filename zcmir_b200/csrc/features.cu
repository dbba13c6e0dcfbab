// Per-image SMI features (the reference's Smi.prepare, src/smi.zig:348-400):
// mean and spread → z → 256-bin histogram mid-rank → [r, r², Sobel |∇r|, fourth] → global ridge
// whitening → autocorrelation at |τ| ≤ 8 → the premultiplied stack [1, f0..f3].
//
// Per-pixel arithmetic is float32 with every operation rounded on its own in the reference's
// order (__fadd_rn & co. keep the compiler from fusing them), so the histogram bins and ranks
// match a float32 restatement bit for bit; the image-wide sums are float64 (the reference sums
// in float32).
#include <cuda_fp16.h>

#include "common.cuh"
#include "kernels.hpp"

namespace zc {
namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ float mean_of(const double* stats, int n) {
    return __double2float_rn(stats[0] / (double)n);
}
__device__ __forceinline__ float spread_of(const double* stats, int n) {
    return __double2float_rn(sqrt(fmax(stats[1] / (double)n, 1e-12)));
}

// f16 texels and back (src/gls.zig:433-442 with half precision)
__global__ void k_quant_half(float* g, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        g[i] = __half2float(__float2half_rn(g[i]));
}

// Σg (shaders/smi.wgsl:520-529 reduce1, float64 here)
__global__ void k_sum(const float* __restrict__ g, int n, double* stats) {
    __shared__ double sh[32];
    double acc = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) acc += (double)g[i];
    acc = block_sum(acc, sh);
    if (threadIdx.x == 0) atomicAdd(&stats[0], acc);
}

// Σ(g − mean)² with g − mean rounded to f32 (zscore_p then feat_moments, smi.wgsl:1548-1570)
__global__ void k_sumsq(const float* __restrict__ g, int n, double* stats) {
    __shared__ double sh[32];
    const float mean = mean_of(stats, n);
    double acc = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double d = (double)__fsub_rn(g[i], mean);
        acc += d * d;
    }
    acc = block_sum(acc, sh);
    if (threadIdx.x == 0) atomicAdd(&stats[1], acc);
}

__device__ __forceinline__ unsigned bin_of(float g, float mean, float spread) {
    const float z = __fdiv_rn(__fsub_rn(g, mean), fmaxf(spread, 1e-8f));
    const float x = __fmul_rn(__fadd_rn(z, 4.0f), 32.0f);
    return (unsigned)fminf(fmaxf(x, 0.0f), 255.0f);
}

// 256-bin histogram of z over [−4, 4] (smi.wgsl:393-399)
__global__ void k_hist(const float* __restrict__ g, int n, const double* stats, unsigned* hist) {
    __shared__ unsigned sh[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) sh[i] = 0;
    __syncthreads();
    const float mean = mean_of(stats, n), spread = spread_of(stats, n);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        atomicAdd(&sh[bin_of(g[i], mean, spread)], 1u);
    __syncthreads();
    for (int i = threadIdx.x; i < 256; i += blockDim.x)
        if (sh[i]) atomicAdd(&hist[i], sh[i]);
}

// mid-rank r = (cdf[b] + ½hist[b]) / N · 2 − 1 (smi.wgsl:401-420); every block scans the
// 256 bins itself
__global__ void k_rank(const float* __restrict__ g, int n, const double* stats, const unsigned* hist,
                       float* __restrict__ rank) {
    __shared__ unsigned sh_h[256], sh_c[256];
    __shared__ unsigned sh_tot;
    if (threadIdx.x < 256) sh_h[threadIdx.x] = hist[threadIdx.x];
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned acc = 0;
        for (int i = 0; i < 256; ++i) {
            sh_c[i] = acc;
            acc += sh_h[i];
        }
        sh_tot = acc > 0 ? acc : 1u;
    }
    __syncthreads();
    const float mean = mean_of(stats, n), spread = spread_of(stats, n);
    const float tot = (float)sh_tot;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const unsigned b = bin_of(g[i], mean, spread);
        const float c = __fadd_rn((float)sh_c[b], __fmul_rn(0.5f, (float)sh_h[b]));
        rank[i] = __fsub_rn(__fmul_rn(__fdiv_rn(c, tot), 2.0f), 1.0f);
    }
}

// [r, r², Sobel |∇r|, fourth] with clamp-to-edge borders (smi.wgsl:422-462)
__global__ void k_feats(const float* __restrict__ r, int w, int h, int mode, float* __restrict__ feat,
                        float* __restrict__ mag) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    auto t = [&](int dx, int dy) {
        const int xx = min(max(x + dx, 0), w - 1), yy = min(max(y + dy, 0), h - 1);
        return __ldg(&r[(size_t)yy * w + xx]);
    };
    const float c = t(0, 0);
    float gx = __fadd_rn(-t(-1, -1), t(1, -1));
    gx = __fsub_rn(gx, __fmul_rn(2.0f, t(-1, 0)));
    gx = __fadd_rn(gx, __fmul_rn(2.0f, t(1, 0)));
    gx = __fsub_rn(gx, t(-1, 1));
    gx = __fadd_rn(gx, t(1, 1));
    float gy = __fsub_rn(-t(-1, -1), __fmul_rn(2.0f, t(0, -1)));
    gy = __fsub_rn(gy, t(1, -1));
    gy = __fadd_rn(gy, t(-1, 1));
    gy = __fadd_rn(gy, __fmul_rn(2.0f, t(0, 1)));
    gy = __fadd_rn(gy, t(1, 1));
    const float g = __fsqrt_rn(__fadd_rn(__fmul_rn(gx, gx), __fmul_rn(gy, gy)));
    float f3 = 0.0f;
    if (mode == 0) {
        f3 = __fadd_rn(__fadd_rn(__fadd_rn(t(-1, 0), t(1, 0)), t(0, -1)), t(0, 1));
        f3 = __fsub_rn(f3, __fmul_rn(4.0f, c));
    } else if (mode == 2) {
        f3 = __fmul_rn(__fmul_rn(c, c), c);
    }
    const size_t n = (size_t)w * h, i = (size_t)y * w + x;
    feat[i] = c;
    feat[n + i] = __fmul_rn(c, c);
    feat[2 * n + i] = g;
    feat[3 * n + i] = f3;
    mag[i] = g;
}

// Σx_i (4) and Σx_i x_j (16) in float64 (smi.wgsl:531-551)
__global__ void k_featmom(const float* __restrict__ feat, int n, double* mom) {
    __shared__ double sh[32];
    double a[20];
#pragma unroll
    for (int k = 0; k < 20; ++k) a[k] = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double x[4];
#pragma unroll
        for (int p = 0; p < 4; ++p) x[p] = (double)feat[(size_t)p * n + i];
#pragma unroll
        for (int p = 0; p < 4; ++p) {
            a[p] += x[p];
#pragma unroll
            for (int q = 0; q < 4; ++q) a[4 + p * 4 + q] += x[p] * x[q];
        }
    }
#pragma unroll
    for (int k = 0; k < 20; ++k) {
        const double v = block_sum(a[k], sh);
        if (threadIdx.x == 0) atomicAdd(&mom[k], v);
    }
}

// global ridge whitening L⁻¹ and μ (smi.wgsl:553-585), float64, stored as f32
__global__ void k_chol(const double* mom, int n, float ridge, float* wt) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const double nn = fmax((double)n, 1.0);
    double mu[4], G[16], L[16] = {0}, X[16];
    for (int i = 0; i < 4; ++i) mu[i] = mom[i] / nn;
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) G[i * 4 + j] = mom[4 + i * 4 + j] / nn - mu[i] * mu[j];
    double tr = 0.0;
    for (int i = 0; i < 4; ++i) tr += G[i * 5];
    const double rg = (double)ridge * fmax(tr * 0.25, 1e-12);
    for (int i = 0; i < 4; ++i) G[i * 5] += rg;
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j <= i; ++j) {
            double s = G[i * 4 + j];
            for (int k = 0; k < j; ++k) s -= L[i * 4 + k] * L[j * 4 + k];
            if (i == j) L[i * 5] = sqrt(fmax(s, 1e-12));
            else L[i * 4 + j] = s / L[j * 5];
        }
    for (int col = 0; col < 4; ++col)
        for (int i = 0; i < 4; ++i) {
            double s = (i == col) ? 1.0 : 0.0;
            for (int k = 0; k < i; ++k) s -= L[i * 4 + k] * X[k * 4 + col];
            X[i * 4 + col] = s / L[i * 5];
        }
    for (int i = 0; i < 16; ++i) wt[i] = (float)X[i];
    for (int i = 0; i < 4; ++i) wt[16 + i] = (float)mu[i];
}

// x ← L⁻¹(x − μ), products rounded one by one in j order (smi.wgsl:587-599)
__global__ void k_whiten(float* __restrict__ feat, int n, const float* __restrict__ wt) {
    __shared__ float X[20];
    if (threadIdx.x < 20) X[threadIdx.x] = wt[threadIdx.x];
    __syncthreads();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float d[4];
#pragma unroll
        for (int p = 0; p < 4; ++p) d[p] = __fsub_rn(feat[(size_t)p * n + i], X[16 + p]);
#pragma unroll
        for (int p = 0; p < 4; ++p) {
            float s = __fmul_rn(X[p * 4], d[0]);
#pragma unroll
            for (int q = 1; q < 4; ++q) s = __fadd_rn(s, __fmul_rn(X[p * 4 + q], d[q]));
            feat[(size_t)p * n + i] = s;
        }
    }
}

// Autocorrelation partial sums (smi.wgsl:935-975): one block per 32×32 tile with an 8-px halo in
// shared memory (zero outside the image, so a pair with either pixel outside adds nothing and
// every lag sums exactly the pairs inside the image). Register-blocked: thread (plane p, row lag
// dy, row group g) takes the tile rows g, g + 4, …, and for each holds the row (32 values) and
// its partner row at dy with the column halo (48 values) in registers, then accumulates all 17
// column lags (544 FMAs per 20 vector shared loads). The four row groups' f32 sums are added in
// shared memory; partials [tile][289][4].
constexpr int kAcfTile = 32, kAcfHalo = 8, kAcfSpan = kAcfTile + 2 * kAcfHalo, kAcfGroups = 4;
constexpr int kAcfThreads = 4 * 17 * kAcfGroups;  // 272

__global__ void __launch_bounds__(kAcfThreads) k_acf(const float* __restrict__ feat, int w, int h,
                                                     float* __restrict__ part) {
    __shared__ __align__(16) float sh[4 * kAcfSpan * kAcfSpan];
    const int x0 = blockIdx.x * kAcfTile, y0 = blockIdx.y * kAcfTile;
    const size_t n = (size_t)w * h;
    for (int k = threadIdx.x; k < kAcfSpan * kAcfSpan; k += blockDim.x) {
        const int gx = x0 - kAcfHalo + k % kAcfSpan, gy = y0 - kAcfHalo + k / kAcfSpan;
        const bool in = gx >= 0 && gy >= 0 && gx < w && gy < h;
        const size_t i = in ? (size_t)gy * w + gx : 0;
#pragma unroll
        for (int p = 0; p < 4; ++p) sh[p * kAcfSpan * kAcfSpan + k] = in ? feat[p * n + i] : 0.0f;
    }
    __syncthreads();
    const int g = threadIdx.x % kAcfGroups, dy = (threadIdx.x / kAcfGroups) % 17, p = threadIdx.x / (kAcfGroups * 17);
    const float* pl = sh + p * kAcfSpan * kAcfSpan;
    float acc[17];
#pragma unroll
    for (int d = 0; d < 17; ++d) acc[d] = 0.f;
    for (int ty = g; ty < kAcfTile; ty += kAcfGroups) {
        float a[32], b[48];
        const float4* ar = reinterpret_cast<const float4*>(pl + (ty + kAcfHalo) * kAcfSpan + kAcfHalo);
        const float4* br = reinterpret_cast<const float4*>(pl + (ty + dy) * kAcfSpan);
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const float4 v = ar[q];
            a[4 * q] = v.x, a[4 * q + 1] = v.y, a[4 * q + 2] = v.z, a[4 * q + 3] = v.w;
        }
#pragma unroll
        for (int q = 0; q < 12; ++q) {
            const float4 v = br[q];
            b[4 * q] = v.x, b[4 * q + 1] = v.y, b[4 * q + 2] = v.z, b[4 * q + 3] = v.w;
        }
#pragma unroll
        for (int d = 0; d < 17; ++d)
#pragma unroll
            for (int x = 0; x < 32; ++x) acc[d] = fmaf(a[x], b[x + d], acc[d]);
    }
    __syncthreads();
    // the row groups' sums: red[g][p·289 + lag] in the (now free) staging array
    float* red = sh;
#pragma unroll
    for (int d = 0; d < 17; ++d) red[g * 1156 + p * 289 + dy * 17 + d] = acc[d];
    __syncthreads();
    const size_t o = (size_t)(blockIdx.y * gridDim.x + blockIdx.x) * 1156;
    for (int k = threadIdx.x; k < 1156; k += blockDim.x) {
        const int lag = k >> 2, pp = k & 3;
        float s = 0.f;
#pragma unroll
        for (int gg = 0; gg < kAcfGroups; ++gg) s += red[gg * 1156 + pp * 289 + lag];
        part[o + k] = s;
    }
}

// Σ over tiles (float64), ÷ the lag's pair count → acf[289][4] (not yet normalised)
__global__ void k_acf_finish(const float* __restrict__ part, int ntiles, int w, int h, double* acf) {
    __shared__ double sh[32];
    const int k = blockIdx.x;  // lag·4 + plane
    double acc = 0.0;
    for (int t = threadIdx.x; t < ntiles; t += blockDim.x) acc += (double)part[(size_t)t * 1156 + k];
    acc = block_sum(acc, sh);
    if (threadIdx.x == 0) {
        const int lag = k / 4, dx = lag % 17 - 8, dy = lag / 17 - 8;
        const double cnt = fmax((double)(w - abs(dx)) * (double)(h - abs(dy)), 1.0);
        acf[k] = (w > abs(dx) && h > abs(dy)) ? acc / cnt : 0.0;
    }
}

// [w, w f0..w f3] with w = 1 (smi.wgsl:608-624)
__global__ void k_stack(const float* __restrict__ feat, int n, float* __restrict__ stack) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        stack[i] = 1.0f;
#pragma unroll
        for (int p = 0; p < 4; ++p) stack[(size_t)(p + 1) * n + i] = feat[(size_t)p * n + i];
    }
}

int grid_for(int n) {
    const int b = (n + kThreads - 1) / kThreads;
    return b < 148 * 8 ? (b > 0 ? b : 1) : 148 * 8;
}

}  // namespace

cudaError_t build_features(float* gray, int w, int h, int mode, bool half, float* rank, float* feat, float* mag,
                           float* stack, FeatScratch& s, cudaStream_t st) {
    const int n = w * h;
    const int gb = grid_for(n);
    cudaMemsetAsync(s.stats, 0, 22 * sizeof(double), st);
    cudaMemsetAsync(s.hist, 0, 256 * sizeof(unsigned), st);
    if (half) k_quant_half<<<gb, kThreads, 0, st>>>(gray, n);
    k_sum<<<gb, kThreads, 0, st>>>(gray, n, s.stats);
    k_sumsq<<<gb, kThreads, 0, st>>>(gray, n, s.stats);
    k_hist<<<gb, kThreads, 0, st>>>(gray, n, s.stats, s.hist);
    k_rank<<<gb, kThreads, 0, st>>>(gray, n, s.stats, s.hist, rank);
    dim3 b2(32, 8), g2((w + 31) / 32, (h + 7) / 8);
    k_feats<<<g2, b2, 0, st>>>(rank, w, h, mode, feat, mag);
    k_featmom<<<grid_for(n) < 296 ? grid_for(n) : 296, kThreads, 0, st>>>(feat, n, s.stats + 2);
    k_chol<<<1, 32, 0, st>>>(s.stats + 2, n, 1e-4f, s.wt);
    k_whiten<<<gb, kThreads, 0, st>>>(feat, n, s.wt);
    k_stack<<<gb, kThreads, 0, st>>>(feat, n, stack);
    return cudaGetLastError();
}

cudaError_t autocorrelation(const float* feat, int w, int h, FeatScratch& s, cudaStream_t st) {
    dim3 ga((w + kAcfTile - 1) / kAcfTile, (h + kAcfTile - 1) / kAcfTile);
    const int ntiles = ga.x * ga.y;
    if ((size_t)ntiles * 1156 > s.acf_part_cap) return cudaErrorInvalidValue;
    k_acf<<<ga, kAcfThreads, 0, st>>>(feat, w, h, s.acf_part);
    k_acf_finish<<<1156, kThreads, 0, st>>>(s.acf_part, ntiles, w, h, s.acf);
    return cudaGetLastError();
}

}  // namespace zc
