// Preprocessing before the features (the reference's Gls.uploadRgba / clahe / bandpass / invert,
// src/gls.zig:411-566, with its kernels in shaders/gls_mift.wgsl rgba_to_gray_buf 283-291,
// gauss_h / gauss_v 293-320, clahe_hist / clahe_cdf / clahe_apply 1975-2057).
//
// The work image holds "texels": with `half` every stored value is rounded to f16, as the
// reference stores its texels, so each step below rounds its output when half is on. Arithmetic
// that decides bins and sums uses IEEE-rounded single operations (no contraction) in the
// reference's order.
#include <cuda_fp16.h>

#include "common.cuh"
#include "kernels.hpp"

namespace zc {
namespace {

__device__ __forceinline__ float texel(float v, bool half) { return half ? __half2float(__float2half_rn(v)) : v; }

// packed RGBA8 → 0.299 R + 0.587 G + 0.114 B with each channel i/255 rounded to f32
__global__ void k_rgba_gray(const uchar4* __restrict__ rgba, int n, float* __restrict__ gray) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uchar4 p = rgba[i];
        const float r = __fdiv_rn((float)p.x, 255.f), g = __fdiv_rn((float)p.y, 255.f), b = __fdiv_rn((float)p.z, 255.f);
        gray[i] = __fadd_rn(__fadd_rn(__fmul_rn(0.299f, r), __fmul_rn(0.587f, g)), __fmul_rn(0.114f, b));
    }
}

struct ClaheGeom {
    int w, h;            // image
    int hg;              // tiles per side
    int nb;              // bins
    int h_pad, w_pad;    // reflected rows / columns added before the image
    int h_tile, w_tile;  // tile size on the padded image
    float clip;          // clip limit (× the mean bin count)
};

__device__ __forceinline__ int clahe_reflect(int i, int n, int pad) {
    int x = i - pad;
    if (n <= 1) return 0;
    if (x < 0) x = -x;
    if (x >= n) x = 2 * n - 2 - x;
    return min(max(x, 0), n - 1);
}

// every padded pixel's bin into its tile's histogram (shared-memory counts, then one add each)
__global__ void __launch_bounds__(256) k_clahe_hist(const float* __restrict__ src, ClaheGeom g,
                                                    unsigned* __restrict__ hist) {
    extern __shared__ unsigned sh[];
    const int nh = g.hg * g.hg * g.nb;
    for (int i = threadIdx.x; i < nh; i += blockDim.x) sh[i] = 0;
    __syncthreads();
    const int pw = g.w + g.w_pad, ph = g.h + g.h_pad;
    const long long total = (long long)pw * ph;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const int y = (int)(i / pw), x = (int)(i - (long long)y * pw);
        const int ox = clahe_reflect(x, g.w, g.w_pad), oy = clahe_reflect(y, g.h, g.h_pad);
        const float v = fminf(fmaxf(src[(size_t)oy * g.w + ox], 0.f), 1.f);
        const float bf = fminf(fmaxf(__fmul_rn(v, (float)(g.nb - 1)), 0.f), (float)(g.nb - 1));
        const int bin = (int)bf;
        const int tile = (y / g.h_tile) * g.hg + x / g.w_tile;
        atomicAdd(&sh[tile * g.nb + bin], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nh; i += blockDim.x)
        if (sh[i]) atomicAdd(&hist[i], sh[i]);
}

// one thread per tile: the clipped histogram, its excess redistributed evenly (the remainder one
// count each to the lowest bins), accumulated into the tile's CDF, in the reference's order
__global__ void k_clahe_cdf(const unsigned* __restrict__ hist, ClaheGeom g, float* __restrict__ cdf) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= g.hg * g.hg) return;
    const int nb = g.nb;
    const unsigned voxels = (unsigned)max(g.h_tile * g.w_tile, 1);
    const float limit = fmaxf(__fdiv_rn(__fmul_rn(g.clip, (float)voxels), (float)nb), 1.f);
    float sumc = 0.f;
    for (int i = 0; i < nb; ++i) sumc = __fadd_rn(sumc, fminf((float)hist[t * nb + i], limit));
    const float clipped = __fsub_rn((float)voxels, sumc);
    const float fnb = (float)nb;
    const int residual = (int)__fsub_rn(clipped, __fmul_rn(fnb, floorf(__fdiv_rn(clipped, fnb))));
    const float redist = __fdiv_rn(__fsub_rn(clipped, (float)residual), fnb);
    const float den = fmaxf((float)voxels, 1.f);
    float acc = 0.f;
    for (int i = 0; i < nb; ++i) {
        float c = __fadd_rn(fminf((float)hist[t * nb + i], limit), redist);
        if (i < residual) c = __fadd_rn(c, 1.f);
        acc = __fadd_rn(acc, c);
        cdf[t * nb + i] = fminf(fmaxf(__fdiv_rn(acc, den), 0.f), 1.f);
    }
}

__device__ __forceinline__ float mixf(float a, float b, float t) { return __fadd_rn(__fmul_rn(a, __fsub_rn(1.f, t)), __fmul_rn(b, t)); }

// each pixel's value through the four nearest tiles' CDFs, blended bilinearly over the tile grid
__global__ void k_clahe_apply(const float* __restrict__ src, ClaheGeom g, const float* __restrict__ cdf, bool half,
                              float* __restrict__ dst) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= g.w || y >= g.h) return;
    const int hg = g.hg, nb = g.nb;
    const float v = fminf(fmaxf(src[(size_t)y * g.w + x], 0.f), 1.f);
    const float gy = __fmul_rn(__fdiv_rn((float)y + 0.5f, (float)g.h), (float)(hg - 1));
    const float gx = __fmul_rn(__fdiv_rn((float)x + 0.5f, (float)g.w), (float)(hg - 1));
    const int y0 = (int)floorf(gy), x0 = (int)floorf(gx);
    const int y1 = min(y0 + 1, hg - 1), x1 = min(x0 + 1, hg - 1);
    const float fy = __fsub_rn(gy, (float)y0), fx = __fsub_rn(gx, (float)x0);
    const float bf = __fmul_rn(v, (float)(nb - 1));
    const int b0 = (int)fminf(fmaxf(floorf(bf), 0.f), (float)(nb - 2));
    const float fb = __fsub_rn(bf, (float)b0);
    const float* c00 = cdf + (y0 * hg + x0) * nb;
    const float* c10 = cdf + (y0 * hg + x1) * nb;
    const float* c01 = cdf + (y1 * hg + x0) * nb;
    const float* c11 = cdf + (y1 * hg + x1) * nb;
    const float a00 = mixf(c00[b0], c00[b0 + 1], fb), a10 = mixf(c10[b0], c10[b0 + 1], fb);
    const float a01 = mixf(c01[b0], c01[b0 + 1], fb), a11 = mixf(c11[b0], c11[b0 + 1], fb);
    dst[(size_t)y * g.w + x] = texel(mixf(mixf(a00, a10, fx), mixf(a01, a11, fx), fy), half);
}

// one pass of the σ = 1 Gaussian (7 taps, clamp to edge) along x (DX) or y
template <bool DX>
__global__ void k_gauss(const float* __restrict__ src, int w, int h, bool half, float* __restrict__ dst) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    float acc = 0.f, wsum = 0.f;
#pragma unroll
    for (int k = -3; k <= 3; ++k) {
        const float ww = expf(__fmul_rn(-0.5f, (float)(k * k)));
        const int xx = DX ? min(max(x + k, 0), w - 1) : x;
        const int yy = DX ? y : min(max(y + k, 0), h - 1);
        acc = __fadd_rn(acc, __fmul_rn(src[(size_t)yy * w + xx], ww));
        wsum = __fadd_rn(wsum, ww);
    }
    dst[(size_t)y * w + x] = texel(__fdiv_rn(acc, wsum), half);
}

// the difference of the fine and coarse blurs, each clamped to [0, 1]; its range into mm (as
// order-preserving keys: [0] smallest, [1] largest)
__device__ __forceinline__ unsigned ord_key(float f) {
    const unsigned u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float ord_float(unsigned k) {
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

__global__ void k_dog(const float* __restrict__ fine, const float* __restrict__ coarse, int n, float* __restrict__ d,
                      unsigned* mm) {
    unsigned lo = 0xffffffffu, hi = 0u;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float v = __fsub_rn(fminf(fmaxf(fine[i], 0.f), 1.f), fminf(fmaxf(coarse[i], 0.f), 1.f));
        d[i] = v;
        const unsigned k = ord_key(v);
        lo = min(lo, k);
        hi = max(hi, k);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(&mm[0], lo);
        atomicMax(&mm[1], hi);
    }
}

// (v − lo)·sc, sc = 1/(hi − lo) (0 for a flat image), as a texel
__global__ void k_dog_rescale(const float* __restrict__ d, int n, const unsigned* mm, bool half, float* __restrict__ out) {
    const float lo = ord_float(mm[0]), hi = ord_float(mm[1]);
    const float sc = hi > lo ? __fdiv_rn(1.f, __fsub_rn(hi, lo)) : 0.f;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        out[i] = texel(__fmul_rn(__fsub_rn(d[i], lo), sc), half);
}

__global__ void k_invert(float* __restrict__ a, int n, bool half) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        a[i] = texel(__fsub_rn(1.f, fminf(fmaxf(a[i], 0.f), 1.f)), half);
}

__global__ void k_texels(float* __restrict__ a, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) a[i] = texel(a[i], true);
}

int grid1(int n) {
    const int b = (n + 255) / 256;
    return b < 148 * 8 ? (b > 0 ? b : 1) : 148 * 8;
}

}  // namespace

cudaError_t rgba_to_gray(const unsigned char* rgba, int n, float* gray, cudaStream_t st) {
    k_rgba_gray<<<grid1(n), 256, 0, st>>>(reinterpret_cast<const uchar4*>(rgba), n, gray);
    return cudaGetLastError();
}

size_t clahe_scratch_bytes(int grid, int bins) {
    const int hg = std::min(8, std::max(2, grid)), nb = std::min(256, std::max(8, bins));
    return (size_t)hg * hg * nb * (sizeof(unsigned) + sizeof(float));
}

cudaError_t clahe(const float* src, int w, int h, double clip, int bins, int grid, bool half, void* scratch,
                  float* dst, cudaStream_t st) {
    ClaheGeom g;
    g.w = w, g.h = h;
    g.hg = std::min(8, std::max(2, grid));
    g.nb = std::min(256, std::max(8, bins));
    g.h_pad = (g.hg - h % g.hg) % g.hg;
    g.w_pad = (g.hg - w % g.hg) % g.hg;
    g.h_tile = std::max(1, (h + g.h_pad) / g.hg);
    g.w_tile = std::max(1, (w + g.w_pad) / g.hg);
    g.clip = (float)clip;
    const int nh = g.hg * g.hg * g.nb;
    unsigned* hist = static_cast<unsigned*>(scratch);
    float* cdf = reinterpret_cast<float*>(hist + nh);
    cudaError_t e = cudaMemsetAsync(hist, 0, (size_t)nh * sizeof(unsigned), st);
    if (e != cudaSuccess) return e;
    const size_t sm = (size_t)nh * sizeof(unsigned);
    cudaFuncSetAttribute(k_clahe_hist, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_clahe_hist<<<grid1((w + g.w_pad) * (h + g.h_pad)), 256, sm, st>>>(src, g, hist);
    k_clahe_cdf<<<1, 64, 0, st>>>(hist, g, cdf);
    dim3 b(32, 8), gg((w + 31) / 32, (h + 7) / 8);
    k_clahe_apply<<<gg, b, 0, st>>>(src, g, cdf, half, dst);
    return cudaGetLastError();
}

cudaError_t gauss_blur(const float* src, int w, int h, bool half, float* tmp, float* dst, cudaStream_t st) {
    dim3 b(32, 8), g((w + 31) / 32, (h + 7) / 8);
    k_gauss<true><<<g, b, 0, st>>>(src, w, h, half, tmp);
    k_gauss<false><<<g, b, 0, st>>>(tmp, w, h, half, dst);
    return cudaGetLastError();
}

cudaError_t dog_rescale(const float* fine, const float* coarse, int n, bool half, float* d, unsigned* mm, float* out,
                        cudaStream_t st) {
    const unsigned init[2] = {0xffffffffu, 0u};
    cudaError_t e = cudaMemcpyAsync(mm, init, sizeof init, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return e;
    k_dog<<<grid1(n), 256, 0, st>>>(fine, coarse, n, d, mm);
    k_dog_rescale<<<grid1(n), 256, 0, st>>>(d, n, mm, half, out);
    return cudaGetLastError();
}

cudaError_t invert_texels(float* a, int n, bool half, cudaStream_t st) {
    k_invert<<<grid1(n), 256, 0, st>>>(a, n, half);
    return cudaGetLastError();
}

cudaError_t round_texels(float* a, int n, cudaStream_t st) {
    k_texels<<<grid1(n), 256, 0, st>>>(a, n);
    return cudaGetLastError();
}

}  // namespace zc
