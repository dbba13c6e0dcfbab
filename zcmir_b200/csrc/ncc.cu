// The NCC overlay metric's own kernels (the reference's src/overlay.zig:130-305 with
// shaders/ncc.wgsl): the pair's union canvas at a pose (the moving work image warped, the fixed
// one pasted), its zero-lag normalised cross-correlation, and the mean-free resampled planes the
// NCC shift map correlates. The correlation itself runs on the shift map's FFT passes (one real
// plane per side, one correlation, the NCC combine).
#include <cuda_fp16.h>

#include "common.cuh"
#include "kernels.hpp"

namespace zc {
namespace {

struct Mat9 {
    float m[9];
};

__device__ __forceinline__ float texel_of(float v, int half) { return half ? __half2float(__float2half_rn(v)) : v; }

// The canvas pixel (x, y) of both sides (src/overlay.zig:144-157 assemble): the moving work image
// through the canvas pose's inverse hi, bilinear, 0 where the source point leaves the image
// (gls_mift.wgsl:1921-1956 warp_homography), stored as a texel; the fixed work image at (x + ox,
// y + oy), 0 outside it (paste_rect 1959-1969).
__device__ __forceinline__ float2 canvas_px(const float* __restrict__ mv, int w, int h, const Mat9& hi, int ok_det,
                                            const float* __restrict__ fx, int fw, int fh, int ox, int oy, int half,
                                            int x, int y) {
    float a = 0.f;
    if (ok_det) {
        const float X = (float)x + 1.0f, Y = (float)y + 1.0f;
        const float qx = hi.m[0] * X + hi.m[1] * Y + hi.m[2];
        const float qy = hi.m[3] * X + hi.m[4] * Y + hi.m[5];
        const float qz = hi.m[6] * X + hi.m[7] * Y + hi.m[8];
        if (fabsf(qz) >= 1e-8f) {
            const float sx = qx / qz - 1.0f, sy = qy / qz - 1.0f;
            if (!(sx < 0.f || sy < 0.f || sx > (float)(w - 1) || sy > (float)(h - 1))) {
                const float flx = floorf(sx), fly = floorf(sy);
                const float tx = sx - flx, ty = sy - fly;
                const int x0 = min(max((int)flx, 0), w - 1), y0 = min(max((int)fly, 0), h - 1);
                const int x1 = min(x0 + 1, w - 1), y1 = min(y0 + 1, h - 1);
                const float v00 = mv[(size_t)y0 * w + x0], v10 = mv[(size_t)y0 * w + x1];
                const float v01 = mv[(size_t)y1 * w + x0], v11 = mv[(size_t)y1 * w + x1];
                const float p = v00 * (1.f - tx) + v10 * tx, q = v01 * (1.f - tx) + v11 * tx;
                a = texel_of(p * (1.f - ty) + q * ty, half);
            }
        }
    }
    const int sx = x + ox, sy = y + oy;
    const float b = (sx >= 0 && sy >= 0 && sx < fw && sy < fh) ? fx[(size_t)sy * fw + sx] : 0.f;
    return make_float2(a, b);
}

// Both canvas planes, written (one thread per pixel).
__global__ void k_ncc_canvas(const float* __restrict__ mv, int w, int h, Mat9 hi, int ok_det,
                             const float* __restrict__ fx, int fw, int fh, int ox, int oy, int half, int W, int Hh,
                             float* __restrict__ ca, float* __restrict__ cb) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= Hh) return;
    const float2 v = canvas_px(mv, w, h, hi, ok_det, fx, fw, fh, ox, oy, half, x, y);
    ca[(size_t)y * W + x] = v.x;
    cb[(size_t)y * W + x] = v.y;
}

// The five zero-lag moments Σa, Σb, Σa², Σb², Σab over the whole canvas in float64, without
// writing it (ncc.wgsl moments): grid-stride over pixels, block sums, one atomic per block.
__global__ void __launch_bounds__(256) k_ncc_moments(const float* __restrict__ mv, int w, int h, Mat9 hi, int ok_det,
                                                     const float* __restrict__ fx, int fw, int fh, int ox, int oy,
                                                     int half, int W, int Hh, double* __restrict__ mom) {
    __shared__ double sh[32];
    double s[5] = {0, 0, 0, 0, 0};
    const size_t n = (size_t)W * Hh;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int y = (int)(i / W), x = (int)(i - (size_t)y * W);
        const float2 v = canvas_px(mv, w, h, hi, ok_det, fx, fw, fh, ox, oy, half, x, y);
        const double a = v.x, b = v.y;
        s[0] += a;
        s[1] += b;
        s[2] += a * a;
        s[3] += b * b;
        s[4] += a * b;
    }
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        const double t = block_sum(s[k], sh);
        if (threadIdx.x == 0) atomicAdd(&mom[k], t);
    }
}

// The canvas resampled onto the cw × ch correlation grid (ncc.wgsl pack): cell (x, y) is the
// bilinear sample, clamped to the canvas edge, at ((x + ½)·W/cw, (y + ½)·Hh/ch) in pixel-centre
// units; written to plane 0 of each side's grid, Σ per side into sums[0..1].
__global__ void __launch_bounds__(256) k_ncc_pack(const float* __restrict__ ca, const float* __restrict__ cb, int W,
                                                  int Hh, int cw, int ch, float* __restrict__ ga, float* __restrict__ gb,
                                                  double* __restrict__ sums) {
    __shared__ double sh[32];
    double sa = 0, sb = 0;
    const int n = cw * ch;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int gy = i / cw, gx = i - gy * cw;
        const float px = ((float)gx + 0.5f) * (float)W / (float)max(cw, 1) - 0.5f;
        const float py = ((float)gy + 0.5f) * (float)Hh / (float)max(ch, 1) - 0.5f;
        const float flx = floorf(px), fly = floorf(py);
        const float tx = px - flx, ty = py - fly;
        const int x0 = min(max((int)flx, 0), W - 1), x1 = min(max((int)flx + 1, 0), W - 1);
        const int y0 = min(max((int)fly, 0), Hh - 1), y1 = min(max((int)fly + 1, 0), Hh - 1);
        const size_t r0 = (size_t)y0 * W, r1 = (size_t)y1 * W;
        const float a = (ca[r0 + x0] * (1.f - tx) + ca[r0 + x1] * tx) * (1.f - ty) +
                        (ca[r1 + x0] * (1.f - tx) + ca[r1 + x1] * tx) * ty;
        const float b = (cb[r0 + x0] * (1.f - tx) + cb[r0 + x1] * tx) * (1.f - ty) +
                        (cb[r1 + x0] * (1.f - tx) + cb[r1 + x1] * tx) * ty;
        ga[i] = a;
        gb[i] = b;
        sa += a;
        sb += b;
    }
    const double ta = block_sum(sa, sh), tb = block_sum(sb, sh);
    if (threadIdx.x == 0) {
        atomicAdd(&sums[0], ta);
        atomicAdd(&sums[1], tb);
    }
}

// The grid planes made mean-free in place (the mean rounded to f32 as the reference's pack takes
// it), Σ v² per side into sums[2..3].
__global__ void __launch_bounds__(256) k_ncc_center(float* __restrict__ ga, float* __restrict__ gb, int n,
                                                    double* __restrict__ sums) {
    __shared__ double sh[32];
    const float ma = (float)(sums[0] / (double)n), mb = (float)(sums[1] / (double)n);
    double qa = 0, qb = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float a = ga[i] - ma, b = gb[i] - mb;
        ga[i] = a;
        gb[i] = b;
        qa += (double)a * a;
        qb += (double)b * b;
    }
    const double ta = block_sum(qa, sh), tb = block_sum(qb, sh);
    if (threadIdx.x == 0) {
        atomicAdd(&sums[2], ta);
        atomicAdd(&sums[3], tb);
    }
}

// ‖a‖·‖b‖ floored at 1e-12: the map's denominator, where the score pass reads it.
__global__ void k_ncc_den(const double* __restrict__ sums, double* __restrict__ den) {
    *den = fmax(sqrt(fmax(sums[2], 0.0)) * sqrt(fmax(sums[3], 0.0)), 1e-12);
}

Mat9 mat9(const float hi[9]) {
    Mat9 m;
    for (int i = 0; i < 9; ++i) m.m[i] = hi[i];
    return m;
}

int blocks_for(size_t n, int threads) {
    return (int)std::min<size_t>((n + threads - 1) / threads, 148 * 8);
}

}  // namespace

cudaError_t ncc_canvas(const float* mv, int w, int h, const float hi[9], bool ok, const float* fx, int fw, int fh, int ox,
                       int oy, bool half, int W, int Hh, float* ca, float* cb, cudaStream_t st) {
    const dim3 b(32, 8), g((W + 31) / 32, (Hh + 7) / 8);
    k_ncc_canvas<<<g, b, 0, st>>>(mv, w, h, mat9(hi), ok ? 1 : 0, fx, fw, fh, ox, oy, half ? 1 : 0, W, Hh, ca, cb);
    return cudaGetLastError();
}

cudaError_t ncc_moments(const float* mv, int w, int h, const float hi[9], bool ok, const float* fx, int fw, int fh,
                        int ox, int oy, bool half, int W, int Hh, double* mom, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(mom, 0, 5 * sizeof(double), st);
    if (e != cudaSuccess) return e;
    k_ncc_moments<<<blocks_for((size_t)W * Hh, 256), 256, 0, st>>>(mv, w, h, mat9(hi), ok ? 1 : 0, fx, fw, fh, ox, oy,
                                                                    half ? 1 : 0, W, Hh, mom);
    return cudaGetLastError();
}

cudaError_t ncc_grid(const float* ca, const float* cb, int W, int Hh, int cw, int ch, float* ga, float* gb,
                     double* sums, double* den, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(sums, 0, 4 * sizeof(double), st);
    if (e != cudaSuccess) return e;
    const int n = cw * ch, nb = blocks_for((size_t)n, 256);
    k_ncc_pack<<<nb, 256, 0, st>>>(ca, cb, W, Hh, cw, ch, ga, gb, sums);
    k_ncc_center<<<nb, 256, 0, st>>>(ga, gb, n, sums);
    k_ncc_den<<<1, 1, 0, st>>>(sums, den);
    return cudaGetLastError();
}

}  // namespace zc
