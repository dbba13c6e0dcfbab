// The roto-scale (log-polar) map's own kernels (the reference's shaders/smi.wgsl
// spatial_logpolar 1434-1452 and rs_finish 1708-1731); its correlations and score are the shift
// map's passes on the log-polar planes, with each row's sums scaled to dest area.
#include "common.cuh"
#include "kernels.hpp"

namespace zc {
namespace {

// One thread per log-polar cell (θ index x < n_θ, log-radius index y < n_λ): the canvas stack
// (5 planes, W × Hh) sampled bilinearly at (cx + ρ cos θ, cy + ρ sin θ), ρ = e^{log0 + (y + ½)/n_λ ·
// span}, θ = (x + ½)/n_θ · 2π, zero where the 2×2 footprint leaves the canvas; each sample times
// ρ, the area weight the correlations integrate with (smi.wgsl pack_pair, theme 1). Output
// plane-major [5][n_λ][n_θ].
__global__ void k_logpolar(const float* __restrict__ canvas, int W, int Hh, float cx, float cy, float log0,
                           float span, int n_th, int n_lam, float* __restrict__ grid) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= n_th || y >= n_lam) return;
    const float t = ((float)y + 0.5f) / (float)max(n_lam, 1);
    const float rho = expf(log0 + t * span);
    const float th = ((float)x + 0.5f) / (float)n_th * 6.28318530718f;
    const float xs = cx + rho * cosf(th), ys = cy + rho * sinf(th);
    const float flx = floorf(xs), fly = floorf(ys);
    const size_t cn = (size_t)W * Hh, gn = (size_t)n_th * n_lam, o = (size_t)y * n_th + x;
    // x0 ≥ 0, x0 + 1 < W (NaN fails), checked before any float → int conversion
    const bool ok = flx >= 0.f && fly >= 0.f && flx < (float)(W - 1) && fly < (float)(Hh - 1);
    if (!ok) {
#pragma unroll
        for (int p = 0; p < 5; ++p) grid[p * gn + o] = 0.f;
        return;
    }
    const int x0 = (int)flx, y0 = (int)fly;
    const float fx = xs - flx, fy = ys - fly;
    const size_t i00 = (size_t)y0 * W + x0;
#pragma unroll
    for (int p = 0; p < 5; ++p) {
        const float* c = canvas + p * cn;
        const float a = c[i00] + (c[i00 + 1] - c[i00]) * fx;
        const float b = c[i00 + W] + (c[i00 + W + 1] - c[i00 + W]) * fx;
        grid[p * gn + o] = (a + (b - a) * fy) * rho;
    }
}

// Per cell t of the n × n map: the forward map, averaged with the inverse-frame map at the
// mirrored lag (−y, −x), or (−y, x) for a reflecting pose, when there is one; rows whose applied
// scale e^{−kΔλ} lies outside [e^lo, e^hi] zeroed; the first-index argmax key into *best and the
// cell at lag 0 into *zero.
__global__ void k_rs_finish(const float* __restrict__ fwd, const float* __restrict__ inv, int mirror, int n,
                            float dlam, float lo, float hi, float* __restrict__ out, unsigned long long* best,
                            float* zero) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long key = 0ull;
    if (t < n * n) {
        const int y = t / n, x = t - y * n;
        float v = fwd[t];
        if (inv) {
            const int ym = (n - y) % n, xm = mirror ? (n - x) % n : x;
            v = 0.5f * (v + inv[ym * n + xm]);
        }
        const float k = y > n / 2 ? (float)(y - n) : (float)y;
        const float sg = -k * dlam;
        if (sg < lo || sg > hi) v = 0.f;
        out[t] = v;
        if (t == 0) *zero = v;
        key = argmax_key(v, (uint32_t)t);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long other = __shfl_xor_sync(0xffffffffu, key, o);
        key = other > key ? other : key;
    }
    if ((threadIdx.x & 31) == 0 && key) atomicMax(best, key);
}

}  // namespace

cudaError_t rs_logpolar(const float* canvas, int W, int Hh, float cx, float cy, float log0, float span, int n_th,
                        int n_lam, float* grid, cudaStream_t st) {
    dim3 b(32, 8), g((n_th + 31) / 32, (n_lam + 7) / 8);
    k_logpolar<<<g, b, 0, st>>>(canvas, W, Hh, cx, cy, log0, span, n_th, n_lam, grid);
    return cudaGetLastError();
}

cudaError_t rs_finish(const float* fwd, const float* inv, bool mirror, int n, float dlam, float lo, float hi,
                      float* out, unsigned long long* best, float* zero, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(best, 0, sizeof(unsigned long long), st);
    if (e != cudaSuccess) return e;
    const int nn = n * n;
    k_rs_finish<<<(nn + 255) / 256, 256, 0, st>>>(fwd, inv, mirror ? 1 : 0, n, dlam, lo, hi, out, best, zero);
    return cudaGetLastError();
}

}  // namespace zc
