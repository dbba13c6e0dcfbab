// The rotation × scale sweep's own kernels (the reference's shaders/sweep.wgsl): the stacks
// interleaved per pixel, each candidate's window of canvas cells packed from k×k bilinear taps
// together with its zero-lag overlap, and the peaks of each candidate's map. The transforms and
// the per-shift score between them are the shift map's kernels (shiftmap.cu), batched over
// candidates.
#include "common.cuh"
#include "kernels.hpp"

namespace zc {
namespace {

// plane-major [5][n] → n float4 (w, w f0, w f1, w f2), then the fifth plane (w f3) as n floats:
// a bilinear tap is one 16-byte load per corner plus a scalar from a plane eight pixels to a
// sector (sweep.wgsl interleave)
__global__ void k_interleave(const float* __restrict__ stack, int n, float4* __restrict__ il) {
    float* p4 = reinterpret_cast<float*>(il + n);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        il[i] = make_float4(stack[i], stack[(size_t)n + i], stack[2 * (size_t)n + i], stack[3 * (size_t)n + i]);
        p4[i] = stack[4 * (size_t)n + i];
    }
}

// Warp w of a block takes the 32 cells x0 .. x0 + 31 of row y of item z's window; the item's
// pose is poses[(slot0 + z)·12 ..]: the dest → source map (row-major 3×3, 1-based pixels), taps
// per side, the window's first canvas cell. The cell's value is the mean of k×k bilinear taps of
// the source stack at the cell's sub-points (sweep.wgsl tap, pack_sweep); a tap whose 2×2
// footprint leaves the image adds nothing. Cells past the G×G canvas are zero. Output plane-major
// [5][win_y][win_x] per item. The taps run across the lanes: in each pass, groups of k lanes take
// ⌊32/k⌋ cells, lane (g, tx) summing tap column tx of its cell over the k tap rows, so adjacent
// lanes read adjacent pixels (one cache line serves several lanes) instead of pixels a cell apart;
// each group's k column sums are then added across its lanes and handed to the lane that owns
// the cell. With fixed weights fw ([Fy][Fx], the fixed window at canvas cell (fx0, fy0)) the
// item's zero-lag overlap Σ w_moving · w_fixed over the cells both windows cover accumulates into
// n0[z] (sweep.wgsl zero_lag reads the same value off the correlation of the weight planes).
__global__ void __launch_bounds__(256) k_sweep_pack(const float4* __restrict__ il, int sw, int sh,
                                                    const float* __restrict__ poses, int slot0, int win_x, int win_y,
                                                    SweepCanvas cv, const float* __restrict__ fw, int fx0, int fy0,
                                                    int Fx, int Fy, float* __restrict__ grid, double* __restrict__ n0) {
    const int lane = threadIdx.x & 31;
    const int x0 = blockIdx.x * 32, y = blockIdx.y * 8 + (threadIdx.x >> 5), z = blockIdx.z;
    const float* P = poses + (size_t)(slot0 + z) * 12;
    const int cy = (int)P[11] + y;
    const int x = x0 + lane;
    const bool in_win = x < win_x && y < win_y;
    const int k = min(max((int)P[9], 1), 32), cpw = 32 / k;
    const float* p4 = reinterpret_cast<const float*>(il + (size_t)sw * sh);  // the fifth plane
    const float h0 = P[0], h1 = P[1], h2 = P[2], h3 = P[3], h4 = P[4], h5 = P[5], h6 = P[6], h7 = P[7], h8 = P[8];
    const float inv = 1.f / (float)(k * k);
    const int grp = lane / k, tx = lane - grp * k;
    float s[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
    for (int c0 = 0; c0 < 32; c0 += cpw) {
        const int xw = x0 + c0 + grp, cx = (int)P[10] + xw;
        const bool act = grp < cpw && c0 + grp < 32 && xw < win_x && y < win_y && cx < cv.G && cy < cv.G;
        float4 a = make_float4(0.f, 0.f, 0.f, 0.f);
        float a4 = 0.f;
        if (act) {
            const float px = cv.ox + ((float)cx + ((float)tx + 0.5f) / (float)k) * cv.cell;
            for (int ty = 0; ty < k; ++ty) {
                const float py = cv.oy + ((float)cy + ((float)ty + 0.5f) / (float)k) * cv.cell;
                const float qx = h0 * px + h1 * py + h2;
                const float qy = h3 * px + h4 * py + h5;
                const float qz = h6 * px + h7 * py + h8;
                if (fabsf(qz) < 1e-8f) continue;
                // affine poses (qz = 1): the division is exact, skip it
                const float fx = (qz == 1.f ? qx : qx / qz) - 1.0f, fy = (qz == 1.f ? qy : qy / qz) - 1.0f;
                const float flx = floorf(fx), fly = floorf(fy);
                // x0 ≥ 0 and x0 + 1 < w (NaN fails both), before any float → int conversion
                if (!(flx >= 0.f && fly >= 0.f && flx < (float)(sw - 1) && fly < (float)(sh - 1))) continue;
                const int ix = (int)flx, iy = (int)fly;
                const float ax = fx - flx, ay = fy - fly;
                const float w00 = (1.f - ax) * (1.f - ay), w10 = ax * (1.f - ay), w01 = (1.f - ax) * ay, w11 = ax * ay;
                const size_t i00 = (size_t)iy * sw + ix, i01 = i00 + sw;
                const float4 p00 = __ldg(&il[i00]), p10 = __ldg(&il[i00 + 1]);
                const float4 p01 = __ldg(&il[i01]), p11 = __ldg(&il[i01 + 1]);
                a.x += w00 * p00.x + w10 * p10.x + w01 * p01.x + w11 * p11.x;
                a.y += w00 * p00.y + w10 * p10.y + w01 * p01.y + w11 * p11.y;
                a.z += w00 * p00.z + w10 * p10.z + w01 * p01.z + w11 * p11.z;
                a.w += w00 * p00.w + w10 * p10.w + w01 * p01.w + w11 * p11.w;
                a4 += w00 * __ldg(&p4[i00]) + w10 * __ldg(&p4[i00 + 1]) + w01 * __ldg(&p4[i01]) +
                      w11 * __ldg(&p4[i01 + 1]);
            }
        }
        // the group's k column sums, added in every lane of the group (k is the same for the warp)
        float t[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
        for (int j = 0; j < k; ++j) {
            const int src = min(grp * k + j, 31);
            t[0] += __shfl_sync(0xffffffffu, a.x, src);
            t[1] += __shfl_sync(0xffffffffu, a.y, src);
            t[2] += __shfl_sync(0xffffffffu, a.z, src);
            t[3] += __shfl_sync(0xffffffffu, a.w, src);
            t[4] += __shfl_sync(0xffffffffu, a4, src);
        }
        // lane L owns strip cell L: this pass holds it when c0 ≤ L < c0 + cpw, in group L − c0
        const int mine = lane - c0;
        const bool here = mine >= 0 && mine < cpw;
        const int src = here ? mine * k : 0;
#pragma unroll
        for (int p = 0; p < 5; ++p) {
            const float v = __shfl_sync(0xffffffffu, t[p], src);
            if (here) s[p] = v * inv;
        }
    }
    if (in_win) {
        const size_t wn = (size_t)win_x * win_y;
        float* g = grid + (size_t)z * 5 * wn + (size_t)y * win_x + x;
#pragma unroll
        for (int p = 0; p < 5; ++p) g[p * wn] = s[p];
    }
    if (!n0) return;
    double v = 0.0;
    if (in_win) {
        const int fx = (int)P[10] + x - fx0, fy = cy - fy0;
        if (fx >= 0 && fy >= 0 && fx < Fx && fy < Fy) v = (double)s[0] * (double)__ldg(&fw[(size_t)fy * Fx + fx]);
    }
    __shared__ double red[32];
    v = block_sum(v, red);
    if (threadIdx.x == 0 && v != 0.0) atomicAdd(&n0[z], v);
}

// One block per item (sweep.wgsl peaks_sweep): lane l < 256 keeps the best 3×3 local maximum
// (periodic, > 0, the first of equal ones) among the shifts t ≡ l (mod 256); the n_peak best lanes
// (equal scores: the lower lane first) are written to slot (slot0 + z) as (score, index), and
// (0, 0xffffffff) where fewer lanes found one. The block's 1024 threads scan each lane's shifts
// four ways (thread (l, q) the shifts l + 256·(q + 4j)) and merge the four bests per lane by the
// same rule (higher score, then lower shift), which is the lane's own best.
__global__ void __launch_bounds__(1024) k_sweep_peaks(const float* __restrict__ maps, int nx, int ny, size_t mstride,
                                                      int n_peak, int slot0, float* __restrict__ ps,
                                                      uint32_t* __restrict__ pi) {
    const float* m = maps + (size_t)blockIdx.x * mstride;
    const int nn = nx * ny;
    const int l = threadIdx.x & 255, q = threadIdx.x >> 8;
    float bv = 0.f;
    uint32_t bi = 0xffffffffu;
    for (int t = l + 256 * q; t < nn; t += 1024) {
        const float v = __ldg(&m[t]);
        if (v <= bv) continue;
        const int y = t / nx, x = t - y * nx;
        const int ym = (y + ny - 1) % ny, yp = (y + 1) % ny, xm = (x + nx - 1) % nx, xp = (x + 1) % nx;
        const bool ok = !(__ldg(&m[ym * nx + xm]) > v || __ldg(&m[ym * nx + x]) > v || __ldg(&m[ym * nx + xp]) > v ||
                          __ldg(&m[y * nx + xm]) > v || __ldg(&m[y * nx + xp]) > v || __ldg(&m[yp * nx + xm]) > v ||
                          __ldg(&m[yp * nx + x]) > v || __ldg(&m[yp * nx + xp]) > v);
        if (ok) {
            bv = v;
            bi = (uint32_t)t;
        }
    }
    __shared__ float sv[3][256];
    __shared__ uint32_t si[3][256];
    if (q > 0) {
        sv[q - 1][l] = bv;
        si[q - 1][l] = bi;
    }
    __syncthreads();
    if (q == 0)
        for (int r = 0; r < 3; ++r) {
            const float v = sv[r][l];
            const uint32_t i = si[r][l];
            if (v > bv || (v == bv && i < bi)) {
                bv = v;
                bi = i;
            }
        }
    // a positive float's bits order like the float: (score, inverted lane) as one key
    unsigned long long key = (q > 0 || bi == 0xffffffffu)
                                 ? 0ull
                                 : ((unsigned long long)__float_as_uint(bv) << 32) | (0xffffffffu - (uint32_t)l);
    __shared__ unsigned long long wmax[32];
    __shared__ unsigned long long top;
    for (int k = 0; k < n_peak; ++k) {
        unsigned long long w = key;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long other = __shfl_xor_sync(0xffffffffu, w, o);
            w = other > w ? other : w;
        }
        if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = w;
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned long long b = 0;
            for (int i = 0; i < 32; ++i) b = wmax[i] > b ? wmax[i] : b;
            top = b;
        }
        __syncthreads();
        const unsigned long long b = top;
        const size_t o = (size_t)(slot0 + blockIdx.x) * n_peak + k;
        if (b == 0ull) {
            if (threadIdx.x == 0) {
                ps[o] = 0.f;
                pi[o] = 0xffffffffu;
            }
        } else if (b == key) {
            ps[o] = bv;
            pi[o] = bi;
            key = 0ull;
        }
        __syncthreads();
    }
}

}  // namespace

cudaError_t sweep_interleave(const float* stack, int n, float4* il, cudaStream_t st) {
    int blocks = (n + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_interleave<<<blocks, 256, 0, st>>>(stack, n, il);
    return cudaGetLastError();
}

cudaError_t sweep_pack(const float4* il, int sw, int sh, const float* poses, int slot0, int batch, int win_x,
                       int win_y, const SweepCanvas& cv, const float* fw, int fx0, int fy0, int Fx, int Fy, float* grid,
                       double* n0, cudaStream_t st) {
    if (n0) {
        const cudaError_t e = cudaMemsetAsync(n0, 0, (size_t)batch * sizeof(double), st);
        if (e != cudaSuccess) return e;
    }
    dim3 g((win_x + 31) / 32, (win_y + 7) / 8, batch);
    k_sweep_pack<<<g, 256, 0, st>>>(il, sw, sh, poses, slot0, win_x, win_y, cv, fw, fx0, fy0, Fx, Fy, grid, n0);
    return cudaGetLastError();
}

cudaError_t sweep_peaks(const float* maps, int nx, int ny, size_t map_stride, int batch, int n_peak, int slot0,
                        float* ps, uint32_t* pi, cudaStream_t st) {
    k_sweep_peaks<<<batch, 1024, 0, st>>>(maps, nx, ny, map_stride, n_peak, slot0, ps, pi);
    return cudaGetLastError();
}

}  // namespace zc
