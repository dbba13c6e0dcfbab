// The SMI shift map on the GPU (the reference's Smi.shiftMap, src/smi.zig:540-572, with its
// kernels in shaders/smi.wgsl:626-931, 1597-1706).
//
// Pipeline for one map (nx × ny FFT grid, cw × ch correlation grid, P real planes, C
// correlations):
//   1. canvas: the moving stack warped by the canvas pose, the fixed stack pasted
//      (warp_stack / paste_stack), then resampled to the grid when the map is coarser.
//   2. forward_rows / forward_cols (per side): the P real planes are formed on the fly from the
//      5 stack values, two per complex row, row-FFT'd (rows < ch only), unpacked into P half
//      spectra (columns 0..nx/2), then column-FFT'd (rows ≥ ch are zero).
//   3. inverse_columns: per correlation and column tile, A·conj(B) and the inverse column FFT.
//   4. inverse_rows_score: per row, correlations paired as c1 + i·c2 on the Hermitian full row,
//      inverse row FFT, and the per-shift score in float64 with its argmax, without writing a
//      correlation plane to memory. Rows longer than shared memory holds for all C correlations
//      are split S ways by one decimation-in-frequency step (output shifts x ≡ s mod S).
#include "combine.cuh"
#include "common.cuh"
#include "kernels.hpp"

namespace zc {
namespace {

// ── canvas (smi.wgsl:1655-1706) ──────────────────────────────────────────────────────────────

struct Mat9f {
    float m[9];
};

__global__ void k_warp_stack(const float* __restrict__ stack, int w, int h, Mat9f hi, int ok_det, int W, int Hh,
                             float* __restrict__ canvas) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= Hh) return;
    const size_t n = (size_t)W * Hh, pix = (size_t)y * W + x, sn = (size_t)w * h;
    bool ok = ok_det != 0;
    float fx = 0.f, fy = 0.f;
    if (ok) {
        const float X = (float)x + 1.0f, Y = (float)y + 1.0f;
        const float qx = hi.m[0] * X + hi.m[1] * Y + hi.m[2];
        const float qy = hi.m[3] * X + hi.m[4] * Y + hi.m[5];
        const float qz = hi.m[6] * X + hi.m[7] * Y + hi.m[8];
        ok = fabsf(qz) >= 1e-8f;
        if (ok) {
            fx = qx / qz - 1.0f;
            fy = qy / qz - 1.0f;
            ok = !(fx < 0.f || fy < 0.f || fx > (float)(w - 1) || fy > (float)(h - 1));
        }
    }
    int x0 = 0, y0 = 0, x1 = 0, y1 = 0;
    float tx = 0.f, ty = 0.f;
    if (ok) {
        const float flx = floorf(fx), fly = floorf(fy);
        tx = fx - flx;
        ty = fy - fly;
        x0 = min(max((int)flx, 0), w - 1);
        y0 = min(max((int)fly, 0), h - 1);
        x1 = min(max((int)flx + 1, 0), w - 1);
        y1 = min(max((int)fly + 1, 0), h - 1);
    }
#pragma unroll
    for (int p = 0; p < 5; ++p) {
        float v = 0.f;
        if (ok) {
            const float* s = stack + p * sn;
            const float v00 = s[(size_t)y0 * w + x0], v10 = s[(size_t)y0 * w + x1];
            const float v01 = s[(size_t)y1 * w + x0], v11 = s[(size_t)y1 * w + x1];
            const float a = v00 * (1.f - tx) + v10 * tx, b = v01 * (1.f - tx) + v11 * tx;
            v = a * (1.f - ty) + b * ty;
        }
        canvas[p * n + pix] = v;
    }
}

__global__ void k_paste_stack(const float* __restrict__ stack, int w, int h, int ox, int oy, int W, int Hh,
                              float* __restrict__ canvas) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= Hh) return;
    const size_t n = (size_t)W * Hh, pix = (size_t)y * W + x, sn = (size_t)w * h;
    const int sx = x + ox, sy = y + oy;
    const bool in = sx >= 0 && sy >= 0 && sx < w && sy < h;
#pragma unroll
    for (int p = 0; p < 5; ++p) canvas[p * n + pix] = in ? stack[p * sn + (size_t)sy * w + sx] : 0.f;
}

// k×k box of bilinear taps per cell (smi.wgsl:626-639, 675-705)
__global__ void k_resample(const float* __restrict__ canvas, int W, int Hh, int cw, int ch, float* __restrict__ grid) {
    const int gx = blockIdx.x * blockDim.x + threadIdx.x, gy = blockIdx.y * blockDim.y + threadIdx.y;
    if (gx >= cw || gy >= ch) return;
    const float fx = (float)W / (float)max(cw, 1), fy = (float)Hh / (float)max(ch, 1);
    const int kx = (int)fminf(fmaxf(ceilf(fx - 1e-4f), 1.f), 8.f);
    const int ky = (int)fminf(fmaxf(ceilf(fy - 1e-4f), 1.f), 8.f);
    const size_t n = (size_t)W * Hh, gn = (size_t)cw * ch;
    float s[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
    for (int j = 0; j < ky; ++j) {
        const float py = ((float)gy + ((float)j + 0.5f) / (float)ky) * fy - 0.5f;
        const float fly = floorf(py);
        const float ay = py - fly;
        const int ya = min(max((int)fly, 0), Hh - 1), yb = min(max((int)fly + 1, 0), Hh - 1);
        for (int i = 0; i < kx; ++i) {
            const float px = ((float)gx + ((float)i + 0.5f) / (float)kx) * fx - 0.5f;
            const float flx = floorf(px);
            const float ax = px - flx;
            const int xa = min(max((int)flx, 0), W - 1), xb = min(max((int)flx + 1, 0), W - 1);
#pragma unroll
            for (int p = 0; p < 5; ++p) {
                const float* c = canvas + p * n;
                const float a = c[(size_t)ya * W + xa] * (1.f - ax) + c[(size_t)ya * W + xb] * ax;
                const float b = c[(size_t)yb * W + xa] * (1.f - ax) + c[(size_t)yb * W + xb] * ax;
                s[p] += a * (1.f - ay) + b * ay;
            }
        }
    }
    const float inv = 1.f / (float)(kx * ky);
#pragma unroll
    for (int p = 0; p < 5; ++p) grid[p * gn + (size_t)gy * cw + gx] = s[p] * inv;
}

__global__ void k_lag0(const float* __restrict__ a, const float* __restrict__ b, int n, double* out) {
    __shared__ double sh[32];
    double acc = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        acc += (double)a[i] * (double)b[i];
    acc = block_sum(acc, sh);
    if (threadIdx.x == 0) atomicAdd(out, acc);
}

// ── forward: real planes → row R2C → column FFT ─────────────────────────────────────────────

// Real correlation plane r of a staged row [5][cw] of premultiplied samples s = [w, w f0..w f3]
// (smi.wgsl:641-649): 0 → w, 1..4 → w f_i, 5..14 → s_i s_j / s_0 (0 where s_0 ≤ 1e-6).
__device__ __forceinline__ float real_plane_row(int r, const float* row, int cw, int x) {
    if (r < 5) return row[r * cw + x];
    const float s0 = row[x];
    if (s0 <= 1e-6f) return 0.f;
    const int k = r - 5;
    const int ti = (k < 4) ? 0 : (k < 7) ? 1 : (k < 9) ? 2 : 3;
    const int tj = (k < 4) ? k : (k < 7) ? k - 3 : (k < 9) ? k - 5 : 3;
    return row[(1 + ti) * cw + x] * row[(1 + tj) * cw + x] / s0;
}

// One block per grid row y < ch; lines = packed plane pairs (2z, 2z+1), lpb of them at a time.
// The row's 5 stack values per cell are staged in shared memory once (after the line buffers).
// Batched over blockIdx.y: item b reads grid + b·gbs and writes half + b·hbs.
template <class F>
__global__ void __launch_bounds__(256, 2) k_fwd_rows(const float* __restrict__ grid, int cw, int ch, int WP,
                                                     CorrPlanDev plan, F f, int lpb, float2* __restrict__ half,
                                                     size_t pstride, size_t gbs, size_t hbs) {
    extern __shared__ float2 smem[];
    const int nx = f.n(), tl = f.tl();
    const int y = blockIdx.x;
    grid += (size_t)blockIdx.y * gbs;
    half += (size_t)blockIdx.y * hbs;
    const int line = threadIdx.x / tl;
    const int t = threadIdx.x - line * tl;
    const int pl = padded_len(nx);
    float2* buf = smem + (line < lpb ? line : 0) * pl;
    float* row = reinterpret_cast<float*>(smem + lpb * pl);  // [5][cw]
    __shared__ int planes[16];
    if (threadIdx.x < 16) planes[threadIdx.x] = threadIdx.x < plan.n_real ? plan.planes[threadIdx.x] : -1;
    const size_t gn = (size_t)cw * ch;
    for (int i = threadIdx.x; i < 5 * cw; i += blockDim.x) {
        const int p = i / cw, x = i - p * cw;
        row[i] = __ldg(&grid[p * gn + (size_t)y * cw + x]);
    }
    __syncthreads();
    const int n_cplx = (plan.n_real + 1) / 2;
    for (int z0 = 0; z0 < n_cplx; z0 += lpb) {
        const int z = z0 + line;
        const bool act = line < lpb && z < n_cplx;
        if (act) {
            const int ra = planes[2 * z];
            const int rb = planes[2 * z + 1];
            for (int x = t; x < nx; x += tl) {
                float2 v = make_float2(0.f, 0.f);
                if (x < cw) {
                    v.x = real_plane_row(ra, row, cw, x);
                    if (rb >= 0) v.y = real_plane_row(rb, row, cw, x);
                }
                buf[pad_idx(x)] = v;
            }
        }
        __syncthreads();
        f.template run<false>(buf, t, act);
        if (act) {
            const bool has_b = 2 * z + 1 < plan.n_real;
            float2* oa = half + (size_t)(2 * z) * pstride + (size_t)y * WP;
            float2* ob = half + (size_t)(2 * z + 1) * pstride + (size_t)y * WP;
            for (int x = t; x <= nx / 2; x += tl) {
                const float2 Z = buf[pad_idx(x)];
                const float2 Zm = buf[pad_idx(x == 0 ? 0 : nx - x)];
                oa[x] = make_float2(0.5f * (Z.x + Zm.x), 0.5f * (Z.y - Zm.y));
                if (has_b) ob[x] = make_float2(0.5f * (Z.y + Zm.y), 0.5f * (Zm.x - Z.x));
            }
        }
        __syncthreads();
    }
}

// Column FFTs of the half spectra, in place: block = a tile of tx columns of one plane; rows
// ≥ rows_in read as zero. Loads and stores go 8 per thread at a time (all in flight together).
template <class F, bool INV>
__global__ void __launch_bounds__(512, 2) k_cols(float2* __restrict__ half, size_t pstride, int WP, int ncols,
                                                 int rows_in, F f, int tx) {
    extern __shared__ float2 smem[];
    const int x0 = blockIdx.x * tx;
    float2* base = half + (size_t)blockIdx.y * pstride;
    const int ny = f.n(), pl = line_pitch(ny), tl = f.tl();
    const int total = tx * ny;
    for (int e0 = 0; e0 < total; e0 += 8 * blockDim.x) {
        float2 v[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int e = e0 + i * blockDim.x + threadIdx.x;
            const int y = e / tx, c = e - y * tx;
            v[i] = (e < total && y < rows_in && x0 + c < ncols) ? base[(size_t)y * WP + x0 + c] : make_float2(0.f, 0.f);
        }
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int e = e0 + i * blockDim.x + threadIdx.x;
            const int y = e / tx, c = e - y * tx;
            if (e < total) smem[c * pl + pad_idx(y)] = v[i];
        }
    }
    __syncthreads();
    const int line = threadIdx.x / tl, t = threadIdx.x - line * tl;
    f.template run<INV>(smem + (line < tx ? line : 0) * pl, t, line < tx);
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
        const int y = e / tx, c = e - y * tx;
        if (x0 + c < ncols) base[(size_t)y * WP + x0 + c] = smem[c * pl + pad_idx(y)];
    }
}

// ── inverse: products and column IFFTs ──────────────────────────────────────────────────────

// block (correlation slot k, column tile, item): P = A·conj(B) on the tile, inverse column FFT
// → Q; item b reads ha + b·abs, hb + b·bbs and writes Q + b·qbs
template <class F>
__global__ void __launch_bounds__(512, 2) k_inv_cols(const float2* __restrict__ ha, const float2* __restrict__ hb,
                                                     size_t pstride, int WP, int ncols, CorrPlanDev plan, F f, int tx,
                                                     float2* __restrict__ Q, size_t abs_, size_t bbs, size_t qbs) {
    extern __shared__ float2 smem[];
    const int k = blockIdx.x;
    const int x0 = blockIdx.y * tx;
    const size_t item = blockIdx.z;
    const float2* A = ha + item * abs_ + (size_t)plan.ca[k] * pstride;
    const float2* B = hb + item * bbs + (size_t)plan.cb[k] * pstride;
    float2* O = Q + item * qbs + (size_t)k * pstride;
    const int ny = f.n(), pl = line_pitch(ny), tl = f.tl();
    const int total = tx * ny;
    for (int e0 = 0; e0 < total; e0 += 4 * blockDim.x) {
        float2 a[4], b[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int e = e0 + i * blockDim.x + threadIdx.x;
            const int y = e / tx, c = e - y * tx;
            const bool ok = e < total && x0 + c < ncols;
            const size_t ix = (size_t)y * WP + x0 + c;
            a[i] = ok ? __ldg(&A[ix]) : make_float2(0.f, 0.f);
            b[i] = ok ? __ldg(&B[ix]) : make_float2(0.f, 0.f);
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int e = e0 + i * blockDim.x + threadIdx.x;
            const int y = e / tx, c = e - y * tx;
            if (e < total) smem[c * pl + pad_idx(y)] = cmulc(a[i], b[i]);
        }
    }
    __syncthreads();
    const int line = threadIdx.x / tl, t = threadIdx.x - line * tl;
    f.template run<true>(smem + (line < tx ? line : 0) * pl, t, line < tx);
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
        const int y = e / tx, c = e - y * tx;
        if (x0 + c < ncols) O[(size_t)y * WP + x0 + c] = smem[c * pl + pad_idx(y)];
    }
}

// ── inverse rows + per-shift score ──────────────────────────────────────────────────────────

// block (row y, split s, item): every correlation pair's row (Hermitian full row from the half
// spectrum) pre-combined for outputs x ≡ s (mod S), inverse FFT of length L = nx/S, the sums
// kept in shared memory; then the score of each of the row's L shifts and the block argmax.
// Item b reads Q + b·qbs and n00p[b], writes map + b·mbs; best and zero_out may be null.
template <class F, int NF, bool EXACT, bool CALIB, int SS>
__global__ void __launch_bounds__(512, 1) k_inv_rows(const float2* __restrict__ Q, size_t pstride, int WP, int nx, int S,
                                                     CorrPlanDev plan, F f, int lpb, const float2* __restrict__ tw_nx,
                                                     CombineParams cp, const double* __restrict__ n00p,
                                                     float* __restrict__ map, unsigned long long* best,
                                                     float* zero_out, size_t qbs, size_t mbs) {
    extern __shared__ float2 smem[];
    const int y = blockIdx.x / S, s = blockIdx.x - (blockIdx.x / S) * S;
    Q += (size_t)blockIdx.y * qbs;
    map += (size_t)blockIdx.y * mbs;
    n00p += blockIdx.y;
    const int L = f.n(), pl = padded_len(L), tl = f.tl();
    float* corr = reinterpret_cast<float*>(smem + lpb * pl);  // [n_corr][L]
    const int line = threadIdx.x / tl, t = threadIdx.x - line * tl;
    float2* buf = smem + (line < lpb ? line : 0) * pl;
    const int npairs = (plan.n_corr + 1) / 2;
    for (int p0 = 0; p0 < npairs; p0 += lpb) {
        const int pr = p0 + line;
        const bool act = line < lpb && pr < npairs;
        const int k1 = 2 * pr, k2 = (2 * pr + 1 < plan.n_corr) ? 2 * pr + 1 : -1;
        if (act) {
            const float2* q1 = Q + (size_t)k1 * pstride + (size_t)y * WP;
            const float2* q2 = (k2 >= 0) ? Q + (size_t)k2 * pstride + (size_t)y * WP : q1;
            const bool has2 = k2 >= 0;
            // the Hermitian full row, pre-combined for x ≡ s (mod S); loads of B points per
            // thread issued together (S·2·B in flight)
            constexpr int B = (SS == 1) ? 8 : 4;
            const int per = (L + tl - 1) / tl;
            for (int b0 = 0; b0 < per; b0 += B) {
                float2 ra[B][SS > 0 ? SS : 1], rb[B][SS > 0 ? SS : 1];
                if constexpr (SS > 0) {
#pragma unroll
                    for (int i = 0; i < B; ++i) {
                        const int m = t + (b0 + i) * tl;
#pragma unroll
                        for (int q = 0; q < SS; ++q) {
                            const int x = m + q * L;
                            const int ix = (x <= nx / 2) ? x : nx - x;
                            const bool ok = m < L;
                            ra[i][q] = ok ? __ldg(&q1[ix]) : make_float2(0.f, 0.f);
                            rb[i][q] = (ok && has2) ? __ldg(&q2[ix]) : make_float2(0.f, 0.f);
                        }
                    }
                }
#pragma unroll
                for (int i = 0; i < B; ++i) {
                    const int m = t + (b0 + i) * tl;
                    if (m >= L) continue;
                    float2 acc = make_float2(0.f, 0.f);
                    const int nq = SS > 0 ? SS : S;
                    for (int q = 0; q < nq; ++q) {
                        const int x = m + q * L;
                        float2 a, bb;
                        if constexpr (SS > 0) {
                            a = ra[i][q];
                            bb = rb[i][q];
                        } else {
                            const int ix = (x <= nx / 2) ? x : nx - x;
                            a = __ldg(&q1[ix]);
                            bb = has2 ? __ldg(&q2[ix]) : make_float2(0.f, 0.f);
                        }
                        // Z = Q1 + i·Q2 on the half row; conj(Q1) + i·conj(Q2) on the mirrored half
                        float2 z = (x <= nx / 2) ? make_float2(a.x - bb.y, a.y + bb.x) : make_float2(a.x + bb.y, bb.x - a.y);
                        if (q > 0 && s > 0) z = cmul(z, cconj(__ldg(&tw_nx[(q * s * L) % nx])));
                        acc = cadd(acc, z);
                    }
                    if (s > 0) acc = cmul(acc, cconj(__ldg(&tw_nx[m * s])));
                    buf[pad_idx(m)] = acc;
                }
            }
        }
        __syncthreads();
        f.template run<true>(buf, t, act);
        if (act) {
            for (int m = t; m < L; m += tl) {
                const float2 z = buf[pad_idx(m)];
                corr[(size_t)k1 * L + m] = z.x;
                if (k2 >= 0) corr[(size_t)k2 * L + m] = z.y;
            }
        }
        __syncthreads();
    }
    const double n00 = *n00p;
    float bv = -3.4e38f;
    uint32_t bi = 0xffffffffu;
    for (int m = threadIdx.x; m < L; m += blockDim.x) {
        const float sc = combine_t<NF, EXACT, CALIB>([&](int k) { return corr[(size_t)k * L + m]; }, cp, n00);
        const int x = m * S + s;
        const uint32_t idx = (uint32_t)y * (uint32_t)nx + (uint32_t)x;
        map[idx] = sc;
        if (sc > bv || (sc == bv && idx < bi)) {
            bv = sc;
            bi = idx;
        }
        if (idx == 0 && zero_out) *zero_out = sc;
    }
    if (!best) return;
    unsigned long long key = (bi == 0xffffffffu) ? 0ull : argmax_key(bv, bi);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long other = __shfl_xor_sync(0xffffffffu, key, o);
        key = other > key ? other : key;
    }
    if ((threadIdx.x & 31) == 0 && key) atomicMax(best, key);
}

// The line policy for a plan: compile-time power-of-two lines for the common lengths, the
// generic mixed-radix schedule otherwise.
template <class Fn>
cudaError_t with_line(const LinePlan& p, Fn&& fn) {
    switch (p.n) {
        case 256: return fn(Pow2Line<256>{p.tw});
        case 512: return fn(Pow2Line<512>{p.tw});
        case 1024: return fn(Pow2Line<1024>{p.tw});
        case 2048: return fn(Pow2Line<2048>{p.tw});
        default: return fn(GenericLine{p});
    }
}

}  // namespace

// ── launchers ────────────────────────────────────────────────────────────────────────────────

cudaError_t warp_stack(const float* stack, int w, int h, const float hi[9], bool ok, int W, int Hh, float* canvas,
                       cudaStream_t st) {
    Mat9f m;
    for (int i = 0; i < 9; ++i) m.m[i] = hi[i];
    dim3 b(32, 8), g((W + 31) / 32, (Hh + 7) / 8);
    k_warp_stack<<<g, b, 0, st>>>(stack, w, h, m, ok ? 1 : 0, W, Hh, canvas);
    return cudaGetLastError();
}

cudaError_t paste_stack(const float* stack, int w, int h, int ox, int oy, int W, int Hh, float* canvas,
                        cudaStream_t st) {
    dim3 b(32, 8), g((W + 31) / 32, (Hh + 7) / 8);
    k_paste_stack<<<g, b, 0, st>>>(stack, w, h, ox, oy, W, Hh, canvas);
    return cudaGetLastError();
}

cudaError_t resample_grid(const float* canvas, int W, int Hh, int cw, int ch, float* grid, cudaStream_t st) {
    dim3 b(32, 8), g((cw + 31) / 32, (ch + 7) / 8);
    k_resample<<<g, b, 0, st>>>(canvas, W, Hh, cw, ch, grid);
    return cudaGetLastError();
}

cudaError_t lag0_count(const float* a, const float* b, int cw, int ch, double* out, cudaStream_t st) {
    cudaMemsetAsync(out, 0, sizeof(double), st);
    const int n = cw * ch;
    int blocks = (n + 255) / 256;
    if (blocks > 296) blocks = 296;
    k_lag0<<<blocks, 256, 0, st>>>(a, b, n, out);
    return cudaGetLastError();
}

static int lines_per_block(int tl, int want_threads) {
    int l = want_threads / tl;
    return l < 1 ? 1 : l;
}

// threads per line of the policy with_line picks for this plan
static int line_threads(const LinePlan& p) {
    switch (p.n) {
        case 256: case 512: case 1024: case 2048: return p.n / 16;
        default: return p.tl;
    }
}

cudaError_t forward_rows(const float* grid, const MapGeom& g, const CorrPlanDev& plan, const LinePlan& row,
                         float2* half, cudaStream_t st, int batch, size_t grid_stride, size_t half_stride) {
    const size_t pstride = (size_t)g.ny * g.WP;
    const int tl = line_threads(row);
    const int n_cplx = (plan.n_real + 1) / 2;
    int lines = lines_per_block(tl, 256);
    if (lines > n_cplx) lines = n_cplx;
    const size_t sm = (size_t)lines * padded_len(g.nx) * sizeof(float2) + (size_t)5 * g.cw * sizeof(float);
    return with_line(row, [&](auto f) {
        cudaFuncSetAttribute(k_fwd_rows<decltype(f)>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        k_fwd_rows<<<dim3(g.ch, batch), lines * tl, sm, st>>>(grid, g.cw, g.ch, g.WP, plan, f, lines, half, pstride,
                                                              grid_stride, half_stride);
        return cudaGetLastError();
    });
}

static int col_tile(const LinePlan& col) {
    int tx = lines_per_block(line_threads(col), 512);
    while (tx > 1 && (size_t)tx * line_pitch(col.n) * sizeof(float2) > 110 * 1024) tx >>= 1;
    return tx;
}

cudaError_t forward_cols(float2* half, const MapGeom& g, const CorrPlanDev& plan, const LinePlan& col,
                         cudaStream_t st, int batch) {
    const size_t pstride = (size_t)g.ny * g.WP;
    const int ncols = g.nx / 2 + 1;
    const int tx = col_tile(col), tl = line_threads(col);
    const size_t sm = (size_t)tx * line_pitch(g.ny) * sizeof(float2);
    dim3 gc((ncols + tx - 1) / tx, plan.n_real * batch);
    return with_line(col, [&](auto f) {
        cudaFuncSetAttribute(k_cols<decltype(f), false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        k_cols<decltype(f), false><<<gc, tx * tl, sm, st>>>(half, pstride, g.WP, ncols, g.ch, f, tx);
        return cudaGetLastError();
    });
}

cudaError_t inverse_columns(const float2* ha, const float2* hb, const MapGeom& g, const CorrPlanDev& plan,
                            const LinePlan& col, float2* Q, cudaStream_t st, int batch, size_t a_stride,
                            size_t b_stride, size_t q_stride) {
    const size_t pstride = (size_t)g.ny * g.WP;
    const int ncols = g.nx / 2 + 1;
    const int tx = col_tile(col), tl = line_threads(col);
    const size_t sm = (size_t)tx * line_pitch(g.ny) * sizeof(float2);
    dim3 gc(plan.n_corr, (ncols + tx - 1) / tx, batch);
    return with_line(col, [&](auto f) {
        cudaFuncSetAttribute(k_inv_cols<decltype(f)>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        k_inv_cols<<<gc, tx * tl, sm, st>>>(ha, hb, pstride, g.WP, ncols, plan, f, tx, Q, a_stride, b_stride, q_stride);
        return cudaGetLastError();
    });
}

// the row pass: power-of-two lines with 8 points per thread, as many lines as fit 512 threads
// (the score phase uses all 512)
static int row_threads(const LinePlan& p) {
    switch (p.n) {
        case 256: case 512: case 1024: case 2048: return p.n / 8;
        default: return p.tl;
    }
}
static int row_lines(int tl) { return lines_per_block(tl, 512) < 4 ? lines_per_block(tl, 512) : 4; }

template <class Fn>
cudaError_t with_row_line(const LinePlan& p, Fn&& fn) {
    switch (p.n) {
        case 256: return fn(Pow2Line<256, 32>{p.tw});
        case 512: return fn(Pow2Line<512, 64>{p.tw});
        case 1024: return fn(Pow2Line<1024, 128>{p.tw});
        case 2048: return fn(Pow2Line<2048, 256>{p.tw});
        default: return fn(GenericLine{p});
    }
}

size_t row_pass_smem(int L, int n_corr, int tl) {
    return (size_t)row_lines(tl) * padded_len(L) * sizeof(float2) + (size_t)n_corr * L * sizeof(float);
}

int row_split(int nx, int n_corr) {
    for (int S = 1; S <= 64; ++S) {
        if (nx % S) continue;
        const int L = nx / S;
        if (L > kMaxLine) continue;
        int tl = (L + 15) / 16;
        tl = ((tl + 31) / 32) * 32;
        if (L == 256 || L == 512 || L == 1024 || L == 2048) tl = L / 8;
        if (tl > 512) continue;
        if (row_pass_smem(L, n_corr, tl) <= 220 * 1024) return S;
    }
    return 0;
}

struct RowBatch {
    int n;
    size_t q, m;
};

template <class F, int NF, bool EXACT, bool CALIB>
static cudaError_t launch_rows(const float2* Q, const MapGeom& g, const CorrPlanDev& plan, F f, int S,
                               const float2* tw_nx, const CombineParams& cp, const double* n00, float* map,
                               unsigned long long* best, float* zero, int lpb, size_t sm, cudaStream_t st,
                               const RowBatch& rb) {
    auto k = S == 1 ? k_inv_rows<F, NF, EXACT, CALIB, 1> : S == 2 ? k_inv_rows<F, NF, EXACT, CALIB, 2>
                                                                 : k_inv_rows<F, NF, EXACT, CALIB, 0>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k<<<dim3(g.ny * S, rb.n), 512, sm, st>>>(Q, (size_t)g.ny * g.WP, g.WP, g.nx, S, plan, f, lpb, tw_nx, cp, n00, map,
                                             best, zero, rb.q, rb.m);
    return cudaGetLastError();
}

cudaError_t inverse_rows_score(const float2* Q, const MapGeom& g, const CorrPlanDev& plan, const LinePlan& line,
                               int S, const float2* tw_nx, const CombineParams& cp, const double* n00, float* map,
                               unsigned long long* best, float* zero, cudaStream_t st, int batch, size_t q_stride,
                               size_t map_stride) {
    const RowBatch rb{batch, q_stride, map_stride};
    const int tl = row_threads(line);
    const int lpb = row_lines(tl);
    if (lpb * tl > 512) return cudaErrorInvalidConfiguration;
    const size_t sm = row_pass_smem(line.n, plan.n_corr, tl);
    return with_row_line(line, [&](auto f) {
        using Fp = decltype(f);
        if (cp.nf == 4) {
            if (!cp.exact) return launch_rows<Fp, 4, false, false>(Q, g, plan, f, S, tw_nx, cp, n00, map, best, zero, lpb, sm, st, rb);
            if (cp.calib) return launch_rows<Fp, 4, true, true>(Q, g, plan, f, S, tw_nx, cp, n00, map, best, zero, lpb, sm, st, rb);
            return launch_rows<Fp, 4, true, false>(Q, g, plan, f, S, tw_nx, cp, n00, map, best, zero, lpb, sm, st, rb);
        }
        if (!cp.exact) return launch_rows<Fp, 3, false, false>(Q, g, plan, f, S, tw_nx, cp, n00, map, best, zero, lpb, sm, st, rb);
        if (cp.calib) return launch_rows<Fp, 3, true, true>(Q, g, plan, f, S, tw_nx, cp, n00, map, best, zero, lpb, sm, st, rb);
        return launch_rows<Fp, 3, true, false>(Q, g, plan, f, S, tw_nx, cp, n00, map, best, zero, lpb, sm, st, rb);
    });
}

}  // namespace zc
