// The four passes of a shift map (and of a batch of sweep candidates' maps) as kernels templated
// on the line-FFT policy, with one launcher per pass. Included by the translation units that
// instantiate them for their line lengths (shiftmap.cu, lines_*.cu); everything here has internal
// linkage, so each unit carries its own instantiations.
//
//   forward rows   real planes → row R2C (rows < ch) into the half spectra [n_real][ny][WP]
//   forward cols   column FFTs of the half spectra, in place (rows ≥ ch read as zero)
//   inverse cols   per correlation and column tile: A·conj(B), inverse column FFT → Q[slot]
//   rows           per row: correlations paired as c1 + i·c2 on the Hermitian full row, inverse
//                  row FFT, the per-shift score in float64 and the argmax; several rows per block
//                  when a row's sums fit shared memory several times over (k_rows_multi), else a
//                  row split S ways by one decimation-in-frequency step (k_inv_rows)
#pragma once

#include <algorithm>

#include "combine.cuh"
#include "common.cuh"
#include "kernels.hpp"

namespace zc {

// line lengths with a compile-time schedule (FixedLine) in some translation unit
constexpr int kFixedLines[] = {48, 64, 96, 128, 144, 192, 256, 288, 384, 432, 512, 1024, 2048};
inline bool fixed_line(int n) {
    for (int v : kFixedLines)
        if (v == n) return true;
    return false;
}
// threads per line of the row pass's compile-time lines: N/8 (8 points a thread), raised to 32
// where N/8 is below 32 and does not divide it, so no short line shares a warp with part of
// another (lines of 24 threads straddled warps: shared-memory bank conflicts between the two
// lines' slots)
__host__ __device__ constexpr int row_tpl(int n) { return (n / 8 >= 32 || 32 % (n / 8) == 0) ? n / 8 : 32; }
// threads per line of the row pass's policy for length L (FixedLine<L, row_tpl(L)>, or the
// generic plan's)
inline int row_tl(int L) {
    if (fixed_line(L)) return row_tpl(L);
    int tl = (L + 15) / 16;
    return ((tl + 31) / 32) * 32;
}
constexpr size_t kRowSmem = 220 * 1024;
// lines the multi-row kernel transforms at a time, and its shared memory for RB rows
inline int multi_lines(int tl) { return std::max(1, std::min(512 / tl, 16)); }
inline size_t multi_row_smem(int nx, int n_corr, int tl, int RB) {
    return (size_t)multi_lines(tl) * padded_len(nx) * sizeof(float2) + (size_t)RB * n_corr * nx * sizeof(float);
}

// Line pitch of a column tile. Lines of 1024 points and more come in tiles of at most 8 lines
// (512 threads of N/16) and keep line_pitch's ≡ 4 (mod 16), a compile-time constant for
// compile-time lines; shorter lines come in wide tiles (the sweep's 192-point columns: 33 lines)
// whose warps touch 32 lines at one point each, which tile_pitch's odd pitch spreads over all
// bank pairs (≡ 4 put them in 4).
__host__ __device__ __forceinline__ constexpr int col_pitch(int n, int tx) {
    return n >= 1024 ? line_pitch(n) : tile_pitch(n, tx);
}

enum class Pass { FwdRows, FwdCols, InvCols, Rows };

// Everything a pass launch needs; the batch's items sit at the given strides (elements).
struct PassArgs {
    MapGeom g{};
    const CorrPlanDev* plan = nullptr;
    int batch = 1;
    const float* grid = nullptr;  // forward rows: [5][ch][cw] per item
    size_t grid_stride = 0;
    float2* half = nullptr;       // forward rows / columns: written; inverse columns: A
    size_t half_stride = 0;
    const float2* half_b = nullptr;  // inverse columns: B (b_stride 0: one fixed side)
    size_t b_stride = 0;
    float2* Q = nullptr;          // inverse columns: written; rows: read
    size_t q_stride = 0;
    int S = 1;                    // rows: the split
    const float2* tw_nx = nullptr;
    const CombineParams* cp = nullptr;
    const double* n00 = nullptr;  // one per item
    float* map = nullptr;
    size_t map_stride = 0;
    unsigned long long* best = nullptr;
    float* zero = nullptr;
};

namespace {

// ── forward: real planes → row R2C → column FFT ─────────────────────────────────────────────

// Real correlation plane r of a staged row [5][cw] of premultiplied samples s = [w, w f0..w f3]
// (smi.wgsl:641-649): 0 → w, 1..4 → w f_i, 5..14 → s_i s_j / s_0 (0 where s_0 ≤ 1e-6), the
// division as a product with inv0[x] = 1 / s_0 (0 where s_0 ≤ 1e-6), staged with the row.
__device__ __forceinline__ float real_plane_row(int r, const float* row, const float* inv0, int cw, int x) {
    if (r < 5) return row[r * cw + x];
    const int k = r - 5;
    const int ti = (k < 4) ? 0 : (k < 7) ? 1 : (k < 9) ? 2 : 3;
    const int tj = (k < 4) ? k : (k < 7) ? k - 3 : (k < 9) ? k - 5 : 3;
    return row[(1 + ti) * cw + x] * row[(1 + tj) * cw + x] * inv0[x];
}

// One block per grid row y < ch; lines = packed plane pairs (2z, 2z+1), lpb of them at a time.
// The row's 5 stack values per cell are staged in shared memory once (after the line buffers).
// Batched over blockIdx.y: item b reads grid + b·gbs and writes half + b·hbs.
// LO: cw ≤ nx/2, so the first butterflies read only the row's lower half.
template <class F, bool LO>
__global__ void __launch_bounds__(512, 1) k_fwd_rows(const float* __restrict__ grid, int cw, int ch, int WP,
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
    float* inv0 = row + 5 * cw;                               // [cw]
    __shared__ int planes[16];
    if (threadIdx.x < 16) planes[threadIdx.x] = threadIdx.x < plan.n_real ? plan.planes[threadIdx.x] : -1;
    const size_t gn = (size_t)cw * ch;
    for (int i = threadIdx.x; i < 5 * cw; i += blockDim.x) {
        const int p = i / cw, x = i - p * cw;
        const float v = __ldg(&grid[p * gn + (size_t)y * cw + x]);
        row[i] = v;
        if (p == 0) inv0[x] = v <= 1e-6f ? 0.f : 1.f / v;
    }
    __syncthreads();
    const int n_cplx = (plan.n_real + 1) / 2;
    for (int z0 = 0; z0 < n_cplx; z0 += lpb) {
        const int z = z0 + line;
        const bool act = line < lpb && z < n_cplx;
        const int ra = act ? planes[2 * z] : 0;
        const int rb = act ? planes[2 * z + 1] : -1;
        // the first butterflies read the staged row directly (real planes ra + i·rb, zero past cw)
        f.template run_in<false, LO>(buf, t, act, [&](int x) {
            float2 v = make_float2(0.f, 0.f);
            if (x < cw) {
                v.x = real_plane_row(ra, row, inv0, cw, x);
                if (rb >= 0) v.y = real_plane_row(rb, row, inv0, cw, x);
            }
            return v;
        });
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
// ≥ rows_in read as zero. Thread (column c, line thread t), c fastest, so each load or store of
// a warp covers 8 rows × 4 adjacent columns (whole 32-byte sectors); the first butterflies read
// global memory and the last write it (run_io), with only the middle stages in shared memory.
// LO: rows_in ≤ n/2, so the first butterflies read only rows y < n/2 (the rest are zero).
template <class F, bool INV, bool LO>
__global__ void __launch_bounds__(512, 2) k_cols(float2* __restrict__ half, size_t pstride, int WP, int ncols,
                                                 int rows_in, F f, int tx) {
    extern __shared__ float2 smem[];
    const int x0 = blockIdx.x * tx;
    float2* base = half + (size_t)blockIdx.y * pstride;
    const int pl = col_pitch(f.n(), tx);
    const int c = threadIdx.x % tx, t = threadIdx.x / tx, col = x0 + c;
    const bool okc = col < ncols;
    float2* p = base + col;
    f.template run_io<INV, LO>(
        smem + c * pl, t, true,
        [&](int y) { return (okc && y < rows_in) ? p[(size_t)y * WP] : make_float2(0.f, 0.f); },
        [&](int y, float2 v) {
            if (okc) p[(size_t)y * WP] = v;
        });
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
    const int c = threadIdx.x % tx, t = threadIdx.x / tx, col = x0 + c;
    const bool okc = col < ncols;
    const float2* A = ha + item * abs_ + (size_t)plan.ca[k] * pstride + col;
    const float2* B = hb + item * bbs + (size_t)plan.cb[k] * pstride + col;
    float2* O = Q + item * qbs + (size_t)k * pstride + col;
    const int pl = col_pitch(f.n(), tx);
    f.template run_io<true>(
        smem + c * pl, t, true,
        [&](int y) {
            return okc ? cmulc(__ldg(&A[(size_t)y * WP]), __ldg(&B[(size_t)y * WP])) : make_float2(0.f, 0.f);
        },
        [&](int y, float2 v) {
            if (okc) O[(size_t)y * WP] = v;
        });
}

// The inverse columns as a persistent pipeline (lines of N points whose first stage has one
// butterfly per line thread: N = 1024, 2048): 1 block per SM walks the items (column tile,
// correlation slot), correlation fastest so the blocks running together share tiles in L2. Each
// thread holds its next item's 2 × R0 products' operands in registers: they load while the
// current item transforms, so the loads' latency hides behind the butterflies instead of
// stalling a whole block (the one-item-per-block kernel above waits on them).
template <int N>
__global__ void __launch_bounds__(512, 1) k_inv_cols_pipe(const float2* __restrict__ ha, const float2* __restrict__ hb,
                                                          size_t pstride, int WP, int ncols, CorrPlanDev plan,
                                                          const float2* __restrict__ tw, int tx, float2* __restrict__ Q,
                                                          int nitems) {
    constexpr int TL = N / 16, R0 = Mix<N>::radix(0), M0 = N / R0;
    static_assert(M0 == TL, "one first-stage butterfly per line thread");
    extern __shared__ float2 smem[];
    const int c = threadIdx.x % tx, t = threadIdx.x / tx;
    float2* buf = smem + c * line_pitch(N);
    const int nk = plan.n_corr;
    float2 pa[R0], pb[R0];
    auto load = [&](int item) {
        const int k = item % nk, col = (item / nk) * tx + c;
        const bool okc = col < ncols;
        const float2* A = ha + (size_t)plan.ca[k] * pstride + (okc ? col : 0);
        const float2* B = hb + (size_t)plan.cb[k] * pstride + (okc ? col : 0);
#pragma unroll
        for (int r = 0; r < R0; ++r) {
            const size_t o = (size_t)(t + r * M0) * WP;
            pa[r] = okc ? __ldg(&A[o]) : make_float2(0.f, 0.f);
            pb[r] = okc ? __ldg(&B[o]) : make_float2(0.f, 0.f);
        }
    };
    int item = blockIdx.x;
    if (item < nitems) load(item);
    for (; item < nitems; item += gridDim.x) {
        float2 v[R0];
#pragma unroll
        for (int r = 0; r < R0; ++r) v[r] = cmulc(pa[r], pb[r]);
        const int k = item % nk, col = (item / nk) * tx + c;
        const bool okc = col < ncols;
        float2* O = Q + (size_t)k * pstride + (okc ? col : 0);
        if (item + (int)gridDim.x < nitems) load(item + gridDim.x);
        mix_fft_regs<N, TL, true>(
            buf, tw, t, true, v,
            [&](int y, float2 val) {
                if (okc) O[(size_t)y * WP] = val;
            },
            [] {});
        __syncthreads();  // the line buffers are refilled by the next item
    }
}

template <class F>
struct FixedN {
    static constexpr int value = 0;
};
template <int N, int TPL>
struct FixedN<FixedLine<N, TPL>> {
    static constexpr int value = N;
};

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
    const double n00 = lag0_units(cp, *n00p);
    const CombineParams cpr = row_params(cp, y, (int)(pstride / WP));
    float bv = -3.4e38f;
    uint32_t bi = 0xffffffffu;
    for (int m = threadIdx.x; m < L; m += blockDim.x) {
        const float sc = combine_t<NF, EXACT, CALIB>([&](int k) { return corr[(size_t)k * L + m]; }, cpr, n00);
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


// block (rows y0 … y0 + RB − 1 of one item): for each row, every correlation pair's row (the
// Hermitian full row from the half spectrum) inverse-transformed, the sums kept in shared memory
// [RB][n_corr][nx]; then the score of each of the block's shifts and the block argmax. Item b
// reads Q + b·qbs and n00p[b], writes map + b·mbs; best and zero_out may be null.
template <class F, int NF, bool EXACT, bool CALIB>
__global__ void __launch_bounds__(512, 1) k_rows_multi(const float2* __restrict__ Q, size_t pstride, int WP, int ny,
                                                       int RB, CorrPlanDev plan, F f, int lpb, CombineParams cp,
                                                       const double* __restrict__ n00p, float* __restrict__ map,
                                                       unsigned long long* best, float* zero_out, size_t qbs,
                                                       size_t mbs) {
    extern __shared__ float2 smem[];
    const int nx = f.n(), pl = padded_len(nx), tl = f.tl();
    const int y0 = blockIdx.x * RB;
    const int rows = min(RB, ny - y0);
    Q += (size_t)blockIdx.y * qbs;
    map += (size_t)blockIdx.y * mbs;
    n00p += blockIdx.y;
    float* corr = reinterpret_cast<float*>(smem + lpb * pl);  // [RB][n_corr][nx]
    const int line = threadIdx.x / tl, t = threadIdx.x - line * tl;
    float2* buf = smem + (line < lpb ? line : 0) * pl;
    const int npairs = (plan.n_corr + 1) / 2;
    const int ntask = rows * npairs;
    for (int p0 = 0; p0 < ntask; p0 += lpb) {
        const int task = p0 + line;
        const bool act = line < lpb && task < ntask;
        const int r = act ? task / npairs : 0;
        const int pr = act ? task - r * npairs : 0;
        const int k1 = 2 * pr, k2 = (2 * pr + 1 < plan.n_corr) ? 2 * pr + 1 : -1;
        const size_t row = (size_t)(y0 + r) * WP;
        const float2* q1 = Q + (size_t)k1 * pstride + row;
        const float2* q2 = (k2 >= 0) ? Q + (size_t)k2 * pstride + row : q1;
        const bool has2 = k2 >= 0;
        float* c = corr + (size_t)r * plan.n_corr * nx;
        // the first butterflies read the Hermitian row from the half spectra, the last write the
        // row's sums straight to the correlation rows
        f.template run_io<true>(
            buf, t, act,
            [&](int x) {
                // Z = Q1 + i·Q2 on the half row; conj(Q1) + i·conj(Q2) on the mirrored half
                const int ix = (x <= nx / 2) ? x : nx - x;
                const float2 a = __ldg(&q1[ix]);
                const float2 bb = has2 ? __ldg(&q2[ix]) : make_float2(0.f, 0.f);
                return (x <= nx / 2) ? make_float2(a.x - bb.y, a.y + bb.x) : make_float2(a.x + bb.y, bb.x - a.y);
            },
            [&](int m, float2 z) {
                c[(size_t)k1 * nx + m] = z.x;
                if (has2) c[(size_t)k2 * nx + m] = z.y;
            });
        __syncthreads();
    }
    const double n00 = lag0_units(cp, *n00p);
    float bv = -3.4e38f;
    uint32_t bi = 0xffffffffu;
    for (int m = threadIdx.x; m < rows * nx; m += blockDim.x) {
        const int r = m / nx, x = m - r * nx;
        const float* c = corr + (size_t)r * plan.n_corr * nx + x;
        const float sc =
            combine_t<NF, EXACT, CALIB>([&](int k) { return c[(size_t)k * nx]; }, row_params(cp, y0 + r, ny), n00);
        const uint32_t idx = (uint32_t)(y0 + r) * (uint32_t)nx + (uint32_t)x;
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


inline int lines_per_block(int tl, int want_threads) { return std::max(1, want_threads / tl); }
// column tile: as many lines as 512 threads hold (no more than the columns), within 110 KB of
// shared memory
inline int col_tile(int n, int tl, int ncols) {
    int tx = std::min(lines_per_block(tl, 512), ncols);
    while (tx > 1 && (size_t)tx * col_pitch(n, tx) * sizeof(float2) > 110 * 1024) tx >>= 1;
    // the same number of tiles, balanced: no last tile of mostly idle columns
    const int tiles = (ncols + tx - 1) / tx;
    return (ncols + tiles - 1) / tiles;
}
// the split row pass: as many lines as fit 512 threads, at most 4 (the score phase uses all 512)
inline int split_lines(int tl) { return std::min(lines_per_block(tl, 512), 4); }

template <class F, int NF, bool EXACT, bool CALIB, bool SPLIT>
cudaError_t launch_rows(F f, const PassArgs& a, cudaStream_t st) {
    const MapGeom& g = a.g;
    const CorrPlanDev& plan = *a.plan;
    const int tl = f.tl(), L = f.n();
    const size_t pstride = (size_t)g.ny * g.WP;
    if (a.S == 1) {
        const int lpb = multi_lines(tl);
        int RB = 1;
        while (RB < 8 && RB < g.ny && multi_row_smem(L, plan.n_corr, tl, RB + 1) <= kRowSmem) ++RB;
        const size_t sm = multi_row_smem(L, plan.n_corr, tl, RB);
        if (sm > kRowSmem || lpb * tl > 512) return cudaErrorInvalidConfiguration;
        auto k = k_rows_multi<F, NF, EXACT, CALIB>;
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        k<<<dim3((g.ny + RB - 1) / RB, a.batch), 512, sm, st>>>(a.Q, pstride, g.WP, g.ny, RB, plan, f, lpb, *a.cp,
                                                                  a.n00, a.map, a.best, a.zero, a.q_stride,
                                                                  a.map_stride);
        return cudaGetLastError();
    }
    if constexpr (SPLIT) {
        const int lpb = split_lines(tl);
        if (lpb * tl > 512) return cudaErrorInvalidConfiguration;
        const size_t sm = (size_t)lpb * padded_len(L) * sizeof(float2) + (size_t)plan.n_corr * L * sizeof(float);
        auto k = a.S == 2 ? k_inv_rows<F, NF, EXACT, CALIB, 2> : k_inv_rows<F, NF, EXACT, CALIB, 0>;
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        k<<<dim3(g.ny * a.S, a.batch), 512, sm, st>>>(a.Q, pstride, g.WP, g.nx, a.S, plan, f, lpb, a.tw_nx, *a.cp,
                                                      a.n00, a.map, a.best, a.zero, a.q_stride, a.map_stride);
        return cudaGetLastError();
    } else {
        return cudaErrorNotSupported;
    }
}

// One pass over a batch with line policy F (SPLIT: also the split row pass, for rows that do
// not fit shared memory whole).
template <Pass P, class F, bool SPLIT>
cudaError_t run_pass(F f, const PassArgs& a, cudaStream_t st) {
    const MapGeom& g = a.g;
    const CorrPlanDev& plan = *a.plan;
    const size_t pstride = (size_t)g.ny * g.WP;
    const int tl = f.tl();
    if constexpr (P == Pass::FwdRows) {
        const int n_cplx = (plan.n_real + 1) / 2;
        // up to 256 threads of lines (one line of more for the longest rows: 8192 points, 512 threads)
        const int lines = std::min(lines_per_block(tl, 256), n_cplx);
        const size_t sm = (size_t)lines * padded_len(g.nx) * sizeof(float2) + (size_t)6 * g.cw * sizeof(float);
        auto k = 2 * g.cw <= g.nx ? k_fwd_rows<F, true> : k_fwd_rows<F, false>;
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        k<<<dim3(g.ch, a.batch), lines * tl, sm, st>>>(a.grid, g.cw, g.ch, g.WP, plan, f, lines, a.half,
                                                                   pstride, a.grid_stride, a.half_stride);
        return cudaGetLastError();
    } else if constexpr (P == Pass::FwdCols) {
        const int ncols = g.nx / 2 + 1;
        const int tx = col_tile(g.ny, tl, ncols);
        const size_t sm = (size_t)tx * col_pitch(g.ny, tx) * sizeof(float2);
        auto k = 2 * g.ch <= g.ny ? k_cols<F, false, true> : k_cols<F, false, false>;
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        k<<<dim3((ncols + tx - 1) / tx, plan.n_real * a.batch), tx * tl, sm, st>>>(
            a.half, pstride, g.WP, ncols, g.ch, f, tx);
        return cudaGetLastError();
    } else if constexpr (P == Pass::InvCols) {
        const int ncols = g.nx / 2 + 1;
        constexpr int NF = FixedN<F>::value;
        if constexpr (NF == 1024 || NF == 2048) {
            if (a.batch == 1 && tl == NF / 16) {
                const int tx = 512 / tl;
                const size_t sm = (size_t)tx * line_pitch(NF) * sizeof(float2);
                const int nitems = plan.n_corr * ((ncols + tx - 1) / tx);
                int dev = 0, sms = 148;
                cudaGetDevice(&dev);
                cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
                cudaFuncSetAttribute(k_inv_cols_pipe<NF>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
                k_inv_cols_pipe<NF><<<std::min(nitems, sms), 512, sm, st>>>(a.half, a.half_b, pstride, g.WP, ncols, plan,
                                                                            f.tw, tx, a.Q, nitems);
                return cudaGetLastError();
            }
        }
        const int tx = col_tile(g.ny, tl, ncols);
        const size_t sm = (size_t)tx * col_pitch(g.ny, tx) * sizeof(float2);
        cudaFuncSetAttribute(k_inv_cols<F>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        k_inv_cols<F><<<dim3(plan.n_corr, (ncols + tx - 1) / tx, a.batch), tx * tl, sm, st>>>(
            a.half, a.half_b, pstride, g.WP, ncols, plan, f, tx, a.Q, a.half_stride, a.b_stride, a.q_stride);
        return cudaGetLastError();
    } else {
        const CombineParams& cp = *a.cp;
        if (cp.nf == 1) return launch_rows<F, 1, false, false, SPLIT>(f, a, st);
        if (cp.nf == 4) {
            if (!cp.exact) return launch_rows<F, 4, false, false, SPLIT>(f, a, st);
            if (cp.calib) return launch_rows<F, 4, true, true, SPLIT>(f, a, st);
            return launch_rows<F, 4, true, false, SPLIT>(f, a, st);
        }
        if (!cp.exact) return launch_rows<F, 3, false, false, SPLIT>(f, a, st);
        if (cp.calib) return launch_rows<F, 3, true, true, SPLIT>(f, a, st);
        return launch_rows<F, 3, true, false, SPLIT>(f, a, st);
    }
}

// A pass with the compile-time line of length N: N/16 threads per line for the forward passes
// and the inverse columns, N/8 for the row pass.
template <int N, bool SPLIT>
cudaError_t run_fixed(Pass p, const float2* tw, const PassArgs& a, cudaStream_t st) {
    switch (p) {
        case Pass::FwdRows: return run_pass<Pass::FwdRows, FixedLine<N, N / 16>, SPLIT>(FixedLine<N, N / 16>{tw}, a, st);
        case Pass::FwdCols: return run_pass<Pass::FwdCols, FixedLine<N, N / 16>, SPLIT>(FixedLine<N, N / 16>{tw}, a, st);
        case Pass::InvCols: return run_pass<Pass::InvCols, FixedLine<N, N / 16>, SPLIT>(FixedLine<N, N / 16>{tw}, a, st);
        default: return run_pass<Pass::Rows, FixedLine<N, row_tpl(N)>, SPLIT>(FixedLine<N, row_tpl(N)>{tw}, a, st);
    }
}

}  // namespace

// the translation units that instantiate the fixed lines; each returns false for lengths it
// does not carry
bool pass_lines_a(Pass p, const LinePlan& L, const PassArgs& a, cudaStream_t st, cudaError_t* e);
bool pass_lines_b(Pass p, const LinePlan& L, const PassArgs& a, cudaStream_t st, cudaError_t* e);
bool pass_lines_c(Pass p, const LinePlan& L, const PassArgs& a, cudaStream_t st, cudaError_t* e);

}  // namespace zc
