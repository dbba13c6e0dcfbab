// Pose scores and gradients on the GPU: the 45 overlap moment sums of many poses at once, the
// score and its gradient coefficients (float64), and the tangent gradient with the Gauss–Newton
// matrix. Restated from the reference's shaders/smi.wgsl (overlap_moments 977-1057, taper
// 336-351, boundary_value 353-366, score_dva 1059-1081, tangent_grad 1123-1272) and
// src/moments.zig (scoreFromMoments 91-172).
//
// One direction warps image a (moving) onto image b (fixed): every b pixel x samples a's
// features bilinearly at H⁻¹(x + 1) − 1, weighted by a 2-px ramp inside a's valid border. Blocks
// of pose p sum their pixels in float32 per thread, then float64 across the block; the pose's
// blocks' totals are added in block order by the last of them to finish (block_add).
#include <array>
#include <atomic>
#include <algorithm>

#include "common.cuh"
#include "kernels.hpp"

namespace zc {
namespace {

constexpr float kTaper = 2.0f;
constexpr int kMom = 45, kCoef = 102, kG0 = 40, kQ0 = 85, kGrad = 44;

__device__ __forceinline__ int tri4(int i, int j) {
    const int a = min(i, j), b = max(i, j);
    return a * 4 - (a * (a + 1)) / 2 + b;
}

// The block's k ≤ 48 float64 totals (thread t < k holds total t; the others pass anything) added
// into out[0 .. k) of this pose. With r.part: every block stores its totals at
// part[(pose · blocks + block) · k], then the pose's last block to finish (the old value of its
// ticket is blocks − 1) adds them in a fixed order — group g of ⌊256 / k⌋ threads takes blocks
// g, g + groups, …, and thread t adds the groups' totals 0, 1, … — and puts the ticket back to
// 0. Every thread of the block calls it. Without r.part: float64 atomics.
__device__ void block_add(double s, int k, double* __restrict__ out, const PoseRed& r, int pose) {
    const int t = threadIdx.x, nblk = gridDim.x;
    if (!r.part) {
        if (t < k) atomicAdd(&out[t], s);
        return;
    }
    __shared__ int last;
    __shared__ double grp[8][48];
    double* part = r.part + (size_t)pose * nblk * k;
    if (t < k) part[(size_t)blockIdx.x * k + t] = s;
    __threadfence();
    __syncthreads();
    if (t == 0) last = atomicAdd(&r.ticket[pose], 1u) == (unsigned)(nblk - 1);
    __syncthreads();
    if (!last) return;  // uniform over the block
    __threadfence();
    const int ng = min((int)blockDim.x / k, 8), g = t / k, e = t - g * k;
    if (g < ng) {
        double a = 0.0;
        for (int b = g; b < nblk; b += ng) a += __ldcg(&part[(size_t)b * k + e]);
        grp[g][e] = a;
    }
    __syncthreads();
    if (t < k) {
        double a = 0.0;
        for (int q = 0; q < ng; ++q) a += grp[q][t];
        out[t] = a;
    }
    if (t == 0) r.ticket[pose] = 0;
}

// (w, ∂w/∂fx, ∂w/∂fy) of the border taper at (fx, fy) in a w×h image
__device__ __forceinline__ void taper(float fx, float fy, float w, float h, float& t, float& tx, float& ty) {
    auto ramp = [](float v, float lo, float hi, float& val, float& dv) {
        const float a = (v - lo) / kTaper, b = (hi - v) / kTaper;
        const float ca = fminf(fmaxf(a, 0.f), 1.f), cb = fminf(fmaxf(b, 0.f), 1.f);
        const float da = (a > 0.f && a < 1.f) ? 1.f / kTaper : 0.f;
        const float db = (b > 0.f && b < 1.f) ? -1.f / kTaper : 0.f;
        val = ca * cb;
        dv = da * cb + ca * db;
    };
    float vx, dx, vy, dy;
    ramp(fx, 2.f, w - 3.f, vx, dx);
    ramp(fy, 2.f, h - 3.f, vy, dy);
    t = vx * vy;
    tx = dx * vy;
    ty = vx * dy;
}

// ── the B-spline (smi.wgsl:198-240 cubic_w, dest_half, ffd_disp) ──

constexpr int kFfdMax = 16;  // lattice side (src/pose.zig:17 FFD_MAX)

__device__ __forceinline__ float4 cubic_w(float t) {
    const float t2 = t * t, t3 = t2 * t;
    return make_float4((1.f - t) * (1.f - t) * (1.f - t) / 6.f, (3.f * t3 - 6.f * t2 + 4.f) / 6.f,
                       (-3.f * t3 + 3.f * t2 + 3.f * t + 1.f) / 6.f, t3 / 6.f);
}
__device__ __forceinline__ float comp4(const float4& v, int i) { return i == 0 ? v.x : i == 1 ? v.y : i == 2 ? v.z : v.w; }

// The 2×2 taps at i00, i00 + 1, i00 + aw, i00 + aw + 1 of an image whose four feature planes are
// interleaved (one float4 per pixel): one 16-byte load per tap instead of one per plane and tap.
struct Taps4 {
    float4 v00, v10, v01, v11;
};
__device__ __forceinline__ Taps4 taps4(const float4* __restrict__ a, size_t i00, int aw) {
    return {__ldg(&a[i00]), __ldg(&a[i00 + 1]), __ldg(&a[i00 + aw]), __ldg(&a[i00 + aw + 1])};
}

// A block's view of a spline: its control points staged in shared memory (c null: none).
struct FfdView {
    const float* c;
    int g, source;
};

// stage pose `pose`'s control points (all threads call it; a __syncthreads must follow)
__device__ __forceinline__ FfdView ffd_view(const PoseFfd& f, float* sh, int pose = 0) {
    if (!f.cps || f.g < 2) return FfdView{nullptr, 0, 0};
    const float* c = f.cps + (size_t)pose * f.stride;
    for (int i = threadIdx.x; i < 2 * f.g * f.g; i += blockDim.x) sh[i] = c[i];
    return FfdView{sh, f.g, f.source};
}

// the displacement (pixels) at the 0-based point (xf, yf) of the lattice's rw × rh image: 0
// outside it; half-image units scaled by (rw/2, rh/2); clamped lattice indices
__device__ __forceinline__ float2 ffd_disp(const FfdView& f, float xf, float yf, float rw, float rh) {
    if (xf < 0.f || yf < 0.f || xf > rw - 1.f || yf > rh - 1.f) return make_float2(0.f, 0.f);
    const int g = f.g;
    const float hx = fmaxf(rw, 1.f) * 0.5f, hy = fmaxf(rh, 1.f) * 0.5f;
    const float spx = fmaxf(rw - 1.f, 1.f) / (float)(g - 1), spy = fmaxf(rh - 1.f, 1.f) / (float)(g - 1);
    const float su = xf / spx, sv = yf / spy;
    const int iu = (int)floorf(su), iv = (int)floorf(sv);
    const float4 bu = cubic_w(fminf(fmaxf(su - (float)iu, 0.f), 1.f));
    const float4 bv = cubic_w(fminf(fmaxf(sv - (float)iv, 0.f), 1.f));
    float dx = 0.f, dy = 0.f;
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) {
        const int j = min(max(iv - 1 + jj, 0), g - 1);
#pragma unroll
        for (int ii = 0; ii < 4; ++ii) {
            const int i = min(max(iu - 1 + ii, 0), g - 1);
            const float w = comp4(bu, ii) * comp4(bv, jj);
            const int o = (j * g + i) * 2;
            dx = dx + w * (f.c[o] * hx);
            dy = dy + w * (f.c[o + 1] * hy);
        }
    }
    return make_float2(dx, dy);
}

// A grid-stride walk over a w × h image in tiles of 8 × 4 pixels, one tile per warp and step
// (lane → (lane mod 8, lane / 8)): a warp's 32 pixels are a compact patch, so the bilinear taps
// they gather on the other image under any rotation fall on few rows (few sectors per load).
// Tile coordinates are stepped along, not divided out per tile.
struct TileWalk {
    int T, nt, step, tx, ty, sx, sy, ntx, lx, ly, w, h;
    __device__ __forceinline__ TileWalk(int w_, int h_) : w(w_), h(h_) {
        ntx = (w + 7) >> 3;
        nt = ntx * ((h + 3) >> 2);
        const int lane = threadIdx.x & 31;
        lx = lane & 7;
        ly = lane >> 3;
        T = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
        step = (int)((gridDim.x * blockDim.x) >> 5);
        ty = T / ntx;
        tx = T - ty * ntx;
        sy = step / ntx;
        sx = step - sy * ntx;
    }
    __device__ __forceinline__ bool ok() const { return T < nt; }
    __device__ __forceinline__ void next() {
        T += step;
        tx += sx;
        ty += sy;
        if (tx >= ntx) {
            tx -= ntx;
            ++ty;
        }
    }
    __device__ __forceinline__ int x() const { return (tx << 3) + lx; }
    __device__ __forceinline__ int y() const { return (ty << 2) + ly; }
    __device__ __forceinline__ bool in() const { return x() < w && y() < h; }
};

// pose sample position of b pixel (x, y) (smi.wgsl overlap_moments 1003-1016): with a spline on
// b the pixel moves first, X = (x + 1 + dx, y + 1 + dy); on a the sample H⁻¹X − 1 moves after.
// ph = H⁻¹X, (Xx, Xy) = X. False when outside a's valid interior.
template <bool FFD>
__device__ __forceinline__ bool sample_pos(const float* Hi, const FfdView& f, int x, int y, int aw, int ah, int bw,
                                           int bh, float& fx, float& fy, float3& ph, float& Xx, float& Xy) {
    Xx = (float)x + 1.f;
    Xy = (float)y + 1.f;
    if (FFD && !f.source) {
        const float2 d = ffd_disp(f, (float)x, (float)y, (float)bw, (float)bh);
        Xx = (float)x + 1.f + d.x;
        Xy = (float)y + 1.f + d.y;
    }
    ph.x = Hi[0] * Xx + Hi[1] * Xy + Hi[2];
    ph.y = Hi[3] * Xx + Hi[4] * Xy + Hi[5];
    ph.z = Hi[6] * Xx + Hi[7] * Xy + Hi[8];
    if (fabsf(ph.z) < 1e-8f) return false;
    if (ph.z == 1.f) {  // affine poses: the division is exact, skip it
        fx = ph.x - 1.f;
        fy = ph.y - 1.f;
    } else {
        fx = ph.x / ph.z - 1.f;
        fy = ph.y / ph.z - 1.f;
    }
    if (FFD && f.source) {
        const float2 d = ffd_disp(f, fx, fy, (float)aw, (float)ah);
        fx = fx + d.x;
        fy = fy + d.y;
    }
    return !(fx < 2.f || fy < 2.f || fx > (float)aw - 3.f || fy > (float)ah - 3.f);
}

// The 45 sums: 0 Σw, 1–4 Σw a, 5–8 Σw b, 9–24 Σw a_i b_j, 25–34 / 35–44 upper triangles of
// Σw a aᵀ and Σw b bᵀ.
template <bool FFD>
__global__ void __launch_bounds__(256, FFD ? 2 : 3) k_pose_moments(const float4* __restrict__ fa, int aw, int ah,
                                                      const float4* __restrict__ fb, int bw, int bh,
                                                      const float* __restrict__ hinv, double* __restrict__ sums,
                                                      PoseFfd ffd, const unsigned char* __restrict__ mask, PoseRed rd) {
    __shared__ float Hs[9];
    __shared__ float red[8][kMom];
    __shared__ float cps[2 * kFfdMax * kFfdMax];
    const int pose = blockIdx.y;
    if (mask && !mask[pose]) return;  // a pose nobody reads (its sums stay 0)
    if (threadIdx.x < 9) Hs[threadIdx.x] = hinv[pose * 9 + threadIdx.x];
    const FfdView fv = ffd_view(ffd, cps, pose);
    __syncthreads();
    float Hi[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) Hi[i] = Hs[i];
    float acc[kMom];
#pragma unroll
    for (int k = 0; k < kMom; ++k) acc[k] = 0.f;
    for (TileWalk pw(bw, bh); pw.ok(); pw.next()) {
        if (!pw.in()) continue;
        const int y = pw.y(), x = pw.x();
        const size_t t = (size_t)y * bw + x;
        float fx, fy, Xx, Xy;
        float3 ph;
        if (!sample_pos<FFD>(Hi, fv, x, y, aw, ah, bw, bh, fx, fy, ph, Xx, Xy)) continue;
        float wt, d1, d2;
        taper(fx, fy, (float)aw, (float)ah, wt, d1, d2);
        if (wt <= 0.f) continue;
        const float flx = floorf(fx), fly = floorf(fy);
        const float ax = fx - flx, ay = fy - fly;
        const size_t i00 = (size_t)(int)fly * aw + (int)flx;  // fx, fy ≥ 2 here
        float va[4], vb[4];
        const Taps4 tp = taps4(fa, i00, aw);
        const float4 b4 = __ldg(&fb[t]);
#pragma unroll
        for (int p = 0; p < 4; ++p) {
            const float v00 = comp4(tp.v00, p), v10 = comp4(tp.v10, p);
            const float v01 = comp4(tp.v01, p), v11 = comp4(tp.v11, p);
            va[p] = (v00 * (1.f - ax) + v10 * ax) * (1.f - ay) + (v01 * (1.f - ax) + v11 * ax) * ay;
            vb[p] = comp4(b4, p);
        }
        acc[0] += wt;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const float wa = wt * va[i], wb = wt * vb[i];
            acc[1 + i] += wa;
            acc[5 + i] += wb;
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[9 + i * 4 + j] += wa * vb[j];
#pragma unroll
            for (int j = i; j < 4; ++j) {
                acc[25 + tri4(i, j)] += wa * va[j];
                acc[35 + tri4(i, j)] += wb * vb[j];
            }
        }
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < kMom; ++k) {
        const float v = warp_sumf(acc[k]);
        if (lane == 0) red[w][k] = v;
    }
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x < kMom)
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) s += (double)red[i][threadIdx.x];
    block_add(s, kMom, sums + (size_t)pose * kMom, rd, pose);
}

// scoreFromMoments (src/moments.zig:91-172) in float64, one thread per pose: the score and the
// 102 coefficients [W 0–15, μ_B 16–19, M̂ 20–35, μ_A 36–39, g = ∂S/∂sums 40–84, Q 85–100, flag]
// the tangent pass reads (zero when the overlap is under 12 or a whitening fails).
__device__ bool chol4(const double* G, double* L) {
    for (int i = 0; i < 16; ++i) L[i] = 0.0;
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j <= i; ++j) {
            double s = G[i * 4 + j];
            for (int k = 0; k < j; ++k) s -= L[i * 4 + k] * L[j * 4 + k];
            if (i == j) {
                if (!(s > 0.0)) return false;
                L[i * 5] = sqrt(s);
            } else {
                L[i * 4 + j] = s / L[j * 5];
            }
        }
    return true;
}

__device__ void chol_inv4(const double* L, double* X) {
    for (int c = 0; c < 4; ++c) {
        double y[4];
        for (int i = 0; i < 4; ++i) {
            double s = (i == c) ? 1.0 : 0.0;
            for (int k = 0; k < i; ++k) s -= L[i * 4 + k] * y[k];
            y[i] = s / L[i * 5];
        }
        for (int i = 3; i >= 0; --i) {
            double s = y[i];
            for (int k = i + 1; k < 4; ++k) s -= L[k * 4 + i] * X[k * 4 + c];
            X[i * 4 + c] = s / L[i * 5];
        }
    }
}

__device__ void mm4(const double* A, const double* B, double* o) {
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
            double s = 0.0;
            for (int k = 0; k < 4; ++k) s += A[i * 4 + k] * B[k * 4 + j];
            o[i * 4 + j] = s;
        }
}

__device__ void tr4(const double* A, double* o) {
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) o[i * 4 + j] = A[j * 4 + i];
}

__global__ void k_pose_coefs(const double* __restrict__ sums, int n, int exact, double ridge, float* __restrict__ coef,
                             double* __restrict__ score) {
    const int pose = blockIdx.x * blockDim.x + threadIdx.x;
    if (pose >= n) return;
    const double* st = sums + pose * kMom;
    float* out = coef + pose * kCoef;
    for (int k = 0; k < kCoef; ++k) out[k] = 0.f;
    score[pose] = 0.0;
    const double nn = st[0];
    if (!(nn >= 12.0)) return;
    double ma[4], mb[4], C[16], W[16], Mh[16] = {0}, Nh[16] = {0};
    for (int i = 0; i < 4; ++i) {
        ma[i] = st[1 + i] / nn;
        mb[i] = st[5 + i] / nn;
    }
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) C[i * 4 + j] = st[9 + i * 4 + j] / nn - ma[i] * mb[j];
    for (int i = 0; i < 16; ++i) W[i] = C[i];
    double phi = 0.0;
    if (!exact) {
        for (int i = 0; i < 16; ++i) phi += C[i] * C[i];
    } else {
        double GA[16], GB[16], LA[16], LB[16], GAi[16], GBi[16], T[16], U[16];
        for (int i = 0; i < 4; ++i)
            for (int j = 0; j < 4; ++j) {
                GA[i * 4 + j] = st[25 + tri4(i, j)] / nn - ma[i] * ma[j];
                GB[i * 4 + j] = st[35 + tri4(i, j)] / nn - mb[i] * mb[j];
            }
        const double ra = ridge * fmax((GA[0] + GA[5] + GA[10] + GA[15]) / 4, 1e-12);
        const double rb = ridge * fmax((GB[0] + GB[5] + GB[10] + GB[15]) / 4, 1e-12);
        for (int i = 0; i < 4; ++i) {
            GA[i * 5] += ra;
            GB[i * 5] += rb;
        }
        if (!chol4(GA, LA) || !chol4(GB, LB)) return;
        chol_inv4(LA, GAi);
        chol_inv4(LB, GBi);
        mm4(GAi, C, T);
        mm4(T, GBi, W);
        for (int i = 0; i < 16; ++i) phi += W[i] * C[i];
        tr4(C, U);
        mm4(W, U, T);
        mm4(T, GAi, Mh);
        tr4(W, U);
        mm4(U, C, T);
        mm4(T, GBi, Nh);
        const double tm = (Mh[0] + Mh[5] + Mh[10] + Mh[15]) * ridge / 4;
        const double tn = (Nh[0] + Nh[5] + Nh[10] + Nh[15]) * ridge / 4;
        for (int i = 0; i < 4; ++i) {
            Mh[i * 5] += tm;
            Nh[i * 5] += tn;
        }
    }
    const double sc = nn * phi;
    if (!isfinite(sc)) return;
    score[pose] = sc;
    for (int i = 0; i < 16; ++i) {
        out[i] = (float)W[i];
        out[20 + i] = (float)Mh[i];
    }
    for (int i = 0; i < 4; ++i) {
        out[16 + i] = (float)mb[i];
        out[36 + i] = (float)ma[i];
    }
    double g[kMom];
    for (int k = 0; k < kMom; ++k) g[k] = 0.0;
    for (int i = 0; i < 4; ++i) {
        double ga = 0.0, gb = 0.0;
        for (int j = 0; j < 4; ++j) {
            ga += -2 * W[i * 4 + j] * mb[j] + 2 * Mh[i * 4 + j] * ma[j];
            gb += -2 * W[j * 4 + i] * ma[j] + 2 * Nh[i * 4 + j] * mb[j];
            g[9 + i * 4 + j] = 2 * W[i * 4 + j];
        }
        g[1 + i] = ga;
        g[5 + i] = gb;
        for (int j = i; j < 4; ++j) {
            const double f = (i == j) ? 1.0 : 2.0;
            g[25 + tri4(i, j)] = -f * Mh[i * 4 + j];
            g[35 + tri4(i, j)] = -f * Nh[i * 4 + j];
        }
    }
    double rest = 0.0;
    for (int k = 1; k < kMom; ++k) rest += g[k] * st[k];
    g[0] = (sc - rest) / nn;
    for (int k = 0; k < kMom; ++k) out[kG0 + k] = (float)g[k];
    double Q[16];
    if (exact) {
        for (int i = 0; i < 16; ++i) Q[i] = Mh[i];
    } else {
        double Ct[16];
        tr4(C, Ct);
        mm4(C, Ct, Q);
    }
    for (int i = 0; i < 16; ++i) out[kQ0 + i] = (float)Q[i];
}

// The gradient over the tangent coordinates and (hess) the Gauss–Newton matrix Σ wt·J_aᵀ Q J_a:
// per pose 44 sums (8 gradient, then the 8×8 upper triangle row by row). Per pixel the gradient
// needs the two scalars cx, cy = (∂S/∂v_a)·∇v_a plus the taper's boundary term, times each
// tangent's flow ∂(sample)/∂ξ_k = ((M_k X)·ph.z − ph·(M_k X).z)/ph.z², M_k = −H⁻¹ G_k.
template <bool FFD>
__global__ void __launch_bounds__(256) k_pose_tangent(const float4* __restrict__ fa, int aw, int ah,
                                                      const float4* __restrict__ fb, int bw, int bh,
                                                      const float* __restrict__ hinv, const float* __restrict__ coef,
                                                      const float* __restrict__ gens, int hess, double* __restrict__ out,
                                                      PoseFfd ffd, const unsigned char* __restrict__ mask, PoseRed rd) {
    __shared__ float Hs[9], Mk[8][9], cf[kCoef];
    __shared__ float red[8][kGrad];
    __shared__ float cps[2 * kFfdMax * kFfdMax];
    const int pose = blockIdx.y;
    if (mask && !mask[pose]) return;  // a pose nobody reads (its sums stay 0)
    if (threadIdx.x < 9) Hs[threadIdx.x] = hinv[pose * 9 + threadIdx.x];
    for (int k = threadIdx.x; k < kCoef; k += blockDim.x) cf[k] = coef[pose * kCoef + k];
    const FfdView fv = ffd_view(ffd, cps, pose);
    __syncthreads();
    if (threadIdx.x < 72) {
        const int k = threadIdx.x / 9, e = threadIdx.x % 9, r = e / 3, c = e % 3;
        const float* G = gens + k * 9;
        Mk[k][e] = -(Hs[r * 3] * G[c] + Hs[r * 3 + 1] * G[3 + c] + Hs[r * 3 + 2] * G[6 + c]);
    }
    __syncthreads();
    float Hi[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) Hi[i] = Hs[i];
    float g8[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    float h36[36];
#pragma unroll
    for (int k = 0; k < 36; ++k) h36[k] = 0.f;
    for (TileWalk pw(bw, bh); pw.ok(); pw.next()) {
        if (!pw.in()) continue;
        const int y = pw.y(), x = pw.x();
        const size_t t = (size_t)y * bw + x;
        float fx, fy, X, Y;
        float3 ph;
        if (!sample_pos<FFD>(Hi, fv, x, y, aw, ah, bw, bh, fx, fy, ph, X, Y)) continue;
        float wt, tpx, tpy;
        taper(fx, fy, (float)aw, (float)ah, wt, tpx, tpy);
        const float flx = floorf(fx), fly = floorf(fy);
        const float ax = fx - flx, ay = fy - fly;
        const size_t i00 = (size_t)(int)fly * aw + (int)flx;  // fx, fy ≥ 2 here
        float va[4], gx[4], gy[4], vb[4];
        const Taps4 tp = taps4(fa, i00, aw);
        const float4 b4 = __ldg(&fb[t]);
#pragma unroll
        for (int p = 0; p < 4; ++p) {
            const float v00 = comp4(tp.v00, p), v10 = comp4(tp.v10, p);
            const float v01 = comp4(tp.v01, p), v11 = comp4(tp.v11, p);
            va[p] = (v00 * (1.f - ax) + v10 * ax) * (1.f - ay) + (v01 * (1.f - ax) + v11 * ax) * ay;
            gx[p] = (v10 - v00) * (1.f - ay) + (v11 - v01) * ay;
            gy[p] = (v01 - v00) * (1.f - ax) + (v11 - v10) * ax;
            vb[p] = comp4(b4, p);
        }
        // ∂S/∂v_a = 2 (W (v_b − μ_B) − M̂ (v_a − μ_A))
        float ra[4];
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            float s = 0.f;
#pragma unroll
            for (int b = 0; b < 4; ++b) s += cf[a * 4 + b] * (vb[b] - cf[16 + b]) - cf[20 + a * 4 + b] * (va[b] - cf[36 + b]);
            ra[a] = 2.f * s;
        }
        // the taper's boundary term: Σ_k g_k φ_k(v_a, v_b)
        float bwv = 0.f;
        if (tpx != 0.f || tpy != 0.f) {
            const float* g = cf + kG0;
            float s = g[0];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                s += g[1 + i] * va[i] + g[5 + i] * vb[i];
#pragma unroll
                for (int j = 0; j < 4; ++j) s += g[9 + i * 4 + j] * va[i] * vb[j];
#pragma unroll
                for (int j = i; j < 4; ++j) s += g[25 + tri4(i, j)] * va[i] * va[j] + g[35 + tri4(i, j)] * vb[i] * vb[j];
            }
            bwv = s;
        }
        float dga = 0.f, dgb = 0.f;
#pragma unroll
        for (int p = 0; p < 4; ++p) {
            dga += ra[p] * gx[p];
            dgb += ra[p] * gy[p];
        }
        const float cx = wt * dga + bwv * tpx, cy = wt * dgb + bwv * tpy;
        const float iz2 = 1.f / fmaxf(ph.z * ph.z, 1e-12f);
        float px[8], py[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const float* M = Mk[k];
            const float wx = M[0] * X + M[1] * Y + M[2];
            const float wy = M[3] * X + M[4] * Y + M[5];
            const float wz = M[6] * X + M[7] * Y + M[8];
            px[k] = (wx * ph.z - ph.x * wz) * iz2;
            py[k] = (wy * ph.z - ph.y * wz) * iz2;
            g8[k] += cx * px[k] + cy * py[k];
        }
        if (hess) {
            float qgx[4], qgy[4];
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                float sx = 0.f, sy = 0.f;
#pragma unroll
                for (int b = 0; b < 4; ++b) {
                    sx += cf[kQ0 + a * 4 + b] * gx[b];
                    sy += cf[kQ0 + a * 4 + b] * gy[b];
                }
                qgx[a] = sx;
                qgy[a] = sy;
            }
            float sxx = 0.f, sxy = 0.f, syx = 0.f, syy = 0.f;
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                sxx += gx[a] * qgx[a];
                sxy += gx[a] * qgy[a];
                syx += gy[a] * qgx[a];
                syy += gy[a] * qgy[a];
            }
            int h = 0;
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const float rk = wt * (sxx * px[k] + syx * py[k]);
                const float sk = wt * (sxy * px[k] + syy * py[k]);
#pragma unroll
                for (int l = k; l < 8; ++l) h36[h++] += rk * px[l] + sk * py[l];
            }
        }
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const float v = warp_sumf(g8[k]);
        if (lane == 0) red[w][k] = v;
    }
#pragma unroll
    for (int k = 0; k < 36; ++k) {
        const float v = warp_sumf(h36[k]);
        if (lane == 0) red[w][8 + k] = v;
    }
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x < kGrad)
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) s += (double)red[i][threadIdx.x];
    block_add(s, kGrad, out + (size_t)pose * kGrad, rd, pose);
}

// ∂score/∂(control points cp0 .. cp0 + 15) of pose 0 (smi.wgsl ffd_grad 1275-1417): per valid
// pixel the two scalars Gx, Gy — (∂S/∂v_a)·∇v_a and the taper's boundary term along the sample's
// motion under a unit x or y displacement of one control point (through H⁻¹ on a b lattice,
// directly on an a lattice), per unit basis weight — then each control point of the chunk takes
// its basis weight B_i(u) B_j(v) (clamped lattice indices summed) times them.
__global__ void __launch_bounds__(256) k_pose_ffd_grad(const float4* __restrict__ fa, int aw, int ah,
                                                       const float4* __restrict__ fb, int bw, int bh,
                                                       const float* __restrict__ hinv, const float* __restrict__ coef,
                                                       PoseFfd ffd, int cp0, double* __restrict__ out, PoseRed rd) {
    __shared__ float Hs[9], cf[kCoef];
    __shared__ float red[8][32];
    __shared__ float cps[2 * kFfdMax * kFfdMax];
    if (threadIdx.x < 9) Hs[threadIdx.x] = hinv[threadIdx.x];
    for (int k = threadIdx.x; k < kCoef; k += blockDim.x) cf[k] = coef[k];
    const FfdView fv = ffd_view(ffd, cps);
    __syncthreads();
    float Hi[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) Hi[i] = Hs[i];
    const int g = fv.g;
    const bool src = fv.source != 0;
    const float lw = src ? (float)aw : (float)bw, lh = src ? (float)ah : (float)bh;
    const float hx = fmaxf(lw, 1.f) * 0.5f, hy = fmaxf(lh, 1.f) * 0.5f;
    const float spx = fmaxf(lw - 1.f, 1.f) / (float)(g - 1), spy = fmaxf(lh - 1.f, 1.f) / (float)(g - 1);
    float acc[32];
#pragma unroll
    for (int k = 0; k < 32; ++k) acc[k] = 0.f;
    for (TileWalk pw(bw, bh); pw.ok(); pw.next()) {
        if (!pw.in()) continue;
        const int y = pw.y(), x = pw.x();
        const size_t t = (size_t)y * bw + x;
        float fx, fy, X, Y;
        float3 ph;
        if (!sample_pos<true>(Hi, fv, x, y, aw, ah, bw, bh, fx, fy, ph, X, Y)) continue;
        float wt, tpx, tpy;
        taper(fx, fy, (float)aw, (float)ah, wt, tpx, tpy);
        const float flx = floorf(fx), fly = floorf(fy);
        const float ax = fx - flx, ay = fy - fly;
        const size_t i00 = (size_t)(int)fly * aw + (int)flx;  // fx, fy ≥ 2 here
        float va[4], gx[4], gy[4], vb[4];
        const Taps4 tp = taps4(fa, i00, aw);
        const float4 b4 = __ldg(&fb[t]);
#pragma unroll
        for (int p = 0; p < 4; ++p) {
            const float v00 = comp4(tp.v00, p), v10 = comp4(tp.v10, p);
            const float v01 = comp4(tp.v01, p), v11 = comp4(tp.v11, p);
            va[p] = (v00 * (1.f - ax) + v10 * ax) * (1.f - ay) + (v01 * (1.f - ax) + v11 * ax) * ay;
            gx[p] = (v10 - v00) * (1.f - ay) + (v11 - v01) * ay;
            gy[p] = (v01 - v00) * (1.f - ax) + (v11 - v10) * ax;
            vb[p] = comp4(b4, p);
        }
        float dga = 0.f, dgb = 0.f;
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            float s = 0.f;
#pragma unroll
            for (int b = 0; b < 4; ++b) s += cf[a * 4 + b] * (vb[b] - cf[16 + b]) - cf[20 + a * 4 + b] * (va[b] - cf[36 + b]);
            dga += 2.f * s * gx[a];
            dgb += 2.f * s * gy[a];
        }
        float bwv = 0.f;
        if (tpx != 0.f || tpy != 0.f) {
            const float* gg = cf + kG0;
            float s = gg[0];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                s += gg[1 + i] * va[i] + gg[5 + i] * vb[i];
#pragma unroll
                for (int j = 0; j < 4; ++j) s += gg[9 + i * 4 + j] * va[i] * vb[j];
#pragma unroll
                for (int j = i; j < 4; ++j) s += gg[25 + tri4(i, j)] * va[i] * va[j] + gg[35 + tri4(i, j)] * vb[i] * vb[j];
            }
            bwv = s;
        }
        // the sample's motion per unit basis weight of a control point's x / y displacement
        float uxx, uxy, uyx, uyy;
        float su, sv;
        if (src) {
            uxx = hx, uxy = 0.f, uyx = 0.f, uyy = hy;
            su = (ph.x / ph.z - 1.f) / spx;
            sv = (ph.y / ph.z - 1.f) / spy;
        } else {
            const float z = ph.z, z2 = fmaxf(z * z, 1e-12f);
            uxx = hx * (Hi[0] * z - ph.x * Hi[6]) / z2;
            uxy = hx * (Hi[3] * z - ph.y * Hi[6]) / z2;
            uyx = hy * (Hi[1] * z - ph.x * Hi[7]) / z2;
            uyy = hy * (Hi[4] * z - ph.y * Hi[7]) / z2;
            su = (float)x / spx;
            sv = (float)y / spy;
        }
        const float Gx = wt * (dga * uxx + dgb * uxy) + bwv * (tpx * uxx + tpy * uxy);
        const float Gy = wt * (dga * uyx + dgb * uyy) + bwv * (tpx * uyx + tpy * uyy);
        if (!(Gx == Gx) || !(Gy == Gy)) continue;
        const int iu = (int)floorf(su), iv = (int)floorf(sv);
        const float4 bu = cubic_w(fminf(fmaxf(su - (float)iu, 0.f), 1.f));
        const float4 bv = cubic_w(fminf(fmaxf(sv - (float)iv, 0.f), 1.f));
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            const int cp = cp0 + k;
            if (cp >= g * g) break;
            const int ci = cp % g, cj = cp / g;
            float wu = 0.f, wv = 0.f;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                if (min(max(iu - 1 + q, 0), g - 1) == ci) wu += comp4(bu, q);
                if (min(max(iv - 1 + q, 0), g - 1) == cj) wv += comp4(bv, q);
            }
            const float bk = wu * wv;
            acc[2 * k] += bk * Gx;
            acc[2 * k + 1] += bk * Gy;
        }
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 32; ++k) {
        const float v = warp_sumf(acc[k]);
        if (lane == 0) red[w][k] = v;
    }
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x < 32)
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) s += (double)red[i][threadIdx.x];
    block_add(s, 32, out, rd, 0);
}

// The spline's Gauss–Newton terms of one lattice cell (smi.wgsl ffd_cells 2065-2264): block =
// (cell, chunk of its pixel tiles). The cell's fixed pixels (the cell itself on a fixed-image
// lattice; the bounding box of the moving cell's corners under H, one pixel wider, on a
// moving-image lattice) in tiles of 256: each thread stages one pixel that samples inside the
// moving image and whose lattice point lies in this cell — its basis weights, K = wt·Jdᵀ S Jd
// (S = ∇vᵀ Q ∇v, Jd the sample's motion per unit control-point displacement) and the
// gradient Jdᵀ (wt ∇S + the taper term) — then thread (task, half) adds its share of the tile:
// tasks 0–99 a pair of symmetric basis products × (K_xx, K_xy, K_yy), 100–115 a tap × ∇.
constexpr int kFcTasks = 116;
__device__ __forceinline__ int tri_i(int k) { return k < 4 ? 0 : k < 7 ? 1 : k < 9 ? 2 : 3; }
__device__ __forceinline__ int tri_j(int k) { return k < 4 ? k : k < 7 ? k - 3 : k < 9 ? k - 5 : 3; }

__global__ void __launch_bounds__(256) k_pose_ffd_cells(const float4* __restrict__ fa, int aw, int ah,
                                                        const float4* __restrict__ fb, int bw, int bh,
                                                        const float* __restrict__ hinv, const float* __restrict__ hpose,
                                                        const float* __restrict__ coef, PoseFfd ffd, int nch,
                                                        float* __restrict__ out) {
    __shared__ float Hs[9], Hp[9], cf[kCoef];
    __shared__ float cps[2 * kFfdMax * kFfdMax];
    __shared__ float4 s_bu[256], s_bv[256], s_k[256];
    __shared__ float s_gy[256];
    __shared__ float3 s_acc[256];
    if (threadIdx.x < 9) {
        Hs[threadIdx.x] = hinv[threadIdx.x];
        Hp[threadIdx.x] = hpose[threadIdx.x];
    }
    for (int k = threadIdx.x; k < kCoef; k += blockDim.x) cf[k] = coef[k];
    const FfdView fv = ffd_view(ffd, cps);
    __syncthreads();
    float Hi[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) Hi[i] = Hs[i];
    const int g = fv.g;
    const int cell = blockIdx.x / nch, chunk = blockIdx.x % nch;
    const int iu = cell % g, iv = cell / g;
    const bool src = fv.source != 0;
    const float rw = (float)bw, rh = (float)bh, sw = (float)aw, shh = (float)ah;
    const float lw = src ? sw : rw, lh = src ? shh : rh;
    const float hx = fmaxf(lw, 1.f) * 0.5f, hy = fmaxf(lh, 1.f) * 0.5f;
    const float spx = fmaxf(lw - 1.f, 1.f) / (float)(g - 1), spy = fmaxf(lh - 1.f, 1.f) / (float)(g - 1);
    float x0 = 0.f, x1 = rw - 1.f, y0 = 0.f, y1 = rh - 1.f;
    if (!src) {
        x0 = fmaxf(0.f, floorf((float)iu * spx) - 1.f);
        x1 = fminf(rw - 1.f, ceilf((float)(iu + 1) * spx) + 1.f);
        y0 = fmaxf(0.f, floorf((float)iv * spy) - 1.f);
        y1 = fminf(rh - 1.f, ceilf((float)(iv + 1) * spy) + 1.f);
    } else {
        float bx0 = 3.0e38f, bx1 = -3.0e38f, by0 = 3.0e38f, by1 = -3.0e38f;
        for (int c = 0; c < 4; ++c) {
            const float mx = (float)(iu + (c & 1)) * spx + 1.f, my = (float)(iv + (c >> 1)) * spy + 1.f;
            const float qx = Hp[0] * mx + Hp[1] * my + Hp[2], qy = Hp[3] * mx + Hp[4] * my + Hp[5];
            const float qz = Hp[6] * mx + Hp[7] * my + Hp[8];
            if (fabsf(qz) < 1e-8f) continue;
            bx0 = fminf(bx0, qx / qz - 1.f);
            bx1 = fmaxf(bx1, qx / qz - 1.f);
            by0 = fminf(by0, qy / qz - 1.f);
            by1 = fmaxf(by1, qy / qz - 1.f);
        }
        x0 = fmaxf(0.f, floorf(bx0) - 1.f);
        x1 = fminf(rw - 1.f, ceilf(bx1) + 1.f);
        y0 = fmaxf(0.f, floorf(by0) - 1.f);
        y1 = fminf(rh - 1.f, ceilf(by1) + 1.f);
    }
    const int bwx = (int)fmaxf(x1 - x0 + 1.f, 0.f), bhy = (int)fmaxf(y1 - y0 + 1.f, 0.f);
    const int total = bwx * bhy;
    const int half = threadIdx.x / kFcTasks, task = threadIdx.x % kFcTasks;
    int bi = 0, bi2 = 0, bj = 0, bj2 = 0;
    if (task < 100) {
        bi = tri_i(task / 10), bi2 = tri_j(task / 10), bj = tri_i(task % 10), bj2 = tri_j(task % 10);
    } else {
        bi = (task - 100) % 4, bj = (task - 100) / 4;
    }
    float3 acc = make_float3(0.f, 0.f, 0.f);
    const int ntile = (total + 255) / 256;
    for (int tile = chunk * ntile / nch; tile < (chunk + 1) * ntile / nch; ++tile) {
        const int base = tile * 256, pidx = base + threadIdx.x;
        bool ok = false;
        float4 bu = make_float4(0.f, 0.f, 0.f, 0.f), bv = bu, kk = bu;
        float gyv = 0.f;
        if (pidx < total) {
            const int xi = (int)x0 + pidx % bwx, yi = (int)y0 + pidx / bwx;
            float fx, fy, X, Y, su, sv;
            float3 ph;
            ok = sample_pos<true>(Hi, fv, xi, yi, aw, ah, bw, bh, fx, fy, ph, X, Y);
            if (fabsf(ph.z) >= 1e-8f) {
                if (src) {
                    su = (ph.x / ph.z - 1.f) / spx;
                    sv = (ph.y / ph.z - 1.f) / spy;
                } else {
                    su = (float)xi / spx;
                    sv = (float)yi / spy;
                }
                // this cell's pixels only (each pixel belongs to exactly one cell)
                if ((int)floorf(su) != iu || (int)floorf(sv) != iv) ok = false;
                if (su < 0.f || sv < 0.f || su > (float)(g - 1) || sv > (float)(g - 1)) ok = false;
            } else {
                ok = false;
                su = sv = 0.f;
            }
            if (ok) {
                const size_t t = (size_t)yi * bw + xi;
                float wt, tpx, tpy;
                taper(fx, fy, sw, shh, wt, tpx, tpy);
                const float flx = floorf(fx), fly = floorf(fy);
                const float ax = fx - flx, ay = fy - fly;
                const size_t i00 = (size_t)(int)fly * aw + (int)flx;  // fx, fy ≥ 2 here
                float va[4], gx[4], gy[4], vb[4];
                const Taps4 tp = taps4(fa, i00, aw);
                const float4 b4 = __ldg(&fb[t]);
#pragma unroll
                for (int p = 0; p < 4; ++p) {
                    const float v00 = comp4(tp.v00, p), v10 = comp4(tp.v10, p);
                    const float v01 = comp4(tp.v01, p), v11 = comp4(tp.v11, p);
                    va[p] = (v00 * (1.f - ax) + v10 * ax) * (1.f - ay) + (v01 * (1.f - ax) + v11 * ax) * ay;
                    gx[p] = (v10 - v00) * (1.f - ay) + (v11 - v01) * ay;
                    gy[p] = (v01 - v00) * (1.f - ax) + (v11 - v10) * ax;
                    vb[p] = comp4(b4, p);
                }
                float rx = 0.f, ry = 0.f;
#pragma unroll
                for (int a = 0; a < 4; ++a) {
                    float s = 0.f;
#pragma unroll
                    for (int b = 0; b < 4; ++b) s += cf[a * 4 + b] * (vb[b] - cf[16 + b]) - cf[20 + a * 4 + b] * (va[b] - cf[36 + b]);
                    rx += 2.f * s * gx[a];
                    ry += 2.f * s * gy[a];
                }
                float bwb = 0.f;
                if (tpx != 0.f || tpy != 0.f) {
                    const float* gg = cf + kG0;
                    float s = gg[0];
#pragma unroll
                    for (int i = 0; i < 4; ++i) {
                        s += gg[1 + i] * va[i] + gg[5 + i] * vb[i];
#pragma unroll
                        for (int j = 0; j < 4; ++j) s += gg[9 + i * 4 + j] * va[i] * vb[j];
#pragma unroll
                        for (int j = i; j < 4; ++j) s += gg[25 + tri4(i, j)] * va[i] * va[j] + gg[35 + tri4(i, j)] * vb[i] * vb[j];
                    }
                    bwb = s;
                }
                float j00, j10, j01, j11;
                if (src) {
                    j00 = hx, j10 = 0.f, j01 = 0.f, j11 = hy;
                } else {
                    const float z = ph.z, z2 = fmaxf(z * z, 1e-12f);
                    j00 = hx * (Hi[0] * z - ph.x * Hi[6]) / z2;
                    j10 = hx * (Hi[3] * z - ph.y * Hi[6]) / z2;
                    j01 = hy * (Hi[1] * z - ph.x * Hi[7]) / z2;
                    j11 = hy * (Hi[4] * z - ph.y * Hi[7]) / z2;
                }
                float sxx = 0.f, sxy = 0.f, syy = 0.f;
#pragma unroll
                for (int a = 0; a < 4; ++a) {
                    float qx = 0.f, qy = 0.f;
#pragma unroll
                    for (int b = 0; b < 4; ++b) {
                        qx += cf[kQ0 + a * 4 + b] * gx[b];
                        qy += cf[kQ0 + a * 4 + b] * gy[b];
                    }
                    sxx += gx[a] * qx;
                    sxy += gx[a] * qy;
                    syy += gy[a] * qy;
                }
                const float px = wt * rx + bwb * tpx, py = wt * ry + bwb * tpy;
                const float gxv = j00 * px + j10 * py;
                gyv = j01 * px + j11 * py;
                const float a0 = sxx * j00 + sxy * j10, a1 = sxy * j00 + syy * j10;
                const float b0 = sxx * j01 + sxy * j11, b1 = sxy * j01 + syy * j11;
                kk = make_float4(wt * (j00 * a0 + j10 * a1), wt * (j00 * b0 + j10 * b1), wt * (j01 * b0 + j11 * b1), gxv);
                bu = cubic_w(fminf(fmaxf(su - floorf(su), 0.f), 1.f));
                bv = cubic_w(fminf(fmaxf(sv - floorf(sv), 0.f), 1.f));
                if (!(fabsf(kk.x) + fabsf(kk.y) + fabsf(kk.z) + fabsf(kk.w) + fabsf(gyv) < 1e30f)) ok = false;
            }
        }
        if (!ok) {
            bu = bv = kk = make_float4(0.f, 0.f, 0.f, 0.f);
            gyv = 0.f;
        }
        s_bu[threadIdx.x] = bu;
        s_bv[threadIdx.x] = bv;
        s_k[threadIdx.x] = kk;
        s_gy[threadIdx.x] = gyv;
        __syncthreads();
        const int m = min(256, total - base);
        if (half < 2) {
            const int e1 = min(m, (half + 1) * 128);
            if (task < 100) {
                for (int e = half * 128; e < e1; ++e) {
                    const float pr = comp4(s_bu[e], bi) * comp4(s_bu[e], bi2) * comp4(s_bv[e], bj) * comp4(s_bv[e], bj2);
                    acc.x += pr * s_k[e].x;
                    acc.y += pr * s_k[e].y;
                    acc.z += pr * s_k[e].z;
                }
            } else {
                for (int e = half * 128; e < e1; ++e) {
                    const float b = comp4(s_bu[e], bi) * comp4(s_bv[e], bj);
                    acc.x += s_k[e].w * b;
                    acc.y += s_gy[e] * b;
                }
            }
        }
        __syncthreads();
    }
    s_acc[threadIdx.x] = acc;
    __syncthreads();
    if (threadIdx.x < kFcTasks) {
        const float3 u = s_acc[threadIdx.x], v = s_acc[threadIdx.x + kFcTasks];
        float* o = out + (size_t)blockIdx.x * kFfdCell;
        if (threadIdx.x < 100) {
            o[threadIdx.x * 3] = u.x + v.x;
            o[threadIdx.x * 3 + 1] = u.y + v.y;
            o[threadIdx.x * 3 + 2] = u.z + v.z;
        } else {
            o[300 + (threadIdx.x - 100) * 2] = u.x + v.x;
            o[300 + (threadIdx.x - 100) * 2 + 1] = u.y + v.y;
        }
    }
}

// Blocks per pose over `pixels` fixed pixels, with `slots` blocks resident on the GPU at once:
// about 16 pixels per thread, rounded so that whole poses fill whole waves (slots / b poses per
// wave, or b a whole number of waves) — a wave and a few blocks would take two waves' time. The
// count depends on the image alone, never on how many poses share the launch, so a pose's sums
// (and score) are the same whatever batch it is scored in.
// zc_tune_parts' knobs (0 keeps the default): pixels per thread (16), the least and the most
// blocks per pose (none, 4096)
std::atomic<unsigned> g_px_per_thread{16}, g_min_blocks{0}, g_max_blocks{4096};

int pose_blocks(size_t pixels, int slots) {
    const size_t ppt = std::max(1u, g_px_per_thread.load(std::memory_order_relaxed));
    const size_t by_work = std::max<size_t>(1, (pixels + 256 * ppt - 1) / (256 * ppt));
    const size_t sl = (size_t)std::max(slots, 1);
    size_t b = by_work >= sl ? sl * (by_work / sl) : sl / ((sl + by_work - 1) / by_work);
    b = std::max<size_t>(b, g_min_blocks.load(std::memory_order_relaxed));
    return (int)std::max<size_t>(1, std::min<size_t>(b, std::max(1u, g_max_blocks.load(std::memory_order_relaxed))));
}

// resident blocks of 256 threads of kernel k across the GPU
template <class K>
int pose_slots(K k) {
    int dev = 0, sms = 148, per = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, 256, 0) != cudaSuccess || per < 1) per = 1;
    return per * sms;
}

}  // namespace

namespace {
__global__ void k_feat_interleave(const float* __restrict__ feat, int n, float4* __restrict__ out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        out[i] = make_float4(feat[i], feat[(size_t)n + i], feat[2 * (size_t)n + i], feat[3 * (size_t)n + i]);
}
}  // namespace

void pose_tune(unsigned px_per_thread, unsigned min_blocks, unsigned max_blocks) {
    if (px_per_thread) g_px_per_thread = std::min(px_per_thread, 4096u);
    if (min_blocks) g_min_blocks = std::min(min_blocks, 4096u);
    if (max_blocks) g_max_blocks = std::min(max_blocks, 4096u);
}

cudaError_t interleave_features(const float* feat, int n, float4* out, cudaStream_t st) {
    const int blocks = std::min((n + 255) / 256, 148 * 8);
    k_feat_interleave<<<std::max(blocks, 1), 256, 0, st>>>(feat, n, out);
    return cudaGetLastError();
}

namespace {
// resident blocks of each pose kernel: moments (spline, plain), tangent (spline, plain), ffd_grad
const std::array<int, 5>& kernel_slots() {
    static const std::array<int, 5> sl{pose_slots(k_pose_moments<true>), pose_slots(k_pose_moments<false>),
                                       pose_slots(k_pose_tangent<true>), pose_slots(k_pose_tangent<false>),
                                       pose_slots(k_pose_ffd_grad)};
    return sl;
}
// part must hold n poses × blocks × k totals and ticket n counters
bool red_fits(const PoseRed& r, int n, int blocks, int k) {
    return !r.part || (r.ticket && r.tickets >= (size_t)n && r.cap >= (size_t)n * blocks * k);
}
}  // namespace

size_t pose_red_need(size_t pixels, int n) {
    int b = 1;
    for (int sl : kernel_slots()) b = std::max(b, pose_blocks(pixels, sl));
    return (size_t)std::max(n, 1) * b * kMom;
}

cudaError_t pose_moments(const PoseSide& a, const PoseSide& b, const float* hinv, int n, double* sums, cudaStream_t st,
                         const PoseFfd& ffd, const unsigned char* mask, const PoseRed& red) {
    if (ffd.cps && (ffd.g < 2 || ffd.g > kFfdMax)) return cudaErrorInvalidValue;
    if (n <= 0) return cudaSuccess;
    dim3 g(pose_blocks((size_t)b.w * b.h, kernel_slots()[ffd.cps ? 0 : 1]), n);
    if (!red_fits(red, n, (int)g.x, kMom)) return cudaErrorInvalidValue;
    cudaMemsetAsync(sums, 0, (size_t)n * kMom * sizeof(double), st);
    if (ffd.cps)
        k_pose_moments<true><<<g, 256, 0, st>>>(a.feat4, a.w, a.h, b.feat4, b.w, b.h, hinv, sums, ffd, mask, red);
    else
        k_pose_moments<false><<<g, 256, 0, st>>>(a.feat4, a.w, a.h, b.feat4, b.w, b.h, hinv, sums, ffd, mask, red);
    return cudaGetLastError();
}

cudaError_t pose_ffd_cells(const PoseSide& a, const PoseSide& b, const float* hinv, const float* hpose,
                           const float* coef, const PoseFfd& ffd, int nch, float* out, cudaStream_t st) {
    if (!ffd.cps || ffd.g < 2 || ffd.g > kFfdMax || nch < 1) return cudaErrorInvalidValue;
    k_pose_ffd_cells<<<ffd.g * ffd.g * nch, 256, 0, st>>>(a.feat4, a.w, a.h, b.feat4, b.w, b.h, hinv, hpose, coef, ffd,
                                                          nch, out);
    return cudaGetLastError();
}

cudaError_t pose_ffd_grad(const PoseSide& a, const PoseSide& b, const float* hinv, const float* coef,
                          const PoseFfd& ffd, int cp0, double* out, cudaStream_t st, const PoseRed& red) {
    if (!ffd.cps || ffd.g < 2 || ffd.g > kFfdMax) return cudaErrorInvalidValue;
    const int blocks = pose_blocks((size_t)b.w * b.h, kernel_slots()[4]);
    if (!red_fits(red, 1, blocks, 32)) return cudaErrorInvalidValue;
    cudaMemsetAsync(out, 0, 32 * sizeof(double), st);
    k_pose_ffd_grad<<<blocks, 256, 0, st>>>(a.feat4, a.w, a.h, b.feat4, b.w, b.h, hinv, coef, ffd, cp0, out, red);
    return cudaGetLastError();
}

cudaError_t pose_coefs(const double* sums, int n, bool exact, float* coef, double* score, cudaStream_t st) {
    k_pose_coefs<<<(n + 63) / 64, 64, 0, st>>>(sums, n, exact ? 1 : 0, 1e-4, coef, score);
    return cudaGetLastError();
}

cudaError_t pose_tangent(const PoseSide& a, const PoseSide& b, const float* hinv, const float* coef, const float* gens,
                         int n, bool hess, double* out, cudaStream_t st, const PoseFfd& ffd, const unsigned char* mask,
                         const PoseRed& red) {
    if (ffd.cps && (ffd.g < 2 || ffd.g > kFfdMax)) return cudaErrorInvalidValue;
    if (n <= 0) return cudaSuccess;
    dim3 g(pose_blocks((size_t)b.w * b.h, kernel_slots()[ffd.cps ? 2 : 3]), n);
    if (!red_fits(red, n, (int)g.x, kGrad)) return cudaErrorInvalidValue;
    cudaMemsetAsync(out, 0, (size_t)n * kGrad * sizeof(double), st);
    if (ffd.cps)
        k_pose_tangent<true><<<g, 256, 0, st>>>(a.feat4, a.w, a.h, b.feat4, b.w, b.h, hinv, coef, gens, hess ? 1 : 0, out, ffd,
                                                mask, red);
    else
        k_pose_tangent<false><<<g, 256, 0, st>>>(a.feat4, a.w, a.h, b.feat4, b.w, b.h, hinv, coef, gens, hess ? 1 : 0, out,
                                                 ffd, mask, red);
    return cudaGetLastError();
}

}  // namespace zc
