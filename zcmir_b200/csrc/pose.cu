// Pose scores and gradients on the GPU: the 45 overlap moment sums of many poses at once, the
// score and its gradient coefficients (float64), and the tangent gradient with the Gauss–Newton
// matrix. Restated from the reference's shaders/smi.wgsl (overlap_moments 977-1057, taper
// 336-351, boundary_value 353-366, score_dva 1059-1081, tangent_grad 1123-1272) and
// src/moments.zig (scoreFromMoments 91-172).
//
// One direction warps image a (moving) onto image b (fixed): every b pixel x samples a's
// features bilinearly at H⁻¹(x + 1) − 1, weighted by a 2-px ramp inside a's valid border. Blocks
// of pose p sum their pixels in float32 per thread, then float64 across the block, and add into
// the pose's float64 sums.
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

struct Hinv {
    float m[9];
};

// pose sample position of b pixel (x, y): false when outside a's valid interior
__device__ __forceinline__ bool sample_pos(const float* Hi, int x, int y, int aw, int ah, float& fx, float& fy, float3& ph) {
    const float X = (float)x + 1.f, Y = (float)y + 1.f;
    ph.x = Hi[0] * X + Hi[1] * Y + Hi[2];
    ph.y = Hi[3] * X + Hi[4] * Y + Hi[5];
    ph.z = Hi[6] * X + Hi[7] * Y + Hi[8];
    if (fabsf(ph.z) < 1e-8f) return false;
    fx = ph.x / ph.z - 1.f;
    fy = ph.y / ph.z - 1.f;
    return !(fx < 2.f || fy < 2.f || fx > (float)aw - 3.f || fy > (float)ah - 3.f);
}

// The 45 sums: 0 Σw, 1–4 Σw a, 5–8 Σw b, 9–24 Σw a_i b_j, 25–34 / 35–44 upper triangles of
// Σw a aᵀ and Σw b bᵀ.
__global__ void __launch_bounds__(256) k_pose_moments(const float* __restrict__ fa, int aw, int ah,
                                                      const float* __restrict__ fb, int bw, int bh,
                                                      const float* __restrict__ hinv, double* __restrict__ sums) {
    __shared__ float Hs[9];
    __shared__ float red[8][kMom];
    const int pose = blockIdx.y;
    if (threadIdx.x < 9) Hs[threadIdx.x] = hinv[pose * 9 + threadIdx.x];
    __syncthreads();
    float Hi[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) Hi[i] = Hs[i];
    float acc[kMom];
#pragma unroll
    for (int k = 0; k < kMom; ++k) acc[k] = 0.f;
    const size_t na = (size_t)aw * ah, nb = (size_t)bw * bh;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < nb; t += (size_t)gridDim.x * blockDim.x) {
        const int y = (int)(t / bw), x = (int)(t - (size_t)y * bw);
        float fx, fy;
        float3 ph;
        if (!sample_pos(Hi, x, y, aw, ah, fx, fy, ph)) continue;
        float wt, d1, d2;
        taper(fx, fy, (float)aw, (float)ah, wt, d1, d2);
        if (wt <= 0.f) continue;
        const float flx = floorf(fx), fly = floorf(fy);
        const float ax = fx - flx, ay = fy - fly;
        const size_t i00 = (size_t)fly * aw + (size_t)flx;
        float va[4], vb[4];
#pragma unroll
        for (int p = 0; p < 4; ++p) {
            const float* P = fa + p * na;
            const float v00 = __ldg(&P[i00]), v10 = __ldg(&P[i00 + 1]);
            const float v01 = __ldg(&P[i00 + aw]), v11 = __ldg(&P[i00 + aw + 1]);
            va[p] = (v00 * (1.f - ax) + v10 * ax) * (1.f - ay) + (v01 * (1.f - ax) + v11 * ax) * ay;
            vb[p] = __ldg(&fb[p * nb + t]);
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
    if (threadIdx.x < kMom) {
        double s = 0.0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) s += (double)red[i][threadIdx.x];
        atomicAdd(&sums[pose * kMom + threadIdx.x], s);
    }
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
__global__ void __launch_bounds__(256) k_pose_tangent(const float* __restrict__ fa, int aw, int ah,
                                                      const float* __restrict__ fb, int bw, int bh,
                                                      const float* __restrict__ hinv, const float* __restrict__ coef,
                                                      const float* __restrict__ gens, int hess, double* __restrict__ out) {
    __shared__ float Hs[9], Mk[8][9], cf[kCoef];
    __shared__ float red[8][kGrad];
    const int pose = blockIdx.y;
    if (threadIdx.x < 9) Hs[threadIdx.x] = hinv[pose * 9 + threadIdx.x];
    for (int k = threadIdx.x; k < kCoef; k += blockDim.x) cf[k] = coef[pose * kCoef + k];
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
    const size_t na = (size_t)aw * ah, nb = (size_t)bw * bh;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < nb; t += (size_t)gridDim.x * blockDim.x) {
        const int y = (int)(t / bw), x = (int)(t - (size_t)y * bw);
        float fx, fy;
        float3 ph;
        if (!sample_pos(Hi, x, y, aw, ah, fx, fy, ph)) continue;
        float wt, tpx, tpy;
        taper(fx, fy, (float)aw, (float)ah, wt, tpx, tpy);
        const float flx = floorf(fx), fly = floorf(fy);
        const float ax = fx - flx, ay = fy - fly;
        const size_t i00 = (size_t)fly * aw + (size_t)flx;
        float va[4], gx[4], gy[4], vb[4];
#pragma unroll
        for (int p = 0; p < 4; ++p) {
            const float* P = fa + p * na;
            const float v00 = __ldg(&P[i00]), v10 = __ldg(&P[i00 + 1]);
            const float v01 = __ldg(&P[i00 + aw]), v11 = __ldg(&P[i00 + aw + 1]);
            va[p] = (v00 * (1.f - ax) + v10 * ax) * (1.f - ay) + (v01 * (1.f - ax) + v11 * ax) * ay;
            gx[p] = (v10 - v00) * (1.f - ay) + (v11 - v01) * ay;
            gy[p] = (v01 - v00) * (1.f - ax) + (v11 - v10) * ax;
            vb[p] = __ldg(&fb[p * nb + t]);
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
        const float X = (float)x + 1.f, Y = (float)y + 1.f;
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
    if (threadIdx.x < kGrad) {
        double s = 0.0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) s += (double)red[i][threadIdx.x];
        atomicAdd(&out[pose * kGrad + threadIdx.x], s);
    }
}

int pose_blocks(size_t pixels, int n) {
    const size_t by_work = (pixels + 256 * 16 - 1) / (256 * 16);  // ≥ 16 pixels per thread
    const size_t by_fill = (1184 + (size_t)n - 1) / (size_t)n;
    size_t b = std::min(by_work, std::max<size_t>(by_fill, 1));
    return (int)std::max<size_t>(1, std::min<size_t>(b, 4096));
}

}  // namespace

cudaError_t pose_moments(const PoseSide& a, const PoseSide& b, const float* hinv, int n, double* sums, cudaStream_t st) {
    cudaMemsetAsync(sums, 0, (size_t)n * kMom * sizeof(double), st);
    dim3 g(pose_blocks((size_t)b.w * b.h, n), n);
    k_pose_moments<<<g, 256, 0, st>>>(a.feat, a.w, a.h, b.feat, b.w, b.h, hinv, sums);
    return cudaGetLastError();
}

cudaError_t pose_coefs(const double* sums, int n, bool exact, float* coef, double* score, cudaStream_t st) {
    k_pose_coefs<<<(n + 63) / 64, 64, 0, st>>>(sums, n, exact ? 1 : 0, 1e-4, coef, score);
    return cudaGetLastError();
}

cudaError_t pose_tangent(const PoseSide& a, const PoseSide& b, const float* hinv, const float* coef, const float* gens,
                         int n, bool hess, double* out, cudaStream_t st) {
    cudaMemsetAsync(out, 0, (size_t)n * kGrad * sizeof(double), st);
    dim3 g(pose_blocks((size_t)b.w * b.h, n), n);
    k_pose_tangent<<<g, 256, 0, st>>>(a.feat, a.w, a.h, b.feat, b.w, b.h, hinv, coef, gens, hess ? 1 : 0, out);
    return cudaGetLastError();
}

}  // namespace zc
