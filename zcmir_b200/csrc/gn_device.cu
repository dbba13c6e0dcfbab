// The batched Gauss–Newton refine on the device: the step, the candidate poses and the choice
// among them, so that a run of iterations needs no host round trip.
//
// Each iteration is, for n poses at once: the poses' inverse maps, their overlap moments,
// scores, tangent gradients and Gauss–Newton matrices (the pose kernels of pose.cu); then, one
// warp per pose, the symmetric pair's gradient and matrix, the unit-ascent candidates (the step
// ladder `amps`) and the Gauss–Newton candidates (the solved step at 0.5, 1, 2, 4, 8 times, each
// capped at a tangent norm of 0.25), each composed onto the pose in normalised fixed
// coordinates; their scores; and, per pose, the first candidate in order that beats the score so
// far (by more than 1e-6 of it), as the host loop of the same search chooses. A pose that did
// not move is frozen. The pose algebra here restates the host's (lie.hpp, geom.hpp: the
// reference's src/lie.zig destN, hat, vee, expm3, projectGroup, composeN, adjointGrad,
// solveLinear) operation for operation in float64, and this file is compiled without fused
// multiply-adds, so the device loop and the host loop produce the same poses bit for bit.
#include <cuda_runtime.h>

#include "kernels.hpp"

namespace zc {
namespace {

// sums per pose row, tangent sums per pose row; candidates per pose: at most 16 ascent steps and
// the 5 Gauss–Newton multiples, one lane each
constexpr int kMomN = 45, kGradN = 44, kMaxTry = 21;

__device__ void d_mul3(const double* a, const double* b, double* o) {
    double t[9];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) t[r * 3 + c] = a[r * 3] * b[c] + a[r * 3 + 1] * b[3 + c] + a[r * 3 + 2] * b[6 + c];
    for (int i = 0; i < 9; ++i) o[i] = t[i];
}

// inverse by the adjugate with one Newton refinement step (geom.hpp inv3)
__device__ void d_inv3(const double* m, double* o) {
    const double a = m[0], b = m[1], c = m[2], d = m[3], e = m[4], f = m[5], g = m[6], h = m[7], i = m[8];
    const double A = e * i - f * h, B = f * g - d * i, C = d * h - e * g;
    const double D = c * h - b * i, E = a * i - c * g, F = b * g - a * h;
    const double G = b * f - c * e, Hh = c * d - a * f, I = a * e - b * d;
    const double det = a * A + b * B + c * C;
    const double sg = det > 0 ? 1.0 : (det < 0 ? -1.0 : 0.0);
    const double s = 1.0 / (sg * fmax(fabs(det), 1e-18));
    const double inv[9] = {A * s, D * s, G * s, B * s, E * s, Hh * s, C * s, F * s, I * s};
    double p[9];
    d_mul3(m, inv, p);
    const double corr[9] = {2 - p[0], -p[1], -p[2], -p[3], 2 - p[4], -p[5], -p[6], -p[7], 2 - p[8]};
    d_mul3(inv, corr, o);
}

__device__ void d_destN(double w0, double h0, double* o) {
    const double w = fmax(w0, 1.0), h = fmax(h0, 1.0);
    const double sx = 0.5 * w, sy = 0.5 * h, cx = 0.5 * (w + 1), cy = 0.5 * (h + 1);
    const double v[9] = {1 / sx, 0, -cx / sx, 0, 1 / sy, -cy / sy, 0, 0, 1};
    for (int i = 0; i < 9; ++i) o[i] = v[i];
}

__device__ void d_hat(const double* x, bool homog, double* o) {
    double px = x[6], py = x[7], iso, z;
    if (!homog) {
        px = py = z = 0;
        iso = x[3];
    } else {
        iso = x[3] / 3;
        z = -2 * iso;
    }
    const double v[9] = {iso + x[4], x[5] - x[2], x[0], x[5] + x[2], iso - x[4], x[1], px, py, z};
    for (int i = 0; i < 9; ++i) o[i] = v[i];
}

__device__ void d_vee(const double* A0, bool homog, double* out) {
    double a = A0[0], e = A0[4];
    const double b = A0[1], c = A0[2], d = A0[3], f = A0[5], g = A0[6], h = A0[7], i = A0[8];
    if (homog) {
        const double tr = (a + e + i) / 3;
        a -= tr;
        e -= tr;
        const double iso = (a + e) / 2;
        const double v[8] = {c, f, (d - b) / 2, iso * 3, (a - e) / 2, (d + b) / 2, g, h};
        for (int k = 0; k < 8; ++k) out[k] = v[k];
        return;
    }
    const double v[8] = {c, f, (d - b) / 2, (a + e) / 2, (a - e) / 2, (d + b) / 2, 0, 0};
    for (int k = 0; k < 8; ++k) out[k] = v[k];
}

// scaling and squaring of a 13-term Taylor series (lie.hpp expm3)
__device__ void d_expm3(const double* A, double* T) {
    double nrm = 0;
    for (int i = 0; i < 9; ++i) nrm = fmax(nrm, fabs(A[i]));
    int s = 0;
    for (double v = nrm; v > 0.5 && s < 10; v *= 0.5) ++s;
    const double sc = ldexp(1.0, -s);
    double B[9], P[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    for (int i = 0; i < 9; ++i) B[i] = A[i] * sc;
    for (int i = 0; i < 9; ++i) T[i] = P[i];
    for (int k = 1; k < 14; ++k) {
        d_mul3(P, B, P);
        for (int i = 0; i < 9; ++i) P[i] /= (double)k;
        for (int i = 0; i < 9; ++i) T[i] += P[i];
    }
    for (int i = 0; i < s; ++i) d_mul3(T, T, T);
}

__device__ void d_project_group(const double* H, bool homog, double* o) {
    const double s = fabs(H[8]) > 1e-12 ? H[8] : 1;
    for (int i = 0; i < 9; ++i) o[i] = H[i] / s;
    if (!homog) {
        o[6] = 0;
        o[7] = 0;
        o[8] = 1;
    }
}

// exp(ξ̂) applied in normalised coordinates of a dw×dh destination (lie.hpp composeN)
__device__ void d_composeN(const double* H0, const double* x, bool homog, double dw, double dh, double* o) {
    double N[9], Ni[9], X[9], E[9], t[9];
    d_destN(dw, dh, N);
    d_inv3(N, Ni);
    d_hat(x, homog, X);
    d_expm3(X, E);
    d_mul3(Ni, E, t);
    d_mul3(t, N, t);
    d_mul3(t, H0, t);
    d_project_group(t, homog, o);
}

// dS/dξ on H given dS/dη on H⁻¹ (lie.hpp adjoint_grad)
__device__ void d_adjoint_grad(const double* g_eta, const double* H, bool homog, double mw, double mh, double fw,
                               double fh, double* out) {
    double Hi[9], Nm[9], Nf[9], Nfi[9], M[9], Mi[9], t[9];
    d_inv3(H, Hi);
    d_destN(mw, mh, Nm);
    d_destN(fw, fh, Nf);
    d_inv3(Nf, Nfi);
    d_mul3(Nm, Hi, t);
    d_mul3(t, Nfi, M);
    d_inv3(M, Mi);
    const int nk = homog ? 8 : 6;
    for (int k = 0; k < 8; ++k) out[k] = 0;
    for (int i = 0; i < nk; ++i) {
        double e[8] = {0, 0, 0, 0, 0, 0, 0, 0}, X[9], cc[8];
        e[i] = 1;
        d_hat(e, homog, X);
        d_mul3(M, X, t);
        d_mul3(t, Mi, t);
        d_vee(t, homog, cc);
        for (int j = 0; j < nk; ++j) out[i] -= g_eta[j] * cc[j];
    }
}

// A·x = b by Gauss–Jordan with partial pivoting (lie.hpp solve_linear)
__device__ bool d_solve_linear(const double* A, const double* b, int n, double* x) {
    double M[64];
    for (int i = 0; i < n * n; ++i) M[i] = A[i];
    for (int i = 0; i < n; ++i) x[i] = b[i];
    for (int i = 0; i < n; ++i) {
        int piv = i;
        for (int r = i + 1; r < n; ++r)
            if (fabs(M[r * n + i]) > fabs(M[piv * n + i])) piv = r;
        if (piv != i) {
            for (int j = 0; j < n; ++j) {
                const double tmp = M[i * n + j];
                M[i * n + j] = M[piv * n + j];
                M[piv * n + j] = tmp;
            }
            const double tmp = x[i];
            x[i] = x[piv];
            x[piv] = tmp;
        }
        const double d = M[i * n + i];
        if (!isfinite(d) || fabs(d) < 1e-300) return false;
        for (int r = 0; r < n; ++r) {
            if (r == i) continue;
            const double f = M[r * n + i] / d;
            if (f == 0) continue;
            for (int j = i; j < n; ++j) M[r * n + j] -= f * M[i * n + j];
            x[r] -= f * x[i];
        }
    }
    for (int i = 0; i < n; ++i) {
        x[i] /= M[i * n + i];
        if (!isfinite(x[i])) return false;
    }
    return true;
}

__device__ __forceinline__ double fin(double v) { return isfinite(v) ? v : 0.0; }

// one direction's gradient and Gauss–Newton matrix from its tangent sums (zero below 12 overlap)
__device__ void unpack(const double* t, double nsum, int nk, double* g, double* A) {
    for (int q = 0; q < 8; ++q) g[q] = 0;
    for (int q = 0; q < 64; ++q) A[q] = 0;
    if (!(nsum >= 12.0)) return;
    for (int q = 0; q < nk; ++q) g[q] = t[q];
    int h = 8;
    for (int q = 0; q < 8; ++q)
        for (int m = q; m < 8; ++m, ++h)
            if (q < nk && m < nk) A[q * nk + m] = A[m * nk + q] = t[h];
}

// the poses' inverse maps for the pose kernels: forward H⁻¹, inverse direction (H⁻¹)⁻¹
__global__ void k_gn_hinv(const double* __restrict__ H, int n, int sym, float* __restrict__ hinv) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double Hi[9];
    d_inv3(H + (size_t)i * 9, Hi);
    for (int k = 0; k < 9; ++k) hinv[(size_t)i * 9 + k] = (float)Hi[k];
    if (sym) {
        double Hii[9];
        d_inv3(Hi, Hii);
        for (int k = 0; k < 9; ++k) hinv[((size_t)n + i) * 9 + k] = (float)Hii[k];
    }
}

// one warp per pose: the lanes share the pull-back's columns, the matrix entries and the
// candidates; each value is still computed by one lane in the host loop's order
__global__ void __launch_bounds__(32) k_gn_propose(GnDims d, GnAmps amps, const double* __restrict__ H,
                                                   const double* __restrict__ sums, const double* __restrict__ score,
                                                   const double* __restrict__ tsum,
                                                   const unsigned char* __restrict__ active, double* __restrict__ cur,
                                                   double* __restrict__ Htry, unsigned char* __restrict__ valid) {
    const int i = blockIdx.x, lane = threadIdx.x;
    const int T = d.T, nk = d.nk, n = d.n;
    const bool homog = d.homog != 0, sym = d.sym != 0;
    __shared__ double g[8], A[64], gf[8], Af[64], gb[8], Ab[64], PT[64], step[8], dv[8];
    __shared__ int use_ascent, use_step;
    unsigned char* ok = valid + (size_t)i * T;
    if (lane < T) ok[lane] = 0;
    if (!active[i]) return;  // uniform over the block
    const double* Hp = H + (size_t)i * 9;
    if (lane == 0) {
        const double fwd = fin(score[i]), inv = sym ? fin(score[n + i]) : 0.0;
        cur[i] = sym ? 0.5 * (fwd + inv) : fwd;
        unpack(tsum + (size_t)i * kGradN, sums[(size_t)i * kMomN], nk, gf, Af);
        if (sym) unpack(tsum + ((size_t)n + i) * kGradN, sums[((size_t)n + i) * kMomN], nk, gb, Ab);
    }
    for (int q = lane; q < 64; q += 32) PT[q] = 0;
    __syncwarp();
    if (!sym) {
        for (int q = lane; q < 64; q += 32) A[q] = Af[q];
        if (lane < 8) g[lane] = gf[lane];
    } else {
        // the pull-back's columns (lanes 0..nk−1) and the pulled inverse-direction gradient (lane 8)
        double col[8];
        if (lane < nk) {
            double e[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            e[lane] = 1;
            d_adjoint_grad(e, Hp, homog, d.mw, d.mh, d.fw, d.fh, col);
            for (int q = 0; q < nk; ++q) PT[q * nk + lane] = col[q];
        } else if (lane == 8) {
            d_adjoint_grad(gb, Hp, homog, d.mw, d.mh, d.fw, d.fh, col);
            for (int q = 0; q < 8; ++q) g[q] = 0;
            for (int q = 0; q < nk; ++q) g[q] = 0.5 * (gf[q] + col[q]);
        }
        for (int q = lane; q < 64; q += 32) A[q] = 0;
        __syncwarp();
        for (int e = lane; e < nk * nk; e += 32) {
            const int p = e / nk, q = e % nk;
            double s2 = 0;
            for (int x = 0; x < nk; ++x)
                for (int y = 0; y < nk; ++y) s2 += PT[p * nk + x] * Ab[x * nk + y] * PT[q * nk + y];
            A[p * nk + q] = 0.5 * (Af[p * nk + q] + s2);
        }
    }
    __syncwarp();
    if (lane == 0) {
        // the unit ascent direction (src/lie.zig unitAscent)
        use_ascent = 0;
        for (int q = 0; q < 8; ++q) dv[q] = 0;
        if (amps.n > 0) {
            double nr = 0;
            for (int q = 0; q < nk; ++q) dv[q] = g[q], nr += dv[q] * dv[q];
            nr = sqrt(nr);
            if (nr >= 1e-18)
                for (int q = 0; q < nk; ++q) dv[q] /= nr;
            double dn = 0;
            for (int q = 0; q < nk; ++q) dn += dv[q] * dv[q];
            use_ascent = sqrt(dn) > 1e-12;
        }
        // the Gauss–Newton step
        double Am[64], half[8], st8[8];
        for (int q = 0; q < nk * nk; ++q) Am[q] = A[q];
        for (int q = 0; q < nk; ++q) Am[q * nk + q] += 1e-4 * fmax(Am[q * nk + q], 1e-12);
        for (int q = 0; q < nk; ++q) half[q] = 0.5 * g[q];
        use_step = d_solve_linear(Am, half, nk, st8) ? 1 : 0;
        for (int q = 0; q < 8; ++q) step[q] = (q < nk && use_step) ? st8[q] : 0;
    }
    __syncwarp();
    // the candidates, one lane each: the step ladder along the ascent direction, then the step's
    // multiples (each capped at a tangent norm of 0.25)
    if (lane < T) {
        double x[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        bool made = false;
        if (lane < amps.n) {
            if (use_ascent) {
                for (int k = 0; k < nk; ++k) x[k] = amps.v[lane] * dv[k];
                made = true;
            }
        } else if (use_step) {
            double nrm = 0;
            for (int q = 0; q < nk; ++q) nrm += step[q] * step[q];
            nrm = sqrt(nrm);
            const double mults[5] = {0.5, 1, 2, 4, 8};
            const double m = mults[lane - amps.n];
            const double sc = m * (nrm * m > 0.25 ? 0.25 / (nrm * m) : 1.0);
            for (int k = 0; k < nk; ++k) x[k] = sc * step[k];
            made = true;
        }
        if (made) {
            d_composeN(Hp, x, homog, d.fw, d.fh, Htry + ((size_t)i * T + lane) * 9);
            ok[lane] = 1;
        }
    }
}

// per pose, in candidate order, the first candidate that beats the score so far becomes the pose
__global__ void k_gn_select(GnDims d, const double* __restrict__ tscore, const unsigned char* __restrict__ valid,
                            const double* __restrict__ Htry, double* __restrict__ H, double* __restrict__ cur,
                            unsigned char* __restrict__ active) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.n) return;
    const int T = d.T, nt = d.n * T;
    const bool sym = d.sym != 0;
    if (!active[i]) return;
    bool moved = false;
    double c = cur[i];
    for (int t = 0; t < T; ++t) {
        const size_t k = (size_t)i * T + t;
        if (!valid[k]) continue;
        const double fwd = fin(tscore[k]), inv = sym ? fin(tscore[nt + k]) : 0.0;
        const double s = sym ? 0.5 * (fwd + inv) : fwd;
        if (s > c + fmax(1e-6 * fabs(c), 1e-12)) {
            c = s;
            for (int q = 0; q < 9; ++q) H[(size_t)i * 9 + q] = Htry[k * 9 + q];
            moved = true;
        }
    }
    cur[i] = c;
    active[i] = moved ? 1 : 0;
}

}  // namespace

cudaError_t gn_hinv(const double* H, int n, int sym, float* hinv, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    k_gn_hinv<<<(n + 127) / 128, 128, 0, st>>>(H, n, sym, hinv);
    return cudaGetLastError();
}

cudaError_t gn_propose(const GnDims& d, const GnAmps& amps, const double* H, const double* sums, const double* score,
                       const double* tsum, const unsigned char* active, double* cur, double* Htry,
                       unsigned char* valid, cudaStream_t st) {
    if (d.n <= 0) return cudaSuccess;
    if (amps.n < 0 || amps.n > 16 || d.T != amps.n + 5 || d.T > kMaxTry) return cudaErrorInvalidValue;
    k_gn_propose<<<d.n, 32, 0, st>>>(d, amps, H, sums, score, tsum, active, cur, Htry, valid);
    return cudaGetLastError();
}

cudaError_t gn_select(const GnDims& d, const double* tscore, const unsigned char* valid, const double* Htry, double* H,
                      double* cur, unsigned char* active, cudaStream_t st) {
    if (d.n <= 0) return cudaSuccess;
    k_gn_select<<<(d.n + 127) / 128, 128, 0, st>>>(d, tscore, valid, Htry, H, cur, active);
    return cudaGetLastError();
}

}  // namespace zc
