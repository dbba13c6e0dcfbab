// Pose algebra for the refine: tangent coordinates ξ = [tx ty th sg al ga px py] as left
// increments in normalised fixed coordinates (the reference's src/lie.zig: destN 27-35, hat
// 120-141, expm3 143-163, projectGroup 165-176, composeN 182-185, vee 187-204, generators
// 209-224, adjointGrad 227-241, solveLinear 343-371).
#pragma once

#include <cmath>

#include "geom.hpp"

namespace zc {

using Coords = std::array<double, 8>;

inline int n_keys(bool homography) { return homography ? 8 : 6; }

inline Mat3 destN(double w0, double h0) {
    const double w = std::max(w0, 1.0), h = std::max(h0, 1.0);
    const double sx = 0.5 * w, sy = 0.5 * h, cx = 0.5 * (w + 1), cy = 0.5 * (h + 1);
    return {1 / sx, 0, -cx / sx, 0, 1 / sy, -cy / sy, 0, 0, 1};
}

inline Mat3 hat(const Coords& x, bool homog) {
    double px = x[6], py = x[7], iso, z;
    if (!homog) {
        px = py = z = 0;
        iso = x[3];
    } else {
        iso = x[3] / 3;
        z = -2 * iso;
    }
    return {iso + x[4], x[5] - x[2], x[0], x[5] + x[2], iso - x[4], x[1], px, py, z};
}

inline Coords vee(const Mat3& A0, bool homog) {
    double a = A0[0], e = A0[4];
    const double b = A0[1], c = A0[2], d = A0[3], f = A0[5], g = A0[6], h = A0[7], i = A0[8];
    if (homog) {
        const double tr = (a + e + i) / 3;
        a -= tr;
        e -= tr;
        const double iso = (a + e) / 2;
        return {c, f, (d - b) / 2, iso * 3, (a - e) / 2, (d + b) / 2, g, h};
    }
    return {c, f, (d - b) / 2, (a + e) / 2, (a - e) / 2, (d + b) / 2, 0, 0};
}

// scaling and squaring of a 13-term Taylor series
inline Mat3 expm3(const Mat3& A) {
    double nrm = 0;
    for (double v : A) nrm = std::max(nrm, std::fabs(v));
    // halvings until the norm is at most 0.5 (at most 10), counted exactly
    int s = 0;
    for (double v = nrm; v > 0.5 && s < 10; v *= 0.5) ++s;
    const double sc = std::ldexp(1.0, -s);
    Mat3 B;
    for (int i = 0; i < 9; ++i) B[i] = A[i] * sc;
    Mat3 T = mat_identity(), P = mat_identity();
    for (int k = 1; k < 14; ++k) {
        P = mul3(P, B);
        for (double& v : P) v /= (double)k;
        for (int i = 0; i < 9; ++i) T[i] += P[i];
    }
    for (int i = 0; i < s; ++i) T = mul3(T, T);
    return T;
}

inline Mat3 project_group(const Mat3& H, bool homog) {
    const double s = std::fabs(H[8]) > 1e-12 ? H[8] : 1;
    Mat3 o;
    for (int i = 0; i < 9; ++i) o[i] = H[i] / s;
    if (!homog) {
        o[6] = 0;
        o[7] = 0;
        o[8] = 1;
    }
    return o;
}

// exp(ξ̂) applied in normalised coordinates of a dw×dh destination (the fixed image)
inline Mat3 composeN(const Mat3& H0, const Coords& x, bool homog, double dw, double dh) {
    const Mat3 N = destN(dw, dh);
    return project_group(mul3(mul3(mul3(inv3(N), expm3(hat(x, homog))), N), H0), homog);
}

// Generators of the tangent space in pixel coordinates of a dw×dh destination (N⁻¹ G N); the
// ones past the group's keys are zero.
inline std::array<Mat3, 8> generators(bool homog, double dw, double dh) {
    std::array<Mat3, 8> out{};
    const int nk = n_keys(homog);
    const Mat3 N = destN(dw, dh), Ni = inv3(N);
    for (int k = 0; k < nk; ++k) {
        Coords x{};
        x[k] = 1;
        out[k] = mul3(mul3(Ni, hat(x, homog)), N);
    }
    return out;
}

// dS/dξ on H, given dS/dη on H⁻¹ (η: a left increment in the moving frame).
inline Coords adjoint_grad(const double* g_eta, const Mat3& H, bool homog, double mw, double mh, double fw, double fh) {
    const Mat3 Hi = inv3(H);
    const Mat3 M = mul3(mul3(destN(mw, mh), Hi), inv3(destN(fw, fh)));
    const Mat3 Mi = inv3(M);
    const int nk = n_keys(homog);
    Coords out{};
    for (int i = 0; i < nk; ++i) {
        Coords e{};
        e[i] = 1;
        const Coords cc = vee(mul3(mul3(M, hat(e, homog)), Mi), homog);
        for (int j = 0; j < nk; ++j) out[i] -= g_eta[j] * cc[j];
    }
    return out;
}

// A·x = b by Gauss–Jordan with partial pivoting (n ≤ 8); false if singular or non-finite.
inline bool solve_linear(const double* A, const double* b, int n, double* x) {
    double M[64];
    for (int i = 0; i < n * n; ++i) M[i] = A[i];
    for (int i = 0; i < n; ++i) x[i] = b[i];
    for (int i = 0; i < n; ++i) {
        int piv = i;
        for (int r = i + 1; r < n; ++r)
            if (std::fabs(M[r * n + i]) > std::fabs(M[piv * n + i])) piv = r;
        if (piv != i) {
            for (int j = 0; j < n; ++j) std::swap(M[i * n + j], M[piv * n + j]);
            std::swap(x[i], x[piv]);
        }
        const double d = M[i * n + i];
        if (!std::isfinite(d) || std::fabs(d) < 1e-300) return false;
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
        if (!std::isfinite(x[i])) return false;
    }
    return true;
}

}  // namespace zc
