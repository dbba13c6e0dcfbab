// The per-shift SMI score, centred and whitened in float64 (the reference's combine_cell,
// shaders/smi.wgsl:825-915), shared by the row-pass kernels.
#pragma once

#include "kernels.hpp"

namespace zc {

// The correlation plan as compile-time tables (src/smi.zig:90-158): the moving and fixed plane
// of correlation c, and its slot in a plan that drops the fourth feature's planes.
__host__ __device__ constexpr int corr_a(int c) {
    return c == 0 ? 0 : c <= 4 ? c : c <= 8 ? 0 : c <= 24 ? 1 + (c - 9) / 4 : c <= 34 ? 5 + (c - 25) : 0;
}
__host__ __device__ constexpr int corr_b(int c) {
    return c <= 4 ? 0 : c <= 8 ? c - 4 : c <= 24 ? 1 + (c - 9) % 4 : c <= 34 ? 0 : 5 + (c - 35);
}
__host__ __device__ constexpr bool fourth_plane(int p) { return p == 4 || p == 8 || p == 11 || p == 13 || p == 14; }
__host__ __device__ constexpr bool corr_kept(int c, bool three) {
    return !three || (!fourth_plane(corr_a(c)) && !fourth_plane(corr_b(c)));
}
__host__ __device__ constexpr int corr_slot(int c, bool three) {
    int s = 0;
    for (int i = 0; i < c; ++i) s += corr_kept(i, three) ? 1 : 0;
    return s;
}

__host__ __device__ constexpr int tri_kc(int i, int j) {
    return (i < j ? i : j) * 4 - ((i < j ? i : j) * ((i < j ? i : j) + 1)) / 2 + (i < j ? j : i);
}

// The score's parameters for the shifts of row y of an ny-row map: a log-polar map scales row
// y's sums by e^{kΔλ}·Δλ·Δθ (k the row's wrapped log-radius lag, smi.wgsl:777-795 extract_pair).
__device__ __forceinline__ CombineParams row_params(const CombineParams& cp, int y, int ny) {
    CombineParams r = cp;
    if (cp.lp_dlam != 0.0) {
        const int k = y <= ny / 2 ? y : y - ny;
        r.inv_nn = cp.inv_nn * exp((double)k * cp.lp_dlam) * cp.lp_dlam * cp.lp_dth;
    }
    return r;
}
// the zero-lag overlap in the map's units (row 0 of a log-polar map carries Δλ·Δθ)
__device__ __forceinline__ double lag0_units(const CombineParams& cp, double n00) {
    return cp.lp_dlam != 0.0 ? n00 * cp.lp_dlam * cp.lp_dth : n00;
}

// Per-shift score (smi.wgsl:825-915, combine_cell): centring, ridge, Cholesky factors and the
// whitened norm in float64, the calibrated map's Wilson–Hilferty transform in float32; every
// index known at compile time (NF features, exact or global whitening, calibrated or not), so the 4×4 algebra stays in
// registers. `get(slot)` returns this shift's (unscaled) sum of the plan's slot `slot`; the
// slots follow the plan (NF = 3 drops the fourth feature's correlations), and every slot passed
// to it is a compile-time constant. Each Cholesky pivot is inverted once (rsqrt) and the
// substitutions multiply by it.
template <int NF, bool EXACT, bool CALIB, class G>
__device__ __forceinline__ float combine_smi(G&& get, const CombineParams& p, double n00) {
    constexpr bool THREE = NF == 3;
    auto S = [&](int c) -> double { return (double)get(corr_slot(c, THREE)) * p.inv_nn; };
    const double n = S(0);
    const double neff = n / fmax(p.area, 1.0);
    double floor_n = fmax((double)p.min_n, 0.08 * fmax(n00, 0.0));
    if (CALIB) floor_n = (double)p.min_n;
    if (n < floor_n || (CALIB && neff <= 10.0)) return 0.f;
    const double rn = 1.0 / fmax(n, 1e-8);
    double ma[NF], mb[NF], C[NF][NF];
#pragma unroll
    for (int i = 0; i < NF; ++i) {
        ma[i] = S(1 + i) * rn;
        mb[i] = S(5 + i) * rn;
    }
#pragma unroll
    for (int i = 0; i < NF; ++i)
#pragma unroll
        for (int j = 0; j < NF; ++j) C[i][j] = S(9 + 4 * i + j) * rn - ma[i] * mb[j];
    if (!EXACT) {
        double s = 0.0;
#pragma unroll
        for (int i = 0; i < NF; ++i)
#pragma unroll
            for (int j = 0; j < NF; ++j) {
                const double c = fmin(fmax(C[i][j], -1.0), 1.0);
                s += c * c;
            }
        const double sc = n * s;
        return (sc == sc) ? (float)sc : 0.f;
    }
    double A[NF][NF], B[NF][NF];
    double tra = 0.0, trb = 0.0;
#pragma unroll
    for (int i = 0; i < NF; ++i) {
#pragma unroll
        for (int j = 0; j <= i; ++j) {
            A[i][j] = S(25 + tri_kc(i, j)) * rn - ma[i] * ma[j];
            B[i][j] = S(35 + tri_kc(i, j)) * rn - mb[i] * mb[j];
        }
        tra += A[i][i];
        trb += B[i][i];
    }
    const double rga = p.ridge * fmax(tra * 0.25, 1e-12), rgb = p.ridge * fmax(trb * 0.25, 1e-12);
    double ia[NF], ib[NF];  // 1 / L_ii
#pragma unroll
    for (int i = 0; i < NF; ++i) {
        A[i][i] += rga;
        B[i][i] += rgb;
    }
#pragma unroll
    for (int i = 0; i < NF; ++i) {
#pragma unroll
        for (int j = 0; j <= i; ++j) {
            double sa = A[i][j], sb = B[i][j];
#pragma unroll
            for (int k = 0; k < j; ++k) {
                sa -= A[i][k] * A[j][k];
                sb -= B[i][k] * B[j][k];
            }
            if (i == j) {
                if (!(sa > 0.0) || !(sb > 0.0)) return 0.f;
                ia[i] = rsqrt(sa);
                ib[i] = rsqrt(sb);
                A[i][i] = sa * ia[i];
                B[i][i] = sb * ib[i];
            } else {
                A[i][j] = sa * ia[j];
                B[i][j] = sb * ib[j];
            }
        }
    }
    // X = L_A⁻¹ C (forward substitution down each column), in place in C
#pragma unroll
    for (int j = 0; j < NF; ++j)
#pragma unroll
        for (int i = 0; i < NF; ++i) {
            double s = C[i][j];
#pragma unroll
            for (int k = 0; k < i; ++k) s -= A[i][k] * C[k][j];
            C[i][j] = s * ia[i];
        }
    // Y = X L_B⁻ᵀ row by row, ‖Y‖² as it goes
    double acc = 0.0;
#pragma unroll
    for (int r = 0; r < NF; ++r) {
        double yv[NF];
#pragma unroll
        for (int i = 0; i < NF; ++i) {
            double s = C[r][i];
#pragma unroll
            for (int k = 0; k < i; ++k) s -= B[i][k] * yv[k];
            yv[i] = s * ib[i];
            acc += yv[i] * yv[i];
        }
    }
    double score = n * acc;
    if (CALIB) {
        // the Wilson–Hilferty transform of the whitened statistic in float32: the float64 steps
        // are the centring and the Cholesky factors above; this tail only rescales their result
        constexpr float q = NF;
        const float v = fminf((float)acc, q - 1e-4f);
        const float nq = (float)neff - q - 1.0f;
        const float fv = nq * v / (q * (q - v));
        constexpr float a = 2.0f / (9.0f * q * q);
        const float b = 2.0f / (9.0f * q * nq);
        const float cc = cbrtf(fmaxf(fv, 0.0f));
        const float z = ((1.0f - b) * cc - (1.0f - a)) * rsqrtf(b * cc * cc + a);
        score = fmaxf(z, 0.0f);
    }
    return (score == score) ? (float)score : 0.f;
}

// The NCC map's value at a lag (src/overlay.zig:256-258): the mean-free correlation over the
// product of the planes' norms (den, carried in the n00 slot), clamped to ±1.5.
template <class G>
__device__ __forceinline__ float combine_ncc(G&& get, const CombineParams& p, double den) {
    const double v = (double)get(0) * p.inv_nn / den;
    return (float)fmin(1.5, fmax(-1.5, v));
}

// NF = 1 selects the NCC map, 3 or 4 the SMI score over that many features.
template <int NF, bool EXACT, bool CALIB, class G>
__device__ __forceinline__ float combine_t(G&& get, const CombineParams& p, double n00) {
    if constexpr (NF == 1)
        return combine_ncc(get, p, n00);
    else
        return combine_smi<NF, EXACT, CALIB>(get, p, n00);
}

}  // namespace zc
