// Host geometry of the rotation × scale (× shear × stretch) sweep, restated from the reference's
// src/search.zig (sweepGrid 89-116, candLinear 120-128, aboutC 130-132, sv2 135-142, ladderSize
// 185-190, the canvas and footprints 300-371, the peaks' poses 460-493, nms4 500-529, simOf
// 616-640), src/lie.zig (mapPt 311-317, unitAscent 243-255) and src/climb.zig (geoAmps 15-24).
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <vector>

#include "geom.hpp"

namespace zc {

struct SweepGrid {
    std::vector<double> thetas, sigmas, shears, anisos;  // θ in radians
    bool wrap = false;                                   // the θ range is the full circle
    size_t count() const { return thetas.size() * sigmas.size() * shears.size() * anisos.size(); }
};

struct SweepGridOpts {
    double rot_lo = -180, rot_hi = 180;  // degrees
    unsigned n_theta = 90;
    double s_min = 0.5, s_max = 2;
    unsigned n_sigma = 20;
    double shear_max = 0;
    unsigned n_shear = 1;
    double aniso_max = 0;
    unsigned n_aniso = 1;
};

inline std::vector<double> sweep_linspace(double lo, double hi, unsigned n0) {
    const unsigned n = std::max(1u, n0);
    std::vector<double> out(n);
    for (unsigned i = 0; i < n; ++i) out[i] = n == 1 ? 0.5 * (lo + hi) : lo + (i * (hi - lo)) / (double)(n - 1);
    return out;
}

// Rotation samples: a 360° span takes n_theta equal steps from −180° (so −180° and +180°, the same
// rotation, are not both taken); a narrower span puts samples on both of its end points. Scale and
// stretch samples are geometric (stretch factors come in reciprocal pairs about 1); shear samples
// are evenly spaced about 0.
inline SweepGrid sweep_grid(const SweepGridOpts& o) {
    SweepGrid g;
    const unsigned nT = std::max(1u, o.n_theta);
    const double lo_d = std::min(o.rot_lo, o.rot_hi), span_d = std::fabs(o.rot_hi - o.rot_lo);
    g.wrap = span_d >= 360 - 1e-9;
    const double rad = M_PI / 180.0;
    for (unsigned i = 0; i < nT; ++i) {
        const double d = g.wrap ? -180 + 360 * (double)i / nT
                                : (nT == 1 ? lo_d + span_d / 2 : lo_d + span_d * (double)i / (double)(nT - 1));
        g.thetas.push_back(d * rad);
    }
    const double llo = std::log(std::max(1e-3, std::min(o.s_min, o.s_max)));
    const double lhi = std::log(std::max(1e-3, std::max(o.s_min, o.s_max)));
    for (double v : sweep_linspace(llo, lhi, o.n_sigma)) g.sigmas.push_back(std::exp(v));
    const double kmax = std::fabs(o.shear_max);
    g.shears = sweep_linspace(-kmax, kmax, kmax > 0 ? o.n_shear : 1);
    const double amax = std::log(1 + std::fabs(o.aniso_max));
    for (double v : sweep_linspace(-amax, amax, amax > 0 ? o.n_aniso : 1)) g.anisos.push_back(std::exp(v));
    return g;
}

using Lin2 = std::array<double, 4>;

// σ R(θ) diag(a, 1/a) [1 k; 0 1] (row-major 2×2)
inline Lin2 cand_linear(double th, double s, double k, double a) {
    const double c = s * std::cos(th), sn = s * std::sin(th);
    const double p00 = a, p01 = a * k, p11 = 1 / a;
    return {c * p00, c * p01 - sn * p11, sn * p00, sn * p01 + c * p11};
}

// X ↦ c + L (X − c)
inline Mat3 about_c(const std::array<double, 2>& c, const Lin2& L) {
    return {L[0], L[1], c[0] - L[0] * c[0] - L[1] * c[1], L[2], L[3], c[1] - L[2] * c[0] - L[3] * c[1], 0, 0, 1};
}

// the 2×2 map's two singular values, the larger first
inline std::array<double, 2> sv2(const Lin2& L) {
    const double a = L[0] * L[0] + L[2] * L[2], b = L[0] * L[1] + L[2] * L[3], d = L[1] * L[1] + L[3] * L[3];
    const double t = 0.5 * (a + d), r = std::sqrt(std::max(0.0, 0.25 * (a - d) * (a - d) + b * b));
    return {std::sqrt(t + r), std::sqrt(std::max(0.0, t - r))};
}

inline std::array<double, 2> map_pt(const Mat3& H, double x, double y) {
    const double X = H[0] * x + H[1] * y + H[2], Y = H[3] * x + H[4] * y + H[5], Z = H[6] * x + H[7] * y + H[8];
    const double z = std::fabs(Z) < 1e-8 ? 1e-8 : Z;
    return {X / z, Y / z};
}

// canvas cells [lo, hi) covering dest-pixel extent [a, b], one cell of margin for the taps
inline std::array<int, 2> sweep_cells(double a, double b, double o0, double c, int G) {
    const long lo = std::clamp((long)std::floor((a - o0) / c) - 1, 0L, (long)G);
    const long hi = std::clamp((long)std::ceil((b - o0) / c) + 1, lo + 1, (long)G);
    return {(int)lo, (int)hi};
}

// plane length for `need` points: the compact list, else the smallest smooth length divisible by 16
inline unsigned sweep_plane_len(unsigned need, bool ladder) {
    static const unsigned kCompact[] = {32, 48, 64, 80, 96, 128, 160, 192, 224, 256, 320, 384, 448, 512};
    if (!ladder)
        for (unsigned L : kCompact)
            if (L >= need) return L;
    return plan_size(need, 16, ladder);
}

// A candidate's map peak: score in fixed pixels, the candidate's grid indices, the canvas shift
// (cells) and the pose T(−d)·H_c.
struct SweepPeak {
    double score;
    int cand, it, is, ik, ia;
    double th, s;
    int sx, sy;
    Mat3 H;
};

// Strongest first (stable); a peak survives only if no stronger survivor lies within ±2 θ steps
// (circular when wrap), ±2 σ steps, ±1 shear and stretch step and 4 cells.
inline std::vector<SweepPeak> nms4(const std::vector<SweepPeak>& peaks, unsigned n_theta, unsigned keep, bool wrap) {
    std::vector<SweepPeak> sorted = peaks;
    std::stable_sort(sorted.begin(), sorted.end(), [](const SweepPeak& a, const SweepPeak& b) { return a.score > b.score; });
    std::vector<SweepPeak> kept;
    for (const SweepPeak& p : sorted) {
        bool ok = true;
        for (const SweepPeak& q : kept) {
            const int a = std::abs(p.it - q.it);
            const int dt = wrap ? std::min(a, (int)n_theta - a) : a;
            if (dt <= 2 && std::abs(p.is - q.is) <= 2 && std::abs(p.ik - q.ik) <= 1 && std::abs(p.ia - q.ia) <= 1 &&
                std::hypot((double)(p.sx - q.sx), (double)(p.sy - q.sy)) <= 4) {
                ok = false;
                break;
            }
        }
        if (ok) {
            kept.push_back(p);
            if (kept.size() >= keep) break;
        }
    }
    return kept;
}

// a0, a0·r, a0·r², …: the step lengths tried along the unit ascent direction
inline std::vector<double> geo_amps(double a0, double ratio, unsigned n) {
    double a = a0 > 0 ? a0 : 0.08;
    const double r = std::min(0.95, std::max(0.2, ratio > 0 ? ratio : 0.5));
    const unsigned k = std::max(2u, std::min(12u, n));
    std::vector<double> out(k);
    for (unsigned i = 0; i < k; ++i, a *= r) out[i] = a;
    return out;
}

// How far H is turned (radians) and scaled from H0, read at moving-image point c (1-based).
inline std::array<double, 2> sim_of(const Mat3& H, const Mat3& H0, double cx, double cy) {
    auto jac = [&](const Mat3& M) -> std::array<double, 4> {
        const double w = M[6] * cx + M[7] * cy + M[8];
        const double x = (M[0] * cx + M[1] * cy + M[2]) / w, y = (M[3] * cx + M[4] * cy + M[5]) / w;
        return {(M[0] - M[6] * x) / w, (M[1] - M[7] * x) / w, (M[3] - M[6] * y) / w, (M[4] - M[7] * y) / w};
    };
    const auto J = jac(H), J0 = jac(H0);
    const double dr = J0[0] * J0[3] - J0[1] * J0[2];
    const double d0 = (dr == 0 || std::isnan(dr)) ? 1e-12 : dr;
    const double q00 = J0[3] / d0, q01 = -J0[1] / d0, q10 = -J0[2] / d0, q11 = J0[0] / d0;
    const double m00 = J[0] * q00 + J[1] * q10, m01 = J[0] * q01 + J[1] * q11;
    const double m10 = J[2] * q00 + J[3] * q10, m11 = J[2] * q01 + J[3] * q11;
    return {std::atan2(m10 - m01, m00 + m11), std::sqrt(std::fabs(m00 * m11 - m01 * m10))};
}

}  // namespace zc
