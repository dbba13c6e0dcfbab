// Host pose geometry for the SMI path: 3×3 algebra, the canvas of a pose and the map plans.
// Restated from the reference's src/lie.zig (inv3 85-117, regFrame 537-574, canvasH 577-579),
// src/smi.zig (autoShiftPlan 35-47, capN 414-422) and src/fft.zig (planSize 20-25, largestSmooth
// 37-43, linearCorrPlanRect 96-109).
#pragma once

#include <algorithm>
#include <array>
#include <cmath>

namespace zc {

using Mat3 = std::array<double, 9>;

inline Mat3 mat_identity() { return {1, 0, 0, 0, 1, 0, 0, 0, 1}; }

inline Mat3 mul3(const Mat3& a, const Mat3& b) {
    Mat3 o{};
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) o[r * 3 + c] = a[r * 3] * b[c] + a[r * 3 + 1] * b[3 + c] + a[r * 3 + 2] * b[6 + c];
    return o;
}

inline double det3(const Mat3& m) {
    return m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) + m[2] * (m[3] * m[7] - m[4] * m[6]);
}

// Inverse with one Newton refinement step (the reference's inv3).
inline Mat3 inv3(const Mat3& m) {
    const double a = m[0], b = m[1], c = m[2], d = m[3], e = m[4], f = m[5], g = m[6], h = m[7], i = m[8];
    const double A = e * i - f * h, B = f * g - d * i, C = d * h - e * g;
    const double D = c * h - b * i, E = a * i - c * g, F = b * g - a * h;
    const double G = b * f - c * e, Hh = c * d - a * f, I = a * e - b * d;
    const double det = a * A + b * B + c * C;
    const double sg = det > 0 ? 1.0 : (det < 0 ? -1.0 : 0.0);
    const double s = 1.0 / (sg * std::max(std::fabs(det), 1e-18));
    const Mat3 inv{A * s, D * s, G * s, B * s, E * s, Hh * s, C * s, F * s, I * s};
    const Mat3 p = mul3(m, inv);
    const Mat3 corr{2 - p[0], -p[1], -p[2], -p[3], 2 - p[4], -p[5], -p[6], -p[7], 2 - p[8]};
    return mul3(inv, corr);
}

// Plain adjugate / determinant inverse (what the canvas warp uses).
inline Mat3 inv3_plain(const Mat3& m) {
    const double a = m[0], b = m[1], c = m[2], d = m[3], e = m[4], f = m[5], g = m[6], h = m[7], i = m[8];
    const double A = e * i - f * h, B = f * g - d * i, C = d * h - e * g;
    const double det = a * A + b * B + c * C;
    const double s = 1.0 / det;
    return {A * s, (c * h - b * i) * s, (b * f - c * e) * s, B * s, (a * i - c * g) * s, (c * d - a * f) * s,
            C * s, (b * g - a * h) * s, (a * e - b * d) * s};
}

inline Mat3 translate(double dx, double dy) { return {1, 0, dx, 0, 1, dy, 0, 0, 1}; }

struct Frame {
    int ox, oy, w, h;
};

// The fixed image plus the moving image's warped corners, clipped to ±2·max(size).
inline Frame reg_frame(const Mat3& H, int lw, int lh, int rw, int rh) {
    double xs_min = 0, ys_min = 0, xs_max = rw, ys_max = rh;
    const double lim = std::max({(double)lw, (double)rw, (double)lh, (double)rh, 8.0}) * 2;
    const double cs[4][2] = {{1, 1}, {(double)lw, 1}, {(double)lw, (double)lh}, {1, (double)lh}};
    for (auto& p : cs) {
        const double x = H[0] * p[0] + H[1] * p[1] + H[2];
        const double y = H[3] * p[0] + H[4] * p[1] + H[5];
        const double z = H[6] * p[0] + H[7] * p[1] + H[8];
        const double zz = std::fabs(z) < 1e-8 ? 1e-8 : z;
        xs_min = std::min(xs_min, x / zz - 1);
        xs_max = std::max(xs_max, x / zz - 1);
        ys_min = std::min(ys_min, y / zz - 1);
        ys_max = std::max(ys_max, y / zz - 1);
    }
    auto clip = [&](double v) { return std::min(lim, std::max(-lim, v)); };
    const double ox = std::min(std::floor(clip(xs_min)), 0.0);
    const double oy = std::min(std::floor(clip(ys_min)), 0.0);
    const double x1 = std::max(std::ceil(clip(xs_max)), (double)rw);
    const double y1 = std::max(std::ceil(clip(ys_max)), (double)rh);
    return {(int)ox, (int)oy, (int)std::max(8.0, x1 - ox), (int)std::max(8.0, y1 - oy)};
}

inline Mat3 canvas_H(const Mat3& H, int ox, int oy) { return mul3(translate(-ox, -oy), H); }

// ── FFT length plans ──

inline bool smooth_len(unsigned n, bool ladder) {
    const unsigned ladder_p[] = {2, 3}, compact_p[] = {2, 3, 5, 7, 11, 13};
    const unsigned* ps = ladder ? ladder_p : compact_p;
    const int np = ladder ? 2 : 6;
    for (int k = 0; k < np; ++k)
        while (n % ps[k] == 0) n /= ps[k];
    return n == 1;
}

inline unsigned plan_size(unsigned target, unsigned div, bool ladder) {
    unsigned n = std::max(target, 1u);
    while (!(n % div == 0 && smooth_len(n, ladder))) ++n;
    return n;
}

inline unsigned largest_smooth(unsigned max_n, bool ladder) {
    unsigned n = std::max(32u, max_n);
    while (n >= 32) {
        if (smooth_len(n, ladder)) return n;
        --n;
    }
    return 32;
}

struct MapPlan {
    int nx, ny, cw, ch;
};

inline unsigned js_round(double x) { return (unsigned)std::floor(x + 0.5); }

inline MapPlan linear_corr_plan_rect(int w, int h, unsigned max_n0, bool ladder) {
    const unsigned max_n = largest_smooth(max_n0, ladder);
    double s = std::min(1.0, (double)std::max(8u, max_n >> 1) / (double)std::max(std::max(w, h), 1));
    for (int i = 0; i < 16; ++i) {
        const unsigned cw = std::max(8u, js_round(w * s)), ch = std::max(8u, js_round(h * s));
        const unsigned nx = std::min(plan_size(std::max(cw + cw - 1, 32u), 1, ladder), max_n);
        const unsigned ny = std::min(plan_size(std::max(ch + ch - 1, 32u), 1, ladder), max_n);
        if (nx >= cw + cw - 1 && ny >= ch + ch - 1) return {(int)nx, (int)ny, (int)cw, (int)ch};
        s *= 0.85;
    }
    const int m = (int)std::max(8u, (max_n + 1) >> 1);
    return {(int)max_n, (int)max_n, m, m};
}

// (n, cw, ch): one FFT length for both axes (src/fft.zig:70-91 linearCorrPlan, the NCC map's)
inline MapPlan linear_corr_plan(int w, int h, unsigned max_n0, bool ladder) {
    const unsigned max_n = largest_smooth(max_n0, ladder);
    double s = std::min(1.0, (double)std::max(8u, max_n >> 1) / (double)std::max(std::max(w, h), 1));
    unsigned n = 8, cw = 8, ch = 8;
    for (int i = 0; i < 16; ++i) {
        cw = std::max(8u, js_round(w * s));
        ch = std::max(8u, js_round(h * s));
        n = std::min(plan_size(std::max({cw + cw - 1, ch + ch - 1, 32u}), 1, ladder), max_n);
        if (n >= cw + cw - 1 && n >= ch + ch - 1) return {(int)n, (int)n, (int)cw, (int)ch};
        s *= 0.85;
    }
    cw = std::max(8u, std::min(cw, (n + 1) >> 1));
    ch = std::max(8u, std::min(ch, (n + 1) >> 1));
    return {(int)n, (int)n, (int)cw, (int)ch};
}

constexpr unsigned kMapAutoMin = 128, kMapAutoMax = 512, kMapCap = 1024;

inline MapPlan auto_shift_plan(int w, int h) {
    const unsigned d = (unsigned)std::max({w, h, 1});
    unsigned g = 1;
    while (2 * ((d + g - 1) / g) - 1 > kMapAutoMax) g *= 2;
    const unsigned cw = std::max(1u, ((unsigned)w + g - 1) / g), ch = std::max(1u, ((unsigned)h + g - 1) / g);
    auto pow2 = [](unsigned need) {
        unsigned p = 1;
        while (p < std::max(need, 1u)) p <<= 1;
        return std::min(std::max(p, kMapAutoMin), kMapAutoMax);
    };
    return {(int)pow2(2 * cw - 1), (int)pow2(2 * ch - 1), (int)cw, (int)ch};
}

}  // namespace zc
