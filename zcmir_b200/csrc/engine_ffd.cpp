// The B-spline free-form deformation on top of the pose (the reference's Ffd state, src/pair.zig:
// 17-37 and 127-150, its control-point gradient ffdGrad 387-410 with src/pose.zig:520-572
// ffdGrads, and the engine's setFfdCps / zc_set_ffd / zc_get_ffd / zc_ffd_gradient,
// src/engine.zig:240-246, 281-285, 769-773): control points in half-image units of the
// lattice's image; the forward direction uses them as set, the inverse direction negated on the
// other image.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "engine.hpp"

namespace zc {

namespace {
constexpr int kMom = 45, kCoef = 102;
constexpr unsigned kFfdMax = 16;
}  // namespace

unsigned Engine::ffd_grid() {
    const unsigned g = std::min(std::max(set.u("ffd_grid"), 2u), kFfdMax);
    if (g != ffd_g_) {
        ffd_g_ = g;
        std::fill(ffd_cps_.begin(), ffd_cps_.end(), 0.f);
    }
    return g;
}

bool Engine::ffd_live() {
    if (!set.b("ffd") || ffd_suspended_) return false;
    const unsigned g = ffd_grid();
    for (size_t i = 0; i < 2 * (size_t)g * g; ++i)
        if (std::fabs(ffd_cps_[i]) > 1e-12) return true;
    return false;
}

bool Engine::set_ffd(const float* cps, size_t n) {
    const unsigned g = ffd_grid();
    if (n != 2 * (size_t)g * g)
        return fail("set_ffd: BadControlPoints (" + std::to_string(n) + " values for a " + std::to_string(g) + "×" +
                    std::to_string(g) + " lattice, which takes " + std::to_string(2 * g * g) + ")");
    std::memcpy(ffd_cps_.data(), cps, n * sizeof(float));
    return true;
}

size_t Engine::get_ffd(float* cps, size_t cap) {
    const unsigned g = ffd_grid();
    const size_t n = 2 * (size_t)g * g;
    if (cps) std::memcpy(cps, ffd_cps_.data(), std::min(n, cap) * sizeof(float));
    return n;
}

bool Engine::ffd_dirs(PoseFfd& fwd, PoseFfd& inv) {
    fwd = PoseFfd{};
    inv = PoseFfd{};
    if (!ffd_live()) return true;
    const unsigned g = ffd_grid();
    const size_t n = 2 * (size_t)g * g;
    // [forward | negated] (2 × 512 floats), stream-ordered before the passes that read it
    std::vector<float> h(2 * 2 * kFfdMax * kFfdMax, 0.f);
    for (size_t i = 0; i < n; ++i) {
        h[i] = ffd_cps_[i];
        h[2 * kFfdMax * kFfdMax + i] = -ffd_cps_[i];
    }
    if (!cuda_ok(ffd_dev_.ensure(h.size() * 4), "spline") ||
        !cuda_ok(cudaMemcpyAsync(ffd_dev_.p, h.data(), h.size() * 4, cudaMemcpyHostToDevice, st), "spline"))
        return false;
    const bool src = set.b("ffd_source");
    fwd = PoseFfd{ffd_dev_.as<float>(), (int)g, src ? 1 : 0};
    inv = PoseFfd{ffd_dev_.as<float>() + 2 * kFfdMax * kFfdMax, (int)g, src ? 0 : 1};
    return true;
}

bool Engine::ffd_gradient(const Mat3& H, double* score, double* grad, size_t len) {
    if (!need_images()) return false;
    if (!metric_ok("ffd_gradient")) return false;
    const unsigned g = ffd_grid();
    const size_t npar = 2 * (size_t)g * g;
    if (len < npar) return fail("ffd_gradient: BufferTooSmall (" + std::to_string(npar) + " values)");
    std::fill(grad, grad + npar, 0.0);
    *score = 0.0;
    if (!set.b("ffd")) return true;  // the spline is off: no gradient, score 0 (pair.zig:389-392)
    const bool live = ffd_live(), sym = set.b("symmetric") && live, exact = set.b("exact");
    // the forward direction takes the spline even when every control point is zero
    std::vector<float> h(2 * 2 * kFfdMax * kFfdMax, 0.f);
    for (size_t i = 0; i < npar; ++i) {
        h[i] = ffd_cps_[i];
        h[2 * kFfdMax * kFfdMax + i] = -ffd_cps_[i];
    }
    const int nchunk = (int)((g * g + 15) / 16), nd = sym ? 2 : 1;
    bool ok = cuda_ok(ffd_dev_.ensure(h.size() * 4), "ffd_gradient") &&
              cuda_ok(pose_hinv_.ensure(2 * 9 * 4), "ffd_gradient") &&
              cuda_ok(pose_sums_.ensure(2 * kMom * 8), "ffd_gradient") &&
              cuda_ok(pose_coef_.ensure(2 * kCoef * 4), "ffd_gradient") &&
              cuda_ok(pose_score_.ensure(2 * 8), "ffd_gradient") &&
              cuda_ok(ffd_out_.ensure((size_t)2 * nchunk * 32 * 8), "ffd_gradient");
    if (!ok) return false;
    const Mat3 Hi = inv3(H), Hii = inv3(Hi);
    float hinv[18];
    for (int k = 0; k < 9; ++k) hinv[k] = (float)Hi[k], hinv[9 + k] = (float)Hii[k];
    const Side &A = side[0], &B = side[1];
    const PoseSide pa{A.feat.as<float>(), A.feat4.as<float4>(), A.w, A.h},
        pb{B.feat.as<float>(), B.feat4.as<float4>(), B.w, B.h};
    const bool src = set.b("ffd_source");
    const PoseFfd ff{ffd_dev_.as<float>(), (int)g, src ? 1 : 0};
    const PoseFfd fi{ffd_dev_.as<float>() + 2 * kFfdMax * kFfdMax, (int)g, src ? 0 : 1};
    float* dh = pose_hinv_.as<float>();
    double* sums = pose_sums_.as<double>();
    float* coef = pose_coef_.as<float>();
    double* out = ffd_out_.as<double>();
    ok = cuda_ok(cudaMemcpyAsync(ffd_dev_.p, h.data(), h.size() * 4, cudaMemcpyHostToDevice, st), "ffd_gradient") &&
         cuda_ok(cudaMemcpyAsync(dh, hinv, sizeof hinv, cudaMemcpyHostToDevice, st), "ffd_gradient");
    PoseRed rd;
    ok = ok && pose_red(1, rd);
    for (int d = 0; ok && d < nd; ++d) {
        const PoseSide &a = d ? pb : pa, &b = d ? pa : pb;
        const PoseFfd& f = d ? fi : ff;
        ok = cuda_ok(pose_moments(a, b, dh + 9 * d, 1, sums + kMom * d, st, f, nullptr, rd), "ffd_gradient") &&
             cuda_ok(pose_coefs(sums + kMom * d, 1, exact, coef + kCoef * d, pose_score_.as<double>() + d, st),
                     "ffd_gradient");
        for (int c = 0; ok && c < nchunk; ++c)
            ok = cuda_ok(pose_ffd_grad(a, b, dh + 9 * d, coef + kCoef * d, f, 16 * c, out + ((size_t)d * nchunk + c) * 32, st,
                                       rd),
                         "ffd_gradient");
    }
    if (!ok) return false;
    std::vector<double> hs(2 * kMom), hsc(2), hg((size_t)2 * nchunk * 32);
    if (!cuda_ok(cudaMemcpyAsync(hs.data(), sums, (size_t)nd * kMom * 8, cudaMemcpyDeviceToHost, st), "ffd_gradient") ||
        !cuda_ok(cudaMemcpyAsync(hsc.data(), pose_score_.p, (size_t)nd * 8, cudaMemcpyDeviceToHost, st), "ffd_gradient") ||
        !cuda_ok(cudaMemcpyAsync(hg.data(), out, (size_t)nd * nchunk * 32 * 8, cudaMemcpyDeviceToHost, st),
                 "ffd_gradient") ||
        !cuda_ok(cudaStreamSynchronize(st), "ffd_gradient"))
        return false;
    counts[0] += nd * (2 + nchunk);
    counts[1]++;
    counts[2] += 3;
    counts[3]++;
    auto fin = [](double v) { return std::isfinite(v) ? v : 0.0; };
    // one direction's gradient: zero under the overlap floor, non-finite entries zeroed
    auto dir = [&](int d, std::vector<double>& gv) {
        gv.assign(npar, 0.0);
        if (!(hs[(size_t)d * kMom] >= 12.0)) return;
        for (size_t k = 0; k < npar; ++k) gv[k] = fin(hg[((size_t)d * nchunk + k / 32) * 32 + k % 32]);
    };
    std::vector<double> gf, gi;
    dir(0, gf);
    if (!sym) {
        for (size_t k = 0; k < npar; ++k) grad[k] = gf[k];
        *score = fin(hsc[0]);
        return true;
    }
    dir(1, gi);
    for (size_t k = 0; k < npar; ++k) grad[k] = 0.5 * (gf[k] - gi[k]);
    *score = 0.5 * (fin(hsc[0]) + fin(hsc[1]));
    return true;
}

}  // namespace zc

namespace zc {

namespace {

constexpr int kPack = 2 * 16 * 16;  // floats per pose in a device pack of control points
constexpr int kFfdMus = 6;           // the spline step's lengths (climb.wgsl FFD_MUS)

// The spline's bending energy as a quadratic form over its parameters (x, y per control point,
// half-image units) (src/gclimb.zig:253-293 bendingEnergy): the thin-plate energy Σ f_xx² +
// 2 f_xy² + f_yy² of the displacement in pixels from second differences on the lattice, the
// spacing's powers included. lw × lh: the lattice's image.
std::vector<double> bending_energy(int g, double lw, double lh) {
    const int n = 2 * g * g;
    std::vector<double> R((size_t)n * n, 0.0);
    const double hx[2] = {std::max(lw, 1.0) * 0.5, std::max(lh, 1.0) * 0.5};
    const double gf = std::max(g, 2) - 1;
    const double sp[2] = {std::max(lw - 1, 1.0) / gf, std::max(lh - 1, 1.0) / gf};
    const double area = sp[0] * sp[1];
    struct Tap {
        int i, j, c;
    };
    auto add = [&](std::initializer_list<Tap> taps, int comp, double w) {
        for (const Tap& a : taps)
            for (const Tap& b : taps) {
                const int ia = a.j * g + a.i, ib = b.j * g + b.i;
                R[(size_t)(2 * ia + comp) * n + 2 * ib + comp] += w * (double)(a.c * b.c);
            }
    };
    for (int comp = 0; comp < 2; ++comp) {
        const double s2 = hx[comp] * hx[comp];
        for (int j = 0; j < g; ++j)
            for (int i = 0; i < g; ++i) {
                if (i >= 1 && i + 1 < g)
                    add({{i - 1, j, 1}, {i, j, -2}, {i + 1, j, 1}}, comp, s2 * area / (sp[0] * sp[0] * sp[0] * sp[0]));
                if (j >= 1 && j + 1 < g)
                    add({{i, j - 1, 1}, {i, j, -2}, {i, j + 1, 1}}, comp, s2 * area / (sp[1] * sp[1] * sp[1] * sp[1]));
                if (i + 1 < g && j + 1 < g)
                    add({{i, j, 1}, {i + 1, j, -1}, {i, j + 1, -1}, {i + 1, j + 1, 1}}, comp,
                        2 * s2 * area / (sp[0] * sp[0] * sp[1] * sp[1]));
            }
    }
    return R;
}

// Q symmetrised and projected onto the positive semi-definite cone (its eigenvalues clipped at
// 0; cyclic Jacobi rotations, smi.wgsl:2020-2062 psd4): the spline's banded Cholesky needs a
// positive definite Gauss–Newton matrix.
void psd4(const float* q, float* out) {
    double a[16], v[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) a[i * 4 + j] = 0.5 * ((double)q[i * 4 + j] + (double)q[j * 4 + i]);
    for (int sweep = 0; sweep < 12; ++sweep)
        for (int p = 0; p < 3; ++p)
            for (int r = p + 1; r < 4; ++r) {
                const double apr = a[p * 4 + r];
                if (std::fabs(apr) < 1e-300) continue;
                const double th = (a[r * 4 + r] - a[p * 4 + p]) / (2.0 * apr);
                const double t = (th >= 0 ? 1.0 : -1.0) / (std::fabs(th) + std::sqrt(th * th + 1.0));
                const double c = 1.0 / std::sqrt(t * t + 1.0), sn = t * c;
                for (int k = 0; k < 4; ++k) {
                    const double akp = a[k * 4 + p], akr = a[k * 4 + r];
                    a[k * 4 + p] = c * akp - sn * akr;
                    a[k * 4 + r] = sn * akp + c * akr;
                }
                for (int k = 0; k < 4; ++k) {
                    const double apk = a[p * 4 + k], ark = a[r * 4 + k];
                    a[p * 4 + k] = c * apk - sn * ark;
                    a[r * 4 + k] = sn * apk + c * ark;
                }
                for (int k = 0; k < 4; ++k) {
                    const double vkp = v[k * 4 + p], vkr = v[k * 4 + r];
                    v[k * 4 + p] = c * vkp - sn * vkr;
                    v[k * 4 + r] = sn * vkp + c * vkr;
                }
            }
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
            double x = 0;
            for (int k = 0; k < 4; ++k) x += v[i * 4 + k] * std::max(a[k * 4 + k], 0.0) * v[j * 4 + k];
            out[i * 4 + j] = (float)x;
        }
}

int tri4h(int a, int b) {
    const int i = std::min(a, b), j = std::max(a, b);
    return i * 4 - (i * (i + 1)) / 2 + j;
}

}  // namespace

namespace {

// the displacement (pixels, float64) of the spline at a 0-based point of its rw × rh image
// (src/export.zig:26-62 ffdDisp)
void disp64(const float* cps, int g, double x, double y, double w, double h, double& dx, double& dy) {
    dx = dy = 0;
    if (g < 2 || x < 0 || y < 0 || x > w - 1 || y > h - 1) return;
    const double hx = w * 0.5, hy = h * 0.5;
    const double spx = std::max(w - 1, 1.0) / (g - 1), spy = std::max(h - 1, 1.0) / (g - 1);
    const double su = x / spx, sv = y / spy, iu = std::floor(su), iv = std::floor(sv);
    auto cw = [](double t, double* b) {
        const double t2 = t * t, t3 = t2 * t;
        b[0] = (1 - t) * (1 - t) * (1 - t) / 6, b[1] = (3 * t3 - 6 * t2 + 4) / 6;
        b[2] = (-3 * t3 + 3 * t2 + 3 * t + 1) / 6, b[3] = t3 / 6;
    };
    double bu[4], bv[4];
    cw(std::min(1.0, std::max(0.0, su - iu)), bu);
    cw(std::min(1.0, std::max(0.0, sv - iv)), bv);
    for (int jj = 0; jj < 4; ++jj) {
        const int j = std::min(g - 1, std::max(0, (int)iv - 1 + jj));
        for (int ii = 0; ii < 4; ++ii) {
            const int i = std::min(g - 1, std::max(0, (int)iu - 1 + ii));
            const double wt = bu[ii] * bv[jj];
            const int o = (j * g + i) * 2;
            dx += wt * cps[o] * hx;
            dy += wt * cps[o + 1] * hy;
        }
    }
}

}  // namespace

bool Engine::displacement(float* out, size_t len) {
    if (!side[0].has || !side[1].has) return fail("displacement: NoImages");
    const int lw = side[0].w, lh = side[0].h, rw = side[1].w, rh = side[1].h;
    const size_t n = (size_t)rw * rh * 2;
    if (len < n) return fail("displacement: BufferTooSmall (" + std::to_string(n) + " values)");
    const bool on = set.b("ffd"), src = set.b("ffd_source");
    const int g = (int)ffd_grid();
    const Mat3 Hi = inv3(H);
    auto apply = [&](double x, double y, double& ox, double& oy) {
        const double X = Hi[0] * x + Hi[1] * y + Hi[2], Y = Hi[3] * x + Hi[4] * y + Hi[5], Z = Hi[6] * x + Hi[7] * y + Hi[8];
        if (std::fabs(Z) < 1e-12) return false;
        ox = X / Z, oy = Y / Z;
        return true;
    };
    for (int y = 0; y < rh; ++y)
        for (int x = 0; x < rw; ++x) {
            double px = NAN, py = NAN, qx, qy, dx, dy;
            if (on && src) {
                if (apply(x + 1, y + 1, qx, qy)) {
                    disp64(ffd_cps_.data(), g, qx - 1, qy - 1, lw, lh, dx, dy);
                    px = qx - 1 + dx, py = qy - 1 + dy;
                }
            } else if (on) {
                disp64(ffd_cps_.data(), g, x, y, rw, rh, dx, dy);
                if (apply(x + 1 + dx, y + 1 + dy, qx, qy)) px = qx - 1, py = qy - 1;
            } else if (apply(x + 1, y + 1, qx, qy)) {
                px = qx - 1, py = qy - 1;
            }
            const size_t k = ((size_t)y * rw + x) * 2;
            out[k] = std::isfinite(px) ? (float)(px - x) : 0.f;
            out[k + 1] = std::isfinite(py) ? (float)(py - y) : 0.f;
        }
    return true;
}

bool Engine::ffd_pose_dirs(const float* cps, int n, PoseFfd& fwd, PoseFfd& inv) {
    const unsigned g = ffd_grid();
    const size_t np = 2 * (size_t)g * g;
    std::vector<float> h((size_t)2 * n * kPack, 0.f);
    for (int p = 0; p < n; ++p)
        for (size_t i = 0; i < np; ++i) {
            h[(size_t)p * kPack + i] = cps[(size_t)p * np + i];
            h[((size_t)n + p) * kPack + i] = -cps[(size_t)p * np + i];
        }
    if (!cuda_ok(ffd_pk_.ensure(h.size() * 4), "spline") ||
        !cuda_ok(cudaMemcpyAsync(ffd_pk_.p, h.data(), h.size() * 4, cudaMemcpyHostToDevice, st), "spline") ||
        !cuda_ok(cudaStreamSynchronize(st), "spline"))
        return false;
    const bool src = set.b("ffd_source");
    fwd = PoseFfd{ffd_pk_.as<float>(), (int)g, src ? 1 : 0, kPack};
    inv = PoseFfd{ffd_pk_.as<float>() + (size_t)n * kPack, (int)g, src ? 0 : 1, kPack};
    return true;
}

bool Engine::spline_stage(const Mat3& H, double& lam, bool& moved, double& score) {
    moved = false;
    const int g = (int)ffd_grid(), np = 2 * g * g, ncell = g * g;
    const bool sym = set.b("symmetric"), src = set.b("ffd_source");
    const int nd = sym ? 2 : 1;
    // the current pose's coefficients in both directions (the spline as it is)
    std::vector<PoseEval> ev;
    if (!eval_poses({H}, false, false, ev)) return false;
    std::vector<float> coef(2 * 102);
    if (!cuda_ok(cudaMemcpyAsync(coef.data(), pose_coef_.p, (size_t)nd * 102 * 4, cudaMemcpyDeviceToHost, st), "spline") ||
        !cuda_ok(cudaStreamSynchronize(st), "spline"))
        return false;
    for (int d = 0; d < nd; ++d) psd4(&coef[d * 102 + 85], &coef[d * 102 + 85]);
    // the spline in both directions, present even when zero (the stage's gradient needs it)
    std::vector<float> cur_cps(ffd_cps_.begin(), ffd_cps_.begin() + np);
    PoseFfd ff, fi;
    if (!ffd_pose_dirs(cur_cps.data(), 1, ff, fi)) return false;
    const Side &A = side[0], &B = side[1];
    const PoseSide pa{A.feat.as<float>(), A.feat4.as<float4>(), A.w, A.h},
        pb{B.feat.as<float>(), B.feat4.as<float4>(), B.w, B.h};
    const Mat3 Hi = inv3(H), Hii = inv3(Hi);
    float mats[36];  // per direction: hinv, pose
    for (int k = 0; k < 9; ++k) {
        mats[k] = (float)Hi[k], mats[9 + k] = (float)H[k];
        mats[18 + k] = (float)Hii[k], mats[27 + k] = (float)Hi[k];
    }
    int nch[2];
    size_t off[2], total = 0;
    for (int d = 0; d < nd; ++d) {
        const PoseSide& b = d ? pa : pb;
        nch[d] = (int)std::min<size_t>(std::max<size_t>(((size_t)b.w * b.h / ncell + 2047) / 2048, 1), 64);
        off[d] = total;
        total += (size_t)ncell * nch[d] * kFfdCell;
    }
    if (!cuda_ok(ffd_coef_.ensure(2 * 102 * 4 + sizeof mats), "spline") || !cuda_ok(ffd_cells_.ensure(total * 4), "spline"))
        return false;
    float* dcoef = ffd_coef_.as<float>();
    float* dmat = dcoef + 2 * 102;
    bool ok = cuda_ok(cudaMemcpyAsync(dcoef, coef.data(), 2 * 102 * 4, cudaMemcpyHostToDevice, st), "spline") &&
              cuda_ok(cudaMemcpyAsync(dmat, mats, sizeof mats, cudaMemcpyHostToDevice, st), "spline");
    for (int d = 0; ok && d < nd; ++d)
        ok = cuda_ok(pose_ffd_cells(d ? pb : pa, d ? pa : pb, dmat + 18 * d, dmat + 18 * d + 9, dcoef + 102 * d,
                                    d ? fi : ff, nch[d], ffd_cells_.as<float>() + off[d], st),
                     "spline");
    std::vector<float> cells(total);
    if (!ok || !cuda_ok(cudaMemcpyAsync(cells.data(), ffd_cells_.p, total * 4, cudaMemcpyDeviceToHost, st), "spline") ||
        !cuda_ok(cudaStreamSynchronize(st), "spline"))
        return false;
    counts[0] += nd;
    counts[2] += 2;
    counts[3]++;
    // assemble the gradient and the Gauss–Newton matrix over the control points (climb.wgsl
    // ffd_assemble): every cell's 4 × 4 taps (clamped, as the displacement clamps) pairwise;
    // symmetric: ½ (A_fwd + A_inv), ½ (g_fwd − g_inv)
    std::vector<double> grad(np, 0.0), Am((size_t)np * np, 0.0);
    for (int d = 0; d < nd; ++d) {
        const double f = nd == 2 ? 0.5 : 1.0, sg = d == 1 ? -1.0 : 1.0;
        std::vector<double> S(kFfdCell);
        for (int cell = 0; cell < ncell; ++cell) {
            std::fill(S.begin(), S.end(), 0.0);
            for (int c = 0; c < nch[d]; ++c) {
                const float* o = &cells[off[d] + ((size_t)cell * nch[d] + c) * kFfdCell];
                for (int q = 0; q < kFfdCell; ++q) S[q] += (double)o[q];
            }
            const int iu = cell % g, iv = cell / g;
            auto cl = [&](int v) { return std::min(std::max(v, 0), g - 1); };
            for (int jj = 0; jj < 4; ++jj)
                for (int ii = 0; ii < 4; ++ii) {
                    const int k = cl(iv - 1 + jj) * g + cl(iu - 1 + ii);
                    const double gx = S[300 + (ii + 4 * jj) * 2], gy = S[300 + (ii + 4 * jj) * 2 + 1];
                    if (std::fabs(gx) < 1e30) grad[2 * k] += f * sg * gx;
                    if (std::fabs(gy) < 1e30) grad[2 * k + 1] += f * sg * gy;
                    for (int jj2 = 0; jj2 < 4; ++jj2)
                        for (int ii2 = 0; ii2 < 4; ++ii2) {
                            const int l = cl(iv - 1 + jj2) * g + cl(iu - 1 + ii2);
                            const int q = (tri4h(ii, ii2) * 10 + tri4h(jj, jj2)) * 3;
                            Am[(size_t)(2 * k) * np + 2 * l] += f * S[q];
                            Am[(size_t)(2 * k) * np + 2 * l + 1] += f * S[q + 1];
                            Am[(size_t)(2 * k + 1) * np + 2 * l] += f * S[q + 1];
                            Am[(size_t)(2 * k + 1) * np + 2 * l + 1] += f * S[q + 2];
                        }
                }
        }
    }
    // λ = c (s L / 2π)⁴ with c the score's curvature per pixel: p1 · tr A at the first spline step
    // (src/gclimb.zig:214-229)
    const double lw = src ? A.w : B.w, lh = src ? A.h : B.h;
    const std::vector<double> R = bending_energy(g, lw, lh);
    if (lam < 0) {
        const double area = std::max(lw - 1, 1.0) * std::max(lh - 1, 1.0);
        const double bsq = (151.0 / 315.0) * (151.0 / 315.0);
        const double s = set.f("ffd_stiffness");
        const double p1 = s * s * s * s * area /
                          (bsq * std::max(lw, 1.0) * 0.5 * std::max(lh, 1.0) * 0.5 * std::pow(2 * M_PI, 4));
        double ta = 0;
        for (int i = 0; i < np; ++i) ta += Am[(size_t)i * np + i];
        lam = ta > 0 ? p1 * ta : 0.0;
    }
    // (A + λR + damping) δ = ½ g − λ R c on the band (climb.wgsl ffd_solve), in float64
    const int hb = 2 * (3 * g + 3) + 1;
    std::vector<double> M((size_t)np * np, 0.0), rhs(np);
    for (int i = 0; i < np; ++i)
        for (int j = std::max(0, i - hb); j < std::min(np, i + hb + 1); ++j)
            M[(size_t)i * np + j] = Am[(size_t)i * np + j] + lam * R[(size_t)i * np + j];
    for (int i = 0; i < np; ++i) {
        double rc = 0;
        for (int j = std::max(0, i - hb); j < std::min(np, i + hb + 1); ++j) rc += R[(size_t)i * np + j] * cur_cps[j];
        rhs[i] = 0.5 * grad[i] - lam * rc;
    }
    double tm = 0;
    for (int i = 0; i < np; ++i) tm += std::fabs(M[(size_t)i * np + i]);
    const double fl = 1e-3 * tm / std::max(np, 1) + 1e-20;
    for (int i = 0; i < np; ++i) M[(size_t)i * np + i] = M[(size_t)i * np + i] * 1.01 + fl;
    bool solved = true;
    for (int j = 0; j < np && solved; ++j) {  // banded Cholesky, L in the lower triangle
        double dj = M[(size_t)j * np + j];
        for (int k = std::max(0, j - hb); k < j; ++k) dj -= M[(size_t)j * np + k] * M[(size_t)j * np + k];
        if (!(dj > 0)) {
            solved = false;
            break;
        }
        dj = std::sqrt(dj);
        M[(size_t)j * np + j] = dj;
        for (int i = j + 1; i < std::min(np, j + hb + 1); ++i) {
            double s = M[(size_t)i * np + j];
            for (int k = std::max(0, i - hb); k < j; ++k) s -= M[(size_t)i * np + k] * M[(size_t)j * np + k];
            M[(size_t)i * np + j] = s / dj;
        }
    }
    std::vector<double> delta(np, 0.0);
    if (solved) {
        for (int i = 0; i < np; ++i) {
            double s = rhs[i];
            for (int k = std::max(0, i - hb); k < i; ++k) s -= M[(size_t)i * np + k] * delta[k];
            delta[i] = s / M[(size_t)i * np + i];
        }
        for (int i = np - 1; i >= 0; --i) {
            double s = delta[i];
            for (int k = i + 1; k < std::min(np, i + hb + 1); ++k) s -= M[(size_t)k * np + i] * delta[k];
            delta[i] = s / M[(size_t)i * np + i];
            if (!(std::fabs(delta[i]) < 1e30)) solved = false;
        }
    }
    // candidates c + μ δ (μ = ½ … 16, the ladder scaled down so its top moves no point more than
    // 0.2 lattice spacings), then c itself; each scored less its bending penalty λ pᵀ R p
    // (climb.wgsl ffd_gn_cands, climb_select)
    const double p0 = 0.2 * 2.0 / (double)(std::max(g, 2) - 1);
    double mx = 0;
    for (double v : delta) mx = std::max(mx, std::fabs(v));
    const double scale = mx * 16.0 > p0 ? p0 / (16.0 * mx) : 1.0;
    const double mus[kFfdMus] = {0.5, 1.0, 2.0, 4.0, 8.0, 16.0};
    std::vector<float> cands((size_t)(kFfdMus + 1) * np);
    double pen[kFfdMus + 1];
    for (int t = 0; t <= kFfdMus; ++t) {
        const double a = (t < kFfdMus && solved) ? mus[t] * scale : 0.0;
        for (int i = 0; i < np; ++i) cands[(size_t)t * np + i] = (float)((double)cur_cps[i] + a * delta[i]);
        double s = 0;
        for (int i = 0; i < np; ++i) {
            double rp = 0;
            for (int j = std::max(0, i - hb); j < std::min(np, i + hb + 1); ++j)
                rp += R[(size_t)i * np + j] * (double)cands[(size_t)t * np + j];
            s += (double)cands[(size_t)t * np + i] * rp;
        }
        pen[t] = std::max(lam, 0.0) * s;
    }
    std::vector<Mat3> Hs(kFfdMus + 1, H);
    std::vector<PoseEval> sc;
    if (!eval_poses(Hs, false, false, sc, false, cands.data())) return false;
    const double cur = sc[kFfdMus].mean - pen[kFfdMus];
    int best = -1;
    double best_s = cur;
    for (int t = 0; t < kFfdMus; ++t) {
        const double o = sc[t].mean - pen[t];
        if (o > cur + std::max(1e-6 * std::fabs(cur), 1e-12) && (best < 0 || o > best_s)) {
            best = t;
            best_s = o;
        }
    }
    score = sc[best < 0 ? kFfdMus : best].mean;
    if (best < 0) return true;
    std::copy(cands.begin() + (size_t)best * np, cands.begin() + (size_t)(best + 1) * np, ffd_cps_.begin());
    moved = true;
    return true;
}

}  // namespace zc
