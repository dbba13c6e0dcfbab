// The roto-scale map (the reference's Smi.rsMap / rsMapFrom, src/smi.zig:574-651, and Engine.rsMap,
// src/engine.zig:831-872): the canvas stacks of a pose resampled on log-polar coordinates about a
// centre, so a rotation becomes a shift in angle and a scaling a shift in log radius; the same
// correlations and score as the shift map on those planes give the score of every rotation and
// scale. Symmetric maps average the inverse-frame map in at the mirrored lag.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "engine.hpp"

namespace zc {

namespace {

constexpr unsigned kRsAutoMin = 128, kRsAutoMax = 512;  // src/smi.zig:29-30

unsigned ceil_pow2(unsigned v) {
    unsigned p = 1;
    while (p < v) p <<= 1;
    return p;
}

}  // namespace

bool Engine::rs_map_one(const Mat3& H, const double c[2], double r0_opt, double r1_opt, bool exact, bool calibrated,
                        unsigned cap, DevBuf& dst, RsPlan& p) {
    const Side &A = side[0], &B = side[1];
    const bool ladder = set.e("fft_sizes") == "ladder";
    if (!ladder) return fail("rs_map: fft_sizes=\"compact\" is not supported by this build (use \"ladder\")");
    const Frame fr = reg_frame(H, A.w, A.h, B.w, B.h);
    const Mat3 Hc = canvas_H(H, fr.ox, fr.oy);
    p = RsPlan{};
    p.cx = c[0] - 1 - fr.ox;
    p.cy = c[1] - 1 - fr.oy;
    // radii: out to the farthest canvas corner unless pinned (the inverse-frame map shares the
    // forward map's), in from r_out/16 clamped to [2, 8]
    double r1 = r1_opt;
    if (r1 == 0) {
        const double W = fr.w, Hh = fr.h;
        const double q[4][2] = {{0, 0}, {W - 1, 0}, {W - 1, Hh - 1}, {0, Hh - 1}};
        for (const auto& v : q) r1 = std::max(r1, std::hypot(v[0] - p.cx, v[1] - p.cy));
    }
    const double r0 = r0_opt > 0 ? r0_opt : std::max(2.0, std::min(r1 / 16, 8.0));
    const double r_out = std::max(r1, 2.0);
    const double r_in = std::min(std::max(r0, 1e-3), r_out / 8);
    const unsigned n_ring = std::max(64u, (unsigned)std::ceil(2 * M_PI * r_out));
    unsigned n;
    if (cap == 0) {
        n = std::clamp(ceil_pow2(n_ring), kRsAutoMin, kRsAutoMax);
    } else {
        n = std::min(plan_size(n_ring, 1, ladder), largest_smooth(std::min<unsigned>(cap, kMaxLine), ladder));
    }
    p.n = (int)n;
    p.n_th = (int)n;
    p.n_lam = std::max(16, (int)(n >> 1));
    p.log0 = std::log(r_in);
    p.span = std::log(r_out) - p.log0;
    p.dlam = p.span / p.n_lam;
    p.dth = 2 * M_PI / p.n_th;
    p.r0 = r_in;
    p.r1 = r_out;
    MapGeom g{};
    g.W = p.n_th, g.Hh = p.n_lam, g.ox = fr.ox, g.oy = fr.oy;
    g.cw = p.n_th, g.ch = p.n_lam, g.nx = p.n, g.ny = p.n;
    g.WP = ((g.nx / 2 + 1) + 7) / 8 * 8;
    const CorrPlanDev plan = corr_plan_dev(exact, side[0].mode == 1);
    LinePlan row, col, line;
    if (!line_plan(g.nx, row) || !line_plan(g.ny, col)) return false;
    const int S = row_split(g.nx, plan.n_corr);
    if (S == 0) return fail("rs_map: a row of " + std::to_string(g.nx) + " does not fit the row pass");
    if (!line_plan(g.nx / S, line)) return false;
    const float2* tw = twiddles(g.nx);
    if (!tw) return fail("rs_map: twiddles: out of device memory");
    const size_t cn = (size_t)fr.w * fr.h, gn = (size_t)p.n_th * p.n_lam, nn = (size_t)p.n * p.n;
    const size_t hs = (size_t)plan.n_real * g.ny * g.WP * sizeof(float2);
    const size_t qs = (size_t)plan.n_corr * g.ny * g.WP * sizeof(float2);
    forget_spectra();  // this map writes the map path's canvas and spectrum buffers
    bool ok = cuda_ok(canvas_a_.ensure(cn * 20), "rs_map") && cuda_ok(canvas_b_.ensure(cn * 20), "rs_map") &&
              cuda_ok(grid_a_.ensure(gn * 20), "rs_map") && cuda_ok(grid_b_.ensure(gn * 20), "rs_map") &&
              cuda_ok(half_a_.ensure(hs), "rs_map") && cuda_ok(half_b_.ensure(hs), "rs_map") &&
              cuda_ok(q_.ensure(qs), "rs_map") && cuda_ok(dst.ensure(nn * 4), "rs_map") &&
              cuda_ok(res_.ensure(64), "rs_map");
    if (!ok) return false;
    const Mat3 hi = inv3_plain(Hc);
    float hif[9];
    for (int i = 0; i < 9; ++i) hif[i] = (float)hi[i];
    const bool okdet = std::fabs(det3(Hc)) >= 1e-12;
    double* n00 = reinterpret_cast<double*>(res_.as<char>() + 16);
    if (!cuda_ok(warp_stack(A.stack.as<float>(), A.w, A.h, hif, okdet, fr.w, fr.h, canvas_a_.as<float>(), st), "rs_map") ||
        !cuda_ok(paste_stack(B.stack.as<float>(), B.w, B.h, fr.ox, fr.oy, fr.w, fr.h, canvas_b_.as<float>(), st),
                 "rs_map") ||
        !cuda_ok(rs_logpolar(canvas_a_.as<float>(), fr.w, fr.h, (float)p.cx, (float)p.cy, (float)p.log0, (float)p.span,
                             p.n_th, p.n_lam, grid_a_.as<float>(), st),
                 "rs_map") ||
        !cuda_ok(rs_logpolar(canvas_b_.as<float>(), fr.w, fr.h, (float)p.cx, (float)p.cy, (float)p.log0, (float)p.span,
                             p.n_th, p.n_lam, grid_b_.as<float>(), st),
                 "rs_map") ||
        !cuda_ok(lag0_count(grid_a_.as<float>(), grid_b_.as<float>(), p.n_th, p.n_lam, n00, st), "rs_map"))
        return false;
    CombineParams cp{};
    cp.exact = exact ? 1 : 0;
    cp.calib = exact && calibrated ? 1 : 0;
    cp.nf = side[0].mode == 1 ? 3 : 4;
    cp.min_n = 12.0f;
    cp.area = std::max(1.0, pair_area());  // the correlation area in pixels (area scale 1)
    cp.ridge = 1e-4;
    cp.inv_nn = 1.0 / ((double)g.nx * (double)g.ny);
    cp.lp_dlam = p.dlam;
    cp.lp_dth = p.dth;
    if (!cuda_ok(forward_rows(grid_a_.as<float>(), g, plan, row, half_a_.as<float2>(), st), "rs_map") ||
        !cuda_ok(forward_rows(grid_b_.as<float>(), g, plan, row, half_b_.as<float2>(), st), "rs_map") ||
        !cuda_ok(forward_cols(half_a_.as<float2>(), g, plan, col, st), "rs_map") ||
        !cuda_ok(forward_cols(half_b_.as<float2>(), g, plan, col, st), "rs_map") ||
        !cuda_ok(inverse_columns(half_a_.as<float2>(), half_b_.as<float2>(), g, plan, col, q_.as<float2>(), st),
                 "rs_map") ||
        !cuda_ok(inverse_rows_score(q_.as<float2>(), g, plan, line, S, tw, cp, n00, dst.as<float>(), nullptr, nullptr,
                                    st),
                 "rs_map"))
        return false;
    counts[0] += 11;
    return true;
}

void Engine::rs_center(const Mat3& H, double c[2]) const {
    const double lw = side[0].w, lh = side[0].h;
    const double q[4][2] = {{1, 1}, {lw, 1}, {lw, lh}, {1, lh}};
    c[0] = c[1] = 0;
    for (const auto& v : q) {
        const auto m = map_pt(H, v[0], v[1]);
        c[0] += 0.25 * m[0], c[1] += 0.25 * m[1];
    }
}

bool Engine::rs_peak(const Mat3& H, const double c[2], double* dth, double* dsg) {
    RsPlan p;
    if (!rs_map_one(H, c, -1, 0, set.b("exact"), set.b("calibrated"), set.u("map_res"), rs_fwd_, p)) return false;
    const bool mirror = H[0] * H[4] - H[1] * H[3] > 0;
    const double smin = set.f("rs_smin"), smax = set.f("rs_smax");
    const double lo = std::log(std::max(smin > 0 ? smin : 0.2, 1e-6));
    const double hi = std::log(std::max(smax > 0 ? smax : 5.0, 1.000001));
    const size_t nn = (size_t)p.n * p.n;
    char* res = res_.as<char>();
    unsigned long long key = 0;
    if (!cuda_ok(rs_map_.ensure(nn * 4), "rs_map") ||
        !cuda_ok(rs_finish(rs_fwd_.as<float>(), nullptr, mirror, p.n, (float)p.dlam, (float)lo, (float)hi,
                           rs_map_.as<float>(), reinterpret_cast<unsigned long long*>(res),
                           reinterpret_cast<float*>(res + 8), st),
                 "rs_map") ||
        !cuda_ok(cudaMemcpyAsync(&key, res, 8, cudaMemcpyDeviceToHost, st), "rs_map") ||
        !cuda_ok(cudaStreamSynchronize(st), "rs_map"))
        return false;
    counts[0] += 1, counts[1]++, counts[2]++, counts[3]++;
    *dth = *dsg = 0;
    const uint32_t idx = 0xffffffffu - (uint32_t)(key & 0xffffffffu);
    if (key != 0 && idx < nn) {
        const int64_t py = idx / p.n, px = idx % p.n;
        const int64_t lx = px <= p.n / 2 ? px : px - p.n, ly = py <= p.n / 2 ? py : py - p.n;
        *dth = -((double)lx / (double)std::max(p.n_th, 1)) * 2 * M_PI;
        *dsg = -(double)ly * p.dlam;
    }
    return true;
}

bool Engine::rs_map(const Mat3& H, const double* c_opt, bool symmetric, zc_rs_result* out, float* map, float* fwd,
                    float* inv, size_t len) {
    if (!need_images()) return false;
    if (!metric_ok("rs_map")) return false;
    const bool exact = set.b("exact"), calibrated = set.b("calibrated");
    const unsigned cap = set.u("map_res");
    // the centre: given, else the moving image's centroid under H (src/lie.zig movingCentroid)
    double c[2];
    if (c_opt) {
        c[0] = c_opt[0], c[1] = c_opt[1];
    } else {
        rs_center(H, c);
    }
    RsPlan p, pi;
    if (!rs_map_one(H, c, -1, 0, exact, calibrated, cap, rs_fwd_, p)) return false;
    if (symmetric) {
        const Mat3 Hi = inv3(H);
        const auto ci = map_pt(Hi, c[0], c[1]);
        const double cc[2] = {ci[0], ci[1]};
        SideSwap sw(side[0], side[1]);
        if (!rs_map_one(Hi, cc, p.r0, p.r1, exact, calibrated, cap, rs_inv_, pi)) return false;
        if (pi.n != p.n) return fail("rs_map: GridMismatch");
    }
    const size_t nn = (size_t)p.n * p.n;
    if ((map || fwd || inv) && len < nn) return fail("rs_map: MapTooSmall");
    const bool mirror = H[0] * H[4] - H[1] * H[3] > 0;
    const double smin = set.f("rs_smin"), smax = set.f("rs_smax");
    const double lo = std::log(std::max(smin > 0 ? smin : 0.2, 1e-6));
    const double hi = std::log(std::max(smax > 0 ? smax : 5.0, 1.000001));
    if (!cuda_ok(rs_map_.ensure(nn * 4), "rs_map")) return false;
    char* res = res_.as<char>();
    unsigned long long* best = reinterpret_cast<unsigned long long*>(res);
    float* zero = reinterpret_cast<float*>(res + 8);
    if (!cuda_ok(rs_finish(rs_fwd_.as<float>(), symmetric ? rs_inv_.as<float>() : nullptr, mirror, p.n, (float)p.dlam,
                           (float)lo, (float)hi, rs_map_.as<float>(), best, zero, st),
                 "rs_map"))
        return false;
    unsigned char host[16];
    bool ok = cuda_ok(cudaMemcpyAsync(host, res, 16, cudaMemcpyDeviceToHost, st), "rs_map");
    if (ok && map) ok = cuda_ok(cudaMemcpyAsync(map, rs_map_.p, nn * 4, cudaMemcpyDeviceToHost, st), "rs_map");
    if (ok && fwd) ok = cuda_ok(cudaMemcpyAsync(fwd, rs_fwd_.p, nn * 4, cudaMemcpyDeviceToHost, st), "rs_map");
    if (ok && inv && symmetric) ok = cuda_ok(cudaMemcpyAsync(inv, rs_inv_.p, nn * 4, cudaMemcpyDeviceToHost, st), "rs_map");
    if (!ok || !cuda_ok(cudaStreamSynchronize(st), "rs_map")) return false;
    counts[0] += 1;
    counts[1]++;
    counts[2] += 1 + (map ? 1 : 0) + (fwd ? 1 : 0) + (inv && symmetric ? 1 : 0);
    counts[3]++;
    unsigned long long key;
    float z;
    std::memcpy(&key, host, 8);
    std::memcpy(&z, host + 8, 4);
    zc_rs_result r{};
    r.n = (uint32_t)p.n;
    r.n_th = (uint32_t)p.n_th;
    r.n_lam = (uint32_t)p.n_lam;
    r.dlam = p.dlam;
    r.r0 = p.r0;
    r.r1 = p.r1;
    r.cx = c[0];
    r.cy = c[1];
    r.peak = key_float((uint32_t)(key >> 32));
    r.zero = z;
    r.symmetric = symmetric ? 1 : 0;
    r.calibrated = exact && calibrated ? 1 : 0;
    const uint32_t idx = 0xffffffffu - (uint32_t)(key & 0xffffffffu);
    if (key != 0 && idx < nn) {
        const int64_t py = idx / p.n, px = idx % p.n;
        const int64_t lx = px <= p.n / 2 ? px : px - p.n;
        const int64_t ly = py <= p.n / 2 ? py : py - p.n;
        r.peak_index = idx;
        r.dth = -((double)lx / (double)std::max(p.n_th, 1)) * 2 * M_PI;
        r.dsg = -(double)ly * p.dlam;
    }
    *out = r;
    return true;
}

}  // namespace zc
