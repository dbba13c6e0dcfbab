// Pose scores, gradients and the Gauss–Newton refine of the B200 engine.
// Restated from the reference's src/pair.zig (parts 162-184, sym 241-268, gradBoth 281-302,
// beats 51-53), src/pose.zig (gradFrom 267-289) and the climb's decision rules
// (src/gclimb.zig:314-489, shaders/climb.wgsl gn_cands 229-292, hop_cand 320-338,
// climb_select 415-459, iter_end 849-857), with the decisions on the host in float64.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>

#include "engine.hpp"
#include "lie.hpp"

namespace zc {

namespace {

constexpr int kMom = 45, kCoef = 102, kGrad = 44;

std::string fmt_mat(const Mat3& H) {
    std::string s = "[";
    for (int i = 0; i < 9; ++i) {
        char b[32];
        snprintf(b, sizeof b, "%s%.17g", i ? "," : "", H[i]);
        s += b;
    }
    return s + "]";
}

std::string json_num(double v) {
    if (!std::isfinite(v)) return "null";
    char b[32];
    snprintf(b, sizeof b, "%.17g", v);
    return b;
}

std::string json_str(const std::string& t) {
    std::string o = "\"";
    for (char c : t) {
        if (c == '"' || c == '\\') o += '\\', o += c;
        else if (c == '\n') o += "\\n";
        else o += c;
    }
    return o + "\"";
}

}  // namespace

void Engine::log_event(const std::string& text) { events.push_back("{\"kind\":\"log\",\"text\":" + json_str(text) + "}"); }

// scratch for n poses per launch onto either side: the pose kernels then add each pose's
// block totals in block order (the same sums on every run, in any batch); fresh tickets are zeroed
bool Engine::pose_red(int n, PoseRed& r) {
    const size_t px = std::max((size_t)side[0].w * side[0].h, (size_t)side[1].w * side[1].h);
    const uint64_t gen = pose_ticket_.gen;
    if (!cuda_ok(pose_part_.ensure(pose_red_need(px, n) * sizeof(double)), "pose sums") ||
        !cuda_ok(pose_ticket_.ensure((size_t)std::max(n, 1) * sizeof(unsigned)), "pose sums"))
        return false;
    if (pose_ticket_.gen != gen && !cuda_ok(cudaMemsetAsync(pose_ticket_.p, 0, pose_ticket_.cap, st), "pose sums"))
        return false;
    r = PoseRed{pose_part_.as<double>(), pose_ticket_.as<unsigned>(), pose_part_.cap / sizeof(double),
                pose_ticket_.cap / sizeof(unsigned)};
    return true;
}

bool Engine::eval_poses(const std::vector<Mat3>& Hs, bool grad, bool hess, std::vector<PoseEval>& out,
                        bool forward_only, const float* pose_cps) {
    if (!need_images()) return false;
    if (!metric_ok("score")) return false;
    const bool sym = set.b("symmetric") && !forward_only, homog = set.e("group") == "homography", exact = set.b("exact");
    const int n = (int)Hs.size(), nd = sym ? 2 : 1, nk = n_keys(homog);
    if (n == 0) return true;
    const size_t m = (size_t)nd * n;
    bool ok = cuda_ok(pose_hinv_.ensure(m * 9 * 4), "score") && cuda_ok(pose_sums_.ensure(m * kMom * 8), "score") &&
              cuda_ok(pose_coef_.ensure(m * kCoef * 4), "score") && cuda_ok(pose_score_.ensure(m * 8), "score") &&
              cuda_ok(pose_tsum_.ensure(m * kGrad * 8), "score") && cuda_ok(pose_gens_.ensure(2 * 72 * 4), "score");
    if (!ok) return false;
    // inverse poses: forward direction H⁻¹; inverse direction (pose H⁻¹) its inverse; written to
    // page-locked memory, as the sums come back into it, so neither copy is staged
    const size_t n_in = m * 9 + 2 * 72, n_out = m * kMom + m + (grad ? m * kGrad : 0);
    if (!cuda_ok(pose_in_pin_.ensure(n_in * sizeof(float)), "score") ||
        !cuda_ok(pose_out_pin_.ensure(n_out * sizeof(double)), "score"))
        return false;
    float* pose_host = pose_in_pin_.as<float>();
    std::fill(pose_host, pose_host + n_in, 0.f);
    for (int i = 0; i < n; ++i) {
        const Mat3 Hi = inv3(Hs[i]);
        for (int k = 0; k < 9; ++k) pose_host[(size_t)i * 9 + k] = (float)Hi[k];
        if (sym) {
            const Mat3 Hii = inv3(Hi);
            for (int k = 0; k < 9; ++k) pose_host[((size_t)n + i) * 9 + k] = (float)Hii[k];
        }
    }
    const Side &A = side[0], &B = side[1];
    // generators in the destination's pixels: the fixed image forward, the moving one inverse
    const auto gf = generators(homog, B.w, B.h), gi = generators(homog, A.w, A.h);
    float* gens = pose_host + m * 9;
    for (int k = 0; k < 8; ++k)
        for (int e = 0; e < 9; ++e) {
            gens[k * 9 + e] = (float)gf[k][e];
            gens[72 + k * 9 + e] = (float)gi[k][e];
        }
    float* dh = pose_hinv_.as<float>();
    float* dg = pose_gens_.as<float>();
    if (!cuda_ok(cudaMemcpyAsync(dh, pose_host, m * 9 * 4, cudaMemcpyHostToDevice, st), "score") ||
        !cuda_ok(cudaMemcpyAsync(dg, gens, 2 * 72 * 4, cudaMemcpyHostToDevice, st), "score"))
        return false;
    const PoseSide pa{A.feat.as<float>(), A.feat4.as<float4>(), A.w, A.h},
        pb{B.feat.as<float>(), B.feat4.as<float4>(), B.w, B.h};
    double* sums = pose_sums_.as<double>();
    double* tsum = pose_tsum_.as<double>();
    float* coef = pose_coef_.as<float>();
    // a live spline moves the samples of both directions (src/pair.zig:127-150)
    PoseFfd ff, fi;
    if (!(pose_cps ? ffd_pose_dirs(pose_cps, n, ff, fi) : ffd_dirs(ff, fi))) return false;
    PoseRed rd;
    if (!pose_red(n, rd)) return false;
    if (!cuda_ok(pose_moments(pa, pb, dh, n, sums, st, ff, nullptr, rd), "moments")) return false;
    if (sym &&
        !cuda_ok(pose_moments(pb, pa, dh + (size_t)n * 9, n, sums + (size_t)n * kMom, st, fi, nullptr, rd), "moments"))
        return false;
    if (!cuda_ok(pose_coefs(sums, (int)m, exact, coef, pose_score_.as<double>(), st), "score")) return false;
    counts[0] += nd + 1;
    if (grad) {
        if (!cuda_ok(pose_tangent(pa, pb, dh, coef, dg, n, hess, tsum, st, ff, nullptr, rd), "gradient")) return false;
        if (sym && !cuda_ok(pose_tangent(pb, pa, dh + (size_t)n * 9, coef + (size_t)n * kCoef, dg + 72, n, hess,
                                         tsum + (size_t)n * kGrad, st, fi, nullptr, rd),
                            "gradient"))
            return false;
        counts[0] += nd;
    }
    double* hs = pose_out_pin_.as<double>();
    double* hsc = hs + m * kMom;
    double* ht = hsc + m;
    if (!cuda_ok(cudaMemcpyAsync(hs, sums, m * kMom * 8, cudaMemcpyDeviceToHost, st), "score") ||
        !cuda_ok(cudaMemcpyAsync(hsc, pose_score_.p, m * 8, cudaMemcpyDeviceToHost, st), "score"))
        return false;
    if (grad && !cuda_ok(cudaMemcpyAsync(ht, tsum, m * kGrad * 8, cudaMemcpyDeviceToHost, st), "score")) return false;
    if (!cuda_ok(cudaStreamSynchronize(st), "score")) return false;
    counts[1]++;
    counts[2] += grad ? 3 : 2;
    counts[3]++;
    out.assign(n, PoseEval{});
    auto fin = [](double v) { return std::isfinite(v) ? v : 0.0; };
    // one direction's gradient and Gauss–Newton matrix (pose.zig gradFrom)
    auto unpack = [&](size_t row, double nsum, Coords& g, std::array<double, 64>& A) {
        g = Coords{};
        A.fill(0.0);
        if (!(nsum >= 12.0)) return;
        const double* t = ht + row * kGrad;
        for (int q = 0; q < nk; ++q) g[q] = t[q];
        int h = 8;
        for (int q = 0; q < 8; ++q)
            for (int mm = q; mm < 8; ++mm, ++h)
                if (q < nk && mm < nk) A[q * nk + mm] = A[mm * nk + q] = t[h];
    };
    for (int i = 0; i < n; ++i) {
        PoseEval& r = out[i];
        for (int k = 0; k < kMom; ++k) r.sums[k] = hs[(size_t)i * kMom + k];
        r.n = r.sums[0];
        r.fwd = fin(hsc[i]);
        r.has_inv = sym;
        r.inv = sym ? fin(hsc[(size_t)n + i]) : 0.0;
        r.mean = sym ? 0.5 * (r.fwd + r.inv) : r.fwd;
        if (!grad) continue;
        Coords gfw, gbk;
        std::array<double, 64> Af, Ab;
        unpack(i, r.n, gfw, Af);
        r.has_grad = true;
        r.has_hess = hess;
        if (!sym) {
            r.grad = gfw;
            r.hess = Af;
            continue;
        }
        unpack((size_t)n + i, hs[((size_t)n + i) * kMom], gbk, Ab);
        // g = ½ (g_fwd + Pᵀ g_inv), A = ½ (A_fwd + Pᵀ A_inv P) (pair.zig sym)
        const Coords pulled = adjoint_grad(gbk.data(), Hs[i], homog, A.w, A.h, B.w, B.h);
        for (int q = 0; q < nk; ++q) r.grad[q] = 0.5 * (gfw[q] + pulled[q]);
        if (hess) {
            double PT[64] = {0};
            for (int j = 0; j < nk; ++j) {
                double e[8] = {0};
                e[j] = 1;
                const Coords col = adjoint_grad(e, Hs[i], homog, A.w, A.h, B.w, B.h);
                for (int q = 0; q < nk; ++q) PT[q * nk + j] = col[q];
            }
            for (int p = 0; p < nk; ++p)
                for (int q = 0; q < nk; ++q) {
                    double s = 0;
                    for (int x = 0; x < nk; ++x)
                        for (int y = 0; y < nk; ++y) s += PT[p * nk + x] * Ab[x * nk + y] * PT[q * nk + y];
                    r.hess[p * nk + q] = 0.5 * (Af[p * nk + q] + s);
                }
        }
    }
    return true;
}

bool Engine::moments(const Mat3& Hm, double* out45) {
    // the forward direction only (src/exports.zig:276-281)
    std::vector<PoseEval> r;
    if (!eval_poses({Hm}, false, false, r, true)) return false;
    for (int k = 0; k < kMom; ++k) out45[k] = r[0].sums[k];
    return true;
}

bool Engine::score3(const Mat3& Hm, double* out3) {
    if (!metric_ok("score")) return false;
    if (set.e("metric") == "ncc") {
        // the NCC metric's score is one-sided (src/engine.zig:752-758): mean = forward, no inverse
        double s;
        if (!ncc_score(Hm, &s)) return false;
        out3[0] = out3[1] = s;
        out3[2] = std::nan("");
        return true;
    }
    std::vector<PoseEval> r;
    if (!eval_poses({Hm}, false, false, r)) return false;
    out3[0] = r[0].mean;
    out3[1] = r[0].fwd;
    out3[2] = r[0].has_inv ? r[0].inv : std::nan("");
    return true;
}

bool Engine::gradient(const Mat3& Hm, bool hess, zc_grad_result* out) {
    std::vector<PoseEval> r;
    if (!eval_poses({Hm}, true, hess, r)) return false;
    const bool homog = set.e("group") == "homography";
    const int nk = n_keys(homog);
    zc_grad_result g{};
    g.score = r[0].mean;
    g.fwd = r[0].fwd;
    g.inv = r[0].has_inv ? r[0].inv : std::nan("");
    g.n = r[0].n;
    for (int q = 0; q < nk; ++q) g.grad[q] = r[0].grad[q];
    if (hess) {
        for (int q = 0; q < nk * nk; ++q) g.hess[q] = r[0].hess[q];
        g.has_hess = 1;
    }
    g.nk = (uint32_t)nk;
    *out = g;
    return true;
}

// ── the refine ────────────────────────────────────────────────────────────────────────────────

bool Engine::climb(zc_climb_result* out) {
    if (!need_images()) return false;
    const bool sym = set.b("symmetric"), homog = set.e("group") == "homography", hop = set.b("hop");
    const bool hop_fm = set.b("hop_fm"), hops = hop || hop_fm, spline = set.b("ffd");
    double lam = -1;  // the spline's bending weight, set at its first step
    const unsigned n_iters = std::max(1u, set.u("g_iters"));
    const int nk = n_keys(homog);
    const double rw = side[1].w, rh = side[1].h;
    // a candidate beats the current score when higher by more than 1e-6 of it (pair.zig beats)
    auto beats = [](double nw, double old) { return nw > old + std::max(1e-6 * std::fabs(old), 1e-12); };
    std::vector<PoseEval> ev;
    Mat3 H = this->H;
    if (!eval_poses({H}, true, true, ev)) return false;
    PoseEval cur = ev[0];
    const double s_start = cur.mean;
    char buf[256];
    snprintf(buf, sizeof buf, "ascent %s score %.4f %s%s%sGauss–Newton%s (B200)", homog ? "homography" : "affine",
             s_start, sym ? "mean " : "", hop ? "shift hop+" : "", hop_fm ? "roto-scale hop+" : "",
             spline ? "+spline" : "");
    log_event(buf);
    cancel = false;
    unsigned iter = 0, stall = 0, n_rec = 0;
    double c[2] = {0, 0};
    // one stage: candidates and the current pose scored together; the best that beats the
    // current pose's fresh score becomes the pose, with its gradient (climb_select)
    auto stage = [&](const std::vector<Mat3>& cands, const char* label, const std::vector<double>& mus, bool& moved) {
        std::vector<Mat3> all = cands;
        all.push_back(H);
        std::vector<PoseEval> sc;
        if (!eval_poses(all, false, false, sc)) return false;
        const double c0 = sc.back().mean;
        int best = -1;
        double best_s = c0;
        for (size_t i = 0; i < cands.size(); ++i) {
            const double s = sc[i].mean;
            if (beats(s, c0) && (best < 0 || s > best_s)) {
                best = (int)i;
                best_s = s;
            }
        }
        moved = best >= 0;
        if (!moved) {
            cur.mean = c0;
            cur.fwd = sc.back().fwd;
            cur.inv = sc.back().inv;
            return true;
        }
        H = cands[best];
        std::vector<PoseEval> g;
        if (!eval_poses({H}, true, true, g)) return false;
        cur = g[0];
        ++n_rec;
        std::string lab = label;
        if (!mus.empty()) {
            snprintf(buf, sizeof buf, "%s ×%g", label, mus[best]);
            lab = buf;
        }
        events.push_back("{\"kind\":\"trail\",\"label\":" + json_str(lab) + ",\"score\":" + json_num(cur.mean) +
                         ",\"fwd\":" + json_num(cur.fwd) + ",\"inv\":" + (sym ? json_num(cur.inv) : "null") +
                         ",\"H\":" + fmt_mat(H) + ",\"cps\":null}");
        return true;
    };
    while (true) {
        bool moved_any = false;
        if (hop) {
            // shift hop: the map's peak as a translation of the pose (hop_cand)
            zc_shift_result r;
            if (!shift_map(H, set.b("exact"), set.b("calibrated"), set.u("map_res"), set.f("min_overlap"), &r, nullptr, 0))
                return false;
            bool moved = false;
            if (!stage({mul3(translate(-r.dx, -r.dy), H)}, "shift hop", {}, moved)) return false;
            moved_any |= moved;
        }
        // up to three Gauss–Newton steps; one that beats nothing ends the block (gn_cands)
        auto gn_block = [&]() {
        for (int step = 0; step < 3; ++step) {
            double A[64], b[8], x[8] = {0};
            for (int i = 0; i < nk; ++i) {
                for (int j = 0; j < nk; ++j) A[i * nk + j] = cur.hess[i * nk + j];
                A[i * nk + i] += 1e-4 * std::max(A[i * nk + i], 1e-12);
                b[i] = 0.5 * cur.grad[i];
            }
            if (!solve_linear(A, b, nk, x)) break;
            double sn = 0;
            for (int i = 0; i < nk; ++i) sn += x[i] * x[i];
            sn = std::sqrt(sn);
            std::vector<Mat3> cands;
            const std::vector<double> mus = {0.5, 1.0, 2.0, 4.0, 8.0};
            for (double mu : mus) {
                const double nrm = sn * mu;
                const double sc = mu * (nrm > 0.25 ? 0.25 / nrm : 1.0);
                Coords xi{};
                for (int i = 0; i < nk; ++i) xi[i] = sc * x[i];
                cands.push_back(composeN(H, xi, homog, rw, rh));
            }
            bool moved = false;
            if (!stage(cands, "GN", mus, moved)) return false;
            moved_any |= moved;
            if (!moved) break;
        }
        return true;
        };
        // the Gauss–Newton block follows the shift hop, and the roto-scale hop when it runs alone
        if ((hop || !hop_fm) && !gn_block()) return false;
        if (hop_fm) {
            // roto-scale hop (rs_cand): the one-sided roto-scale map's peak about the moving
            // image's centroid as a rotation and scale of the pose, then a fresh GN block; the
            // centre is the one of the pose that each batch of 8 iterations starts from
            if (iter % 8 == 0) rs_center(H, c);
            double dth = 0, dsg = 0;
            if (!rs_peak(H, c, &dth, &dsg)) return false;
            if (!(std::fabs(dth) < 2e-4 && std::fabs(dsg) < 2e-4)) {
                const double sc = std::exp(dsg), a = sc * std::cos(dth), b = -sc * std::sin(dth);
                const double d = sc * std::sin(dth), e = sc * std::cos(dth);
                const Mat3 S = {a, b, c[0] - a * c[0] - b * c[1], d, e, c[1] - d * c[0] - e * c[1], 0, 0, 1};
                bool moved = false;
                if (!stage({project_group(mul3(S, H), homog)}, "roto-scale hop", {}, moved)) return false;
                moved_any |= moved;
            }
            if (!gn_block()) return false;
        }
        if (spline) {
            // the spline stage (src/gclimb.zig:206-246): a Gauss–Newton step of the control
            // points under the bending penalty; a win moves the spline, then the current pose's
            // gradient is taken again with it
            bool moved = false;
            double sc_now = 0;
            if (!spline_stage(H, lam, moved, sc_now)) return false;
            if (moved) {
                std::vector<PoseEval> g;
                if (!eval_poses({H}, true, true, g)) return false;
                cur = g[0];
                ++n_rec;
                std::string cj = "[";
                const unsigned gg = ffd_grid();
                for (size_t i = 0; i < 2 * (size_t)gg * gg; ++i) cj += (i ? "," : "") + json_num(ffd_cps_[i]);
                events.push_back("{\"kind\":\"trail\",\"label\":\"spline\",\"score\":" + json_num(cur.mean) +
                                 ",\"fwd\":" + json_num(cur.fwd) + ",\"inv\":" + (sym ? json_num(cur.inv) : "null") +
                                 ",\"H\":" + fmt_mat(H) + ",\"cps\":" + cj + "]}");
            } else {
                cur.mean = sc_now;
            }
            moved_any |= moved;
        }
        // iter_end: a move resets the stall count; with the shift hop on, two iterations in a
        // row without a move end the climb (one without it), as does the iteration budget
        stall = moved_any ? 0 : stall + 1;
        ++iter;
        std::string pj = "null";
        if (spline) {
            pj = "[";
            const unsigned gg = ffd_grid();
            for (size_t i = 0; i < 2 * (size_t)gg * gg; ++i) pj += (i ? "," : "") + json_num(ffd_cps_[i]);
            pj += "]";
        }
        events.push_back("{\"kind\":\"pose\",\"H\":" + fmt_mat(H) + ",\"cps\":" + pj + "}");
        snprintf(buf, sizeof buf, "ascent %u/%u score %.4f  stall %u  (%u steps so far)", iter, n_iters, cur.mean, stall,
                 n_rec);
        log_event(buf);
        if ((!moved_any && (!hops || stall >= 2)) || iter >= n_iters) break;
        if (cancel) {
            snprintf(buf, sizeof buf, "ascent stopped  score %.4f", cur.mean);
            log_event(buf);
            break;
        }
    }
    this->H = H;
    snprintf(buf, sizeof buf, "ascent done  score %.4f", cur.mean);
    log_event(buf);
    zc_climb_result r{};
    for (int i = 0; i < 9; ++i) r.H[i] = H[i];
    r.score = cur.mean;
    r.iterations = iter;
    r.moved = (n_rec > 0 && cur.mean > s_start) ? 1 : 0;
    *out = r;
    return true;
}

}  // namespace zc
