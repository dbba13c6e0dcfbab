// The NCC overlay metric (the reference's src/overlay.zig:209-305, nccShiftMap and nccScore,
// reached through Engine.score and Engine.shiftMapSettings, src/engine.zig:752-766, when the
// settings' metric is "ncc"): the pair's union canvas at the pose, its zero-lag normalised
// cross-correlation as the pose score, and the NCC of every shift as a map on the shift map's
// FFT passes (one mean-free plane per side, one correlation).
#include <algorithm>
#include <cmath>
#include <cstring>

#include "engine.hpp"

namespace zc {

namespace {

// the NCC map's longest FFT line: min(maxFftN, 1024) in src/overlay.zig:217
constexpr unsigned kNccMaxN = 1024;

struct NccCanvas {
    Frame fr;
    float hi[9];
    bool ok;
};

NccCanvas ncc_canvas_of(const Mat3& H, const Side& A, const Side& B) {
    NccCanvas c;
    c.fr = reg_frame(H, A.w, A.h, B.w, B.h);
    const Mat3 Hc = canvas_H(H, c.fr.ox, c.fr.oy);
    const Mat3 hi = inv3_plain(Hc);
    for (int i = 0; i < 9; ++i) c.hi[i] = (float)hi[i];
    c.ok = std::fabs(det3(Hc)) >= 1e-12;
    return c;
}

}  // namespace

bool Engine::metric_ok(const char* what) {
    const std::string m = set.e("metric");
    if (m == "smi" || m == "ncc") return true;
    return fail(std::string(what) + ": metric \"" + m + "\" is not part of this build (metric=\"smi\" or \"ncc\")");
}

bool Engine::ncc_score(const Mat3& H, double* out) {
    if (!need_images()) return false;
    const Side &A = side[0], &B = side[1];
    const NccCanvas c = ncc_canvas_of(H, A, B);
    if (!cuda_ok(res_.ensure(128), "score")) return false;
    double* mom = reinterpret_cast<double*>(res_.as<char>() + 64);
    double s[5];
    if (!cuda_ok(ncc_moments(A.work.as<float>(), A.w, A.h, c.hi, c.ok, B.work.as<float>(), B.w, B.h, c.fr.ox, c.fr.oy,
                             A.half, c.fr.w, c.fr.h, mom, st),
                 "score") ||
        !cuda_ok(cudaMemcpyAsync(s, mom, sizeof s, cudaMemcpyDeviceToHost, st), "score") ||
        !cuda_ok(cudaStreamSynchronize(st), "score"))
        return false;
    counts[0] += 1, counts[1]++, counts[2]++, counts[3]++;
    // src/overlay.zig:299-304: Pearson's r over every canvas pixel, clamped to ±1.5
    const double nf = (double)c.fr.w * c.fr.h;
    const double cov = s[4] - s[0] * s[1] / nf;
    const double va = std::max(s[2] - s[0] * s[0] / nf, 0.0), vb = std::max(s[3] - s[1] * s[1] / nf, 0.0);
    *out = std::min(1.5, std::max(-1.5, cov / std::sqrt(std::max(va * vb, 1e-24))));
    return true;
}

bool Engine::ncc_shift_map(const Mat3& H, zc_shift_result* out, float* map, size_t map_len) {
    if (!need_images()) return false;
    const bool ladder = set.e("fft_sizes") == "ladder";
    if (!ladder) return fail("shift_map: fft_sizes=\"compact\" is not supported by this build (use \"ladder\")");
    const Side &A = side[0], &B = side[1];
    const NccCanvas c = ncc_canvas_of(H, A, B);
    const MapPlan mp = linear_corr_plan(c.fr.w, c.fr.h, kNccMaxN, ladder);
    MapJob job;
    job.fr = c.fr;
    MapGeom& g = job.g;
    g.W = c.fr.w, g.Hh = c.fr.h, g.ox = c.fr.ox, g.oy = c.fr.oy;
    g.cw = mp.cw, g.ch = mp.ch, g.nx = mp.nx, g.ny = mp.ny;
    g.WP = ((g.nx / 2 + 1) + 7) / 8 * 8;
    const size_t nn = (size_t)g.nx * g.ny;
    if (map && map_len < nn) return fail("shift_map: MapTooSmall");
    // one real plane per side (plane 0 of its grid) and their one correlation
    CorrPlanDev plan{};
    plan.n_real = 1;
    plan.n_corr = 1;
    LinePlan row, col, line;
    if (!line_plan(g.nx, row) || !line_plan(g.ny, col)) return false;
    const int S = row_split(g.nx, plan.n_corr);
    if (S == 0) return fail("shift_map: a row of " + std::to_string(g.nx) + " does not fit the row pass");
    if (!line_plan(g.nx / S, line)) return false;
    const float2* tw = twiddles(g.nx);
    if (!tw) return fail("shift_map: twiddles: out of device memory");
    const size_t cn = (size_t)g.W * g.Hh, gn = (size_t)g.cw * g.ch;
    const size_t hs = (size_t)g.ny * g.WP * sizeof(float2);
    forget_spectra();  // this map writes the map path's canvas and spectrum buffers
    bool ok = cuda_ok(canvas_a_.ensure(cn * 4), "shift_map") && cuda_ok(canvas_b_.ensure(cn * 4), "shift_map") &&
              cuda_ok(grid_a_.ensure(gn * 20), "shift_map") && cuda_ok(grid_b_.ensure(gn * 20), "shift_map") &&
              cuda_ok(half_a_.ensure(hs), "shift_map") && cuda_ok(half_b_.ensure(hs), "shift_map") &&
              cuda_ok(q_.ensure(hs), "shift_map") && cuda_ok(map_.ensure(nn * 4), "shift_map") &&
              cuda_ok(res_.ensure(128), "shift_map");
    if (!ok) return false;
    char* res = res_.as<char>();
    unsigned long long* best = reinterpret_cast<unsigned long long*>(res);
    float* zero = reinterpret_cast<float*>(res + 8);
    double* den = reinterpret_cast<double*>(res + 16);
    double* sums = reinterpret_cast<double*>(res + 32);
    CombineParams cp{};
    cp.nf = 1;
    cp.inv_nn = 1.0 / ((double)g.nx * (double)g.ny);
    if (!cuda_ok(ncc_canvas(A.work.as<float>(), A.w, A.h, c.hi, c.ok, B.work.as<float>(), B.w, B.h, g.ox, g.oy, A.half,
                            g.W, g.Hh, canvas_a_.as<float>(), canvas_b_.as<float>(), st),
                 "shift_map") ||
        !cuda_ok(ncc_grid(canvas_a_.as<float>(), canvas_b_.as<float>(), g.W, g.Hh, g.cw, g.ch, grid_a_.as<float>(),
                          grid_b_.as<float>(), sums, den, st),
                 "shift_map") ||
        !cuda_ok(cudaMemsetAsync(best, 0, 8, st), "shift_map") ||
        !cuda_ok(forward_rows(grid_a_.as<float>(), g, plan, row, half_a_.as<float2>(), st), "shift_map") ||
        !cuda_ok(forward_rows(grid_b_.as<float>(), g, plan, row, half_b_.as<float2>(), st), "shift_map") ||
        !cuda_ok(forward_cols(half_a_.as<float2>(), g, plan, col, st), "shift_map") ||
        !cuda_ok(forward_cols(half_b_.as<float2>(), g, plan, col, st), "shift_map") ||
        !cuda_ok(inverse_columns(half_a_.as<float2>(), half_b_.as<float2>(), g, plan, col, q_.as<float2>(), st),
                 "shift_map") ||
        !cuda_ok(inverse_rows_score(q_.as<float2>(), g, plan, line, S, tw, cp, den, map_.as<float>(), best, zero, st),
                 "shift_map"))
        return false;
    unsigned char host[16];
    ok = cuda_ok(cudaMemcpyAsync(host, res, 16, cudaMemcpyDeviceToHost, st), "shift_map");
    if (ok && map) ok = cuda_ok(cudaMemcpyAsync(map, map_.p, nn * 4, cudaMemcpyDeviceToHost, st), "shift_map");
    if (!ok || !cuda_ok(cudaStreamSynchronize(st), "shift_map")) return false;
    counts[0] += 11;
    counts[1]++;
    counts[2] += map ? 2 : 1;
    counts[3]++;
    unsigned long long key;
    float z;
    std::memcpy(&key, host, 8);
    std::memcpy(&z, host + 8, 4);
    // the NCC result carries no correlation area and neither whitening flag (src/overlay.zig:266-272)
    job.exact = false;
    job.calibrated = false;
    map_result(job, key, z, 0.0, out);
    return true;
}

}  // namespace zc
