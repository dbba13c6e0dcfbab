// The zc_* C ABI of the B200 engine (the reference's src/exports.zig and src/native_api.zig):
// every name the reference's ctypes loader binds (python/zcmir/_native.py:79-133), with the same
// argument meanings, struct layouts, return values and error reporting (0 / -1 and zc_error).
// Calls outside this build's SMI path return their failure value with a message saying so.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

#include "../../include/zcmir_b200.h"
#include "engine.hpp"

struct zc_engine : zc::Engine {
    using zc::Engine::Engine;
};

static_assert(sizeof(zc_shift_result) == 88, "ShiftResult layout");
static_assert(sizeof(zc_rs_result) == 96, "RsResult layout");
static_assert(sizeof(zc_grad_result) == 616, "GradResult layout");
static_assert(sizeof(zc_climb_result) == 88, "ClimbResult layout");
static_assert(sizeof(zc_detect_result) == 16, "DetectResult layout");
static_assert(sizeof(zc_match_result) == 112, "MatchResult layout");
static_assert(sizeof(zc_search_result) == 104, "SearchResult layout");
static_assert(sizeof(zc_canvas_info) == 88, "Canvas layout");

namespace {

char g_create_err[512];
size_t g_create_err_len = 0;

size_t copy_out(const std::string& s, char* buf, size_t cap) {
    const size_t n = std::min(s.size(), cap);
    if (buf && n) memcpy(buf, s.data(), n);
    return n;
}

zc::Mat3 mat(const double* H) {
    zc::Mat3 m;
    for (int i = 0; i < 9; ++i) m[i] = H[i];
    return m;
}

int32_t unsupported(zc_engine* e, const char* what) {
    if (e) e->fail(std::string(what) + ": not part of this build (the B200 SMI path: maps, scores, refine, sweep)");
    return -1;
}

template <class F>
int32_t guarded(zc_engine* e, const char* what, F&& f) {
    if (!e) return -1;
    e->err.clear();
    try {
        return f() ? 0 : -1;
    } catch (const std::exception& x) {
        e->fail(std::string(what) + ": " + x.what());
        return -1;
    }
}

}  // namespace

extern "C" {

const char* zc_version(void) { return "0.1.4"; }

zc_engine* zc_create(const char* /*wgpu_path: the reference's WebGPU library, unused here*/) {
    g_create_err_len = 0;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        const std::string m = std::string("GPU init failed: no CUDA device (") + cudaGetErrorString(e) + ")";
        g_create_err_len = copy_out(m, g_create_err, sizeof g_create_err);
        return nullptr;
    }
    int dev = 0;
    cudaGetDevice(&dev);
    try {
        zc_engine* eng = new zc_engine(dev);
        // the no-allocation pose scores' device array: looked up (its module loaded) here, once
        // per device, so that zcb_score_static itself reserves nothing
        zc::static_scratch_setup(dev);
        return eng;
    } catch (const std::exception& x) {
        const std::string m = std::string("engine init failed: ") + x.what();
        g_create_err_len = copy_out(m, g_create_err, sizeof g_create_err);
        return nullptr;
    }
}

size_t zc_create_error(char* buf, size_t cap) {
    const size_t n = std::min(g_create_err_len, cap);
    if (n) memcpy(buf, g_create_err, n);
    return n;
}

void zc_destroy(zc_engine* e) { delete e; }

size_t zc_adapter(zc_engine* e, char* buf, size_t cap) {
    if (!e) return 0;
    char s[256];
    snprintf(s, sizeof s, "%s (CUDA, sm_%d%d, %d SMs, %.0f GB)", e->prop.name, e->prop.major, e->prop.minor,
             e->prop.multiProcessorCount, (double)e->prop.totalGlobalMem / 1e9);
    return copy_out(s, buf, cap);
}

size_t zc_error(zc_engine* e, char* buf, size_t cap) {
    if (!e) return 0;
    const size_t n = copy_out(e->err, buf, cap);
    e->err.clear();
    return n;
}

int32_t zc_configure(zc_engine* e, const char* json, size_t len) {
    return guarded(e, "configure", [&] {
        std::string m;
        if (!e->set.apply(json, len, m)) return e->fail(m);
        return true;
    });
}

size_t zc_settings(zc_engine* e, char* buf, size_t cap) {
    if (!e) return 0;
    const std::string j = e->set.to_json();
    copy_out(j, buf, cap);
    return j.size();
}

int32_t zc_set_image_gray(zc_engine* e, uint32_t side, const float* data, uint32_t w, uint32_t h,
                          uint32_t preprocess) {
    return guarded(e, "set_image_gray", [&] { return e->set_image((int)side, data, (int)w, (int)h, preprocess != 0); });
}

int32_t zc_set_image(zc_engine* e, uint32_t side, const float* data, uint32_t w, uint32_t h) {
    return zc_set_image_gray(e, side, data, w, h, 0);
}

int32_t zc_set_image_rgba(zc_engine* e, uint32_t side, const uint8_t* data, uint32_t w, uint32_t h) {
    return guarded(e, "set_image_rgba", [&] { return e->set_image_rgba((int)side, data, (int)w, (int)h); });
}

int32_t zc_work_image(zc_engine* e, uint32_t side, float* out, size_t len) {
    return guarded(e, "work_image", [&] { return e->work_image((int)side, out, len); });
}

int32_t zc_features(zc_engine* e, uint32_t side, float* out, size_t len) {
    return guarded(e, "features", [&] { return e->features((int)side, out, len); });
}

void zc_image_size(zc_engine* e, uint32_t side, uint32_t out[2]) {
    if (!e || side > 1 || !e->side[side].has) {
        out[0] = out[1] = 0;
        return;
    }
    out[0] = (uint32_t)e->side[side].w;
    out[1] = (uint32_t)e->side[side].h;
}

void zc_swap(zc_engine* e) {
    if (e) std::swap(e->side[0], e->side[1]);
}

int32_t zc_moments(zc_engine* e, const double H[9], double out[45]) {
    return guarded(e, "moments", [&] { return e->moments(mat(H), out); });
}

int32_t zc_score(zc_engine* e, const double H[9], double out[3]) {
    return guarded(e, "score", [&] { return e->score3(mat(H), out); });
}

int32_t zc_gradient(zc_engine* e, const double H[9], uint32_t hess, zc_grad_result* out) {
    return guarded(e, "gradient", [&] { return e->gradient(mat(H), hess != 0, out); });
}

int32_t zc_shift_map(zc_engine* e, const double H[9], uint32_t flags, uint32_t cap, zc_shift_result* out, float* map,
                     size_t map_len) {
    // explicit flags (1 exact, 2 calibrated), no overlap floor; cap 0 = the 1024 default
    // (src/engine.zig:822-829)
    return guarded(e, "shift_map", [&] {
        return e->shift_map(mat(H), (flags & 1) != 0, (flags & 2) != 0, cap == 0 ? zc::kMapCap : cap, 0.0, out, map,
                            map_len);
    });
}

int32_t zc_shift_map_set(zc_engine* e, const double H[9], zc_shift_result* out, float* map, size_t map_len) {
    return guarded(e, "shift_map", [&] { return e->shift_map_settings(mat(H), out, map, map_len); });
}

int32_t zc_rs_map(zc_engine* e, const double H[9], const double* c, uint32_t symmetric, zc_rs_result* out, float* map,
                  float* fwd, float* inv, size_t len) {
    return guarded(e, "rs_map", [&] { return e->rs_map(mat(H), c, symmetric != 0, out, map, fwd, inv, len); });
}

void zc_set_pose(zc_engine* e, const double H[9]) {
    if (e) e->H = mat(H);
}

void zc_get_pose(zc_engine* e, double H[9]) {
    if (e)
        for (int i = 0; i < 9; ++i) H[i] = e->H[i];
}

int32_t zc_climb(zc_engine* e, zc_climb_result* out) {
    return guarded(e, "climb", [&] { return e->climb(out); });
}
int32_t zc_search(zc_engine* e, zc_search_result* out) {
    return guarded(e, "search", [&] { return e->search(out); });
}

void zc_cancel(zc_engine* e) {
    if (e) e->cancel = true;
}

size_t zc_events(zc_engine* e, char* buf, size_t cap) {
    if (!e) return 0;
    size_t n = 0;
    while (!e->events.empty()) {
        const std::string& l = e->events.front();
        if (n + l.size() + 1 > cap) break;
        memcpy(buf + n, l.data(), l.size());
        n += l.size();
        buf[n++] = '\n';
        e->events.pop_front();
    }
    return n;
}

int32_t zc_profile(zc_engine* e, uint32_t on) {
    if (!e) return 0;
    e->profiling = on != 0;
    return 1;
}

size_t zc_profile_report(zc_engine* e, char* buf, size_t cap) {
    if (!e) return 0;
    std::vector<std::pair<std::string, std::pair<double, uint32_t>>> v(e->prof.begin(), e->prof.end());
    std::sort(v.begin(), v.end(), [](const auto& a, const auto& b) { return a.second.first > b.second.first; });
    std::string s;
    for (auto& kv : v) {
        char line[160];
        snprintf(line, sizeof line, "%9.3f ms %6u  %s\n", kv.second.first, kv.second.second, kv.first.c_str());
        s += line;
    }
    e->prof.clear();
    return copy_out(s, buf, cap);
}

void zc_gpu_counts(zc_engine* e, uint32_t out[4]) {
    if (!e) return;
    for (int i = 0; i < 4; ++i) {
        out[i] = e->counts[i];
        e->counts[i] = 0;
    }
}

int32_t zc_bench_moments(zc_engine* e, uint32_t n_poses, uint32_t iters) {
    // `iters` score passes over n_poses poses spread about the current pose (src/exports.zig:123-136)
    return guarded(e, "bench_moments", [&] {
        std::vector<zc::Mat3> Hs(std::max(1u, n_poses));
        for (size_t i = 0; i < Hs.size(); ++i) {
            const double t = (double)i * 0.37, a = 0.01 * std::sin(t);
            Hs[i] = zc::mul3({std::cos(a), -std::sin(a), 3 * std::cos(t), std::sin(a), std::cos(a), 3 * std::sin(t), 0, 0, 1},
                             e->H);
        }
        std::vector<zc::PoseEval> r;
        for (uint32_t k = 0; k < std::max(1u, iters); ++k)
            if (!e->eval_poses(Hs, false, false, r, true)) return false;
        return true;
    });
}

// The reference's knobs of its per-pixel sum kernels (src/exports.zig:115-121) mapped onto this
// build's pose kernels: pixels per thread, the least blocks per pose (fill_wg), the most blocks
// per pose (tg_cap); tg_px (the reference's pixels per tile group) has no counterpart, since a
// warp here always takes an 8 × 4 tile. 0 keeps a knob's value.
void zc_tune_parts(uint32_t px_per_thread, uint32_t fill_wg, uint32_t /*tg_px*/, uint32_t tg_cap) {
    zc::pose_tune(px_per_thread, fill_wg, tg_cap);
}

int32_t zc_compile_wgsl(zc_engine*, const char*, size_t, const char*, size_t, char*, size_t) {
    return -1;  // "unsupported here" (python/zcmir/__init__.py:315-325)
}

int32_t zc_pg_info(zc_engine* e, double*) { return unsupported(e, "pg_info"); }
int32_t zc_pg_maps(zc_engine* e, uint32_t, float*, size_t) { return unsupported(e, "pg_maps"); }
int32_t zc_pg_descriptors(zc_engine* e, uint32_t, float*, size_t) { return unsupported(e, "pg_descriptors"); }
int32_t zc_match_scores(zc_engine* e, float*, size_t) { return unsupported(e, "match_scores"); }
// Keypoints are outside this build's SMI path. So that callers which start a registration from
// keypoints (the reference's register() without a start pose, register_stack's first pair and its
// re-detections) run unchanged, zc_detect finds no keypoints and succeeds, and zc_match takes its
// fit from the SMI sweep search instead of a keypoint fit (Engine::match_by_sweep). The keypoint
// and match listings below stay refused.
int32_t zc_detect(zc_engine* e, zc_detect_result* out) {
    return guarded(e, "detect", [&] {
        if (!e->need_images()) return false;
        if (out) *out = zc_detect_result{};
        e->log_event("detect  no keypoint detector in this build: 0 keypoints (zc_match fits by the SMI sweep)");
        return true;
    });
}
int32_t zc_match(zc_engine* e, zc_match_result* out) {
    return guarded(e, "match", [&] {
        zc_match_result r{};
        if (!e->match_by_sweep(&r)) return false;
        if (out) *out = r;
        return true;
    });
}
int32_t zc_auto(zc_engine* e, zc_climb_result*) { return unsupported(e, "auto"); }
int32_t zc_keypoints(zc_engine* e, uint32_t, float*, size_t) { return unsupported(e, "keypoints"); }
int32_t zc_keypoint_frames(zc_engine* e, uint32_t, float*, size_t) { return unsupported(e, "keypoint_frames"); }
int32_t zc_matches(zc_engine* e, uint32_t*, size_t) { return unsupported(e, "matches"); }

int32_t zc_set_ffd(zc_engine* e, const float* cps, size_t n) {
    return guarded(e, "set_ffd", [&] { return e->set_ffd(cps, n); });
}

size_t zc_get_ffd(zc_engine* e, float* cps, size_t cap) {
    if (!e) return 0;
    return e->get_ffd(cps, cap);
}

uint32_t zc_fit_check(zc_engine* e, const double*) {
    if (e) e->fail("fit_check: not part of this build");
    return 7;  // "it fails the sanity check" (python/zcmir/__init__.py:178-181)
}

int32_t zc_ffd_gradient(zc_engine* e, const double* H, double* score, double* grad, size_t len) {
    return guarded(e, "ffd_gradient", [&] { return e->ffd_gradient(mat(H), score, grad, len); });
}

int32_t zc_canvas(zc_engine* e, const double H[9], uint32_t inverse, zc_canvas_info* out) {
    // src/overlay.zig:122-128 (host arithmetic only)
    return guarded(e, "canvas", [&] {
        if (!e->side[0].has || !e->side[1].has) return e->fail("canvas: NoImages");
        const zc::Side& a = e->side[inverse ? 1 : 0];
        const zc::Side& b = e->side[inverse ? 0 : 1];
        const zc::Mat3 Hp = inverse ? zc::inv3(mat(H)) : mat(H);
        const zc::Frame fr = zc::reg_frame(Hp, a.w, a.h, b.w, b.h);
        const zc::Mat3 Hc = zc::canvas_H(Hp, fr.ox, fr.oy);
        out->ox = fr.ox;
        out->oy = fr.oy;
        out->ow = (uint32_t)fr.w;
        out->oh = (uint32_t)fr.h;
        for (int i = 0; i < 9; ++i) out->Hc[i] = Hc[i];
        return true;
    });
}

int32_t zc_overlay(zc_engine* e, const double*, uint32_t, zc_canvas_info*, float*, float*, size_t) {
    return unsupported(e, "overlay");
}
int32_t zc_tile_heat(zc_engine* e, const double*, uint32_t, uint32_t, double*, float*, float*, size_t) {
    return unsupported(e, "tile_heat");
}
int64_t zc_export_warp(zc_engine* e, const char*, size_t, void*, size_t) { return unsupported(e, "export_warp"); }
int32_t zc_displacement(zc_engine* e, float* out, size_t len) {
    return guarded(e, "displacement", [&] { return e->displacement(out, len); });
}

void zc_result_sizes(uint32_t out[4]) {
    out[0] = sizeof(zc_shift_result);
    out[1] = sizeof(zc_rs_result);
    out[2] = sizeof(zc_grad_result);
    out[3] = 0;
}

// ── the B200 build's own entry points (include/zcmir_b200.h) ──

int32_t zcb_bench_maps(zc_engine* e, const double H[9], uint32_t flags, uint32_t cap, uint32_t warmup, uint32_t steps,
                       double* out, size_t out_len) {
    return guarded(e, "bench_maps", [&] { return e->bench_maps(mat(H), flags, cap, warmup, steps, out, out_len); });
}

int32_t zcb_settings_apply(const char* json, size_t len, char* out, size_t cap, size_t* out_len, char* err,
                           size_t err_cap, size_t* err_len) {
    zc::Settings st;
    std::string m;
    if (!st.apply(json, len, m)) {
        if (err_len) *err_len = copy_out(m, err, err_cap);
        return -1;
    }
    const std::string j = st.to_json();
    copy_out(j, out, cap);
    if (out_len) *out_len = j.size();
    if (err_len) *err_len = 0;
    return 0;
}

int32_t zcb_refine_poses(zc_engine* e, const double* Hs, uint32_t n, uint32_t iters, double* Hout, double* scores) {
    return guarded(e, "refine_poses", [&] {
        if (n > 0 && (!Hs || !Hout || !scores)) return e->fail("refine_poses: null poses or outputs");
        if (!e->search_check()) return false;
        std::vector<zc::Mat3> in(n);
        for (uint32_t i = 0; i < n; ++i) in[i] = mat(Hs + 9 * (size_t)i);
        const std::vector<double> amps = zc::geo_amps(e->set.f("g_a0"), e->set.f("g_decay"),
                                                      e->set.u("g_steps") > 0 ? e->set.u("g_steps") : 7);
        std::vector<zc::ScoredPose> out;
        if (!e->gn_batch(in, iters, amps, out)) return false;
        for (uint32_t i = 0; i < n; ++i) {
            std::memcpy(Hout + 9 * (size_t)i, out[i].H.data(), 9 * sizeof(double));
            scores[i] = out[i].score;
        }
        return true;
    });
}

int32_t zcb_search_lanes(zc_engine* e, const float* scores, const uint32_t* idx, size_t n, zc_search_result* out) {
    return guarded(e, "search_lanes", [&] { return e->search_lanes(scores, idx, n, out); });
}

int32_t zcb_sweep(zc_engine* e, const double H0p[9], uint32_t n_peak, uint32_t batch, uint32_t shard, uint32_t nshard,
                  float* scores, uint32_t* idx, size_t cap, double* info, size_t info_len) {
    return guarded(e, "sweep", [&] {
        if (info_len < 16 || !info) return e->fail("sweep: info needs 16 entries");
        zc::SweepGrid gv;
        int G;
        zc::Mat3 Hd;
        e->sweep_settings(gv, G, Hd);
        const zc::Mat3 H0 = H0p ? mat(H0p) : Hd;
        const double min_ov = std::min(0.5, std::max(0.0, e->set.f("min_overlap")));
        zc::SweepOut r;
        if (!e->sweep_maps(H0, gv, G, e->set.b("exact"), (int)n_peak, min_ov, r, (int)batch, (int)shard,
                           (int)std::max(nshard, 1u)))
            return false;
        const size_t n = r.lane_score.size();
        if (scores && idx) {
            if (cap < n) return e->fail("sweep: BufferTooSmall");
            std::copy(r.lane_score.begin(), r.lane_score.end(), scores);
            std::copy(r.lane_idx.begin(), r.lane_idx.end(), idx);
        }
        const double v[16] = {(double)r.cands.size(), r.cell, (double)r.ms, (double)r.G, (double)r.Fx, (double)r.Fy,
                              (double)r.fx0, (double)r.fy0, (double)r.min_n, (double)r.n, (double)r.groups,
                              (double)r.batches, (double)r.launches, r.ox, r.oy, (double)r.peaks.size()};
        std::copy(v, v + 16, info);
        return true;
    });
}

int32_t zcb_stack_maps(zc_engine* e, uint32_t n, const float* const* images, const uint32_t* w, const uint32_t* h,
                       const double* priors, uint32_t flags, uint32_t cap, zc_shift_result* out, double* ms) {
    return guarded(e, "stack_maps", [&] {
        std::vector<int> ws(n), hs(n);
        for (uint32_t i = 0; i < n; ++i) ws[i] = (int)w[i], hs[i] = (int)h[i];
        std::vector<zc::Mat3> pr;
        if (priors)
            for (uint32_t k = 0; k + 1 < n; ++k) pr.push_back(mat(priors + 9 * k));
        float t = 0;
        if (!e->stack_maps((int)n, images, ws.data(), hs.data(), priors ? pr.data() : nullptr, (flags & 1) != 0,
                           (flags & 2) != 0, cap, out, &t))
            return false;
        if (ms) *ms = t;
        return true;
    });
}

int32_t zcb_stack_load(zc_engine* e, uint32_t n, const float* const* images, const uint32_t* w, const uint32_t* h,
                       const double* priors, uint32_t flags, uint32_t cap) {
    return guarded(e, "stack_load", [&] {
        if (n > 0 && (!w || !h)) return e->fail("stack_load: null sizes");
        std::vector<int> ws(n), hs(n);
        for (uint32_t i = 0; i < n; ++i) ws[i] = (int)w[i], hs[i] = (int)h[i];
        std::vector<zc::Mat3> pr;
        if (priors)
            for (uint32_t k = 0; k + 1 < n; ++k) pr.push_back(mat(priors + 9 * k));
        return e->stack_load((int)n, images, ws.data(), hs.data(), priors ? pr.data() : nullptr, (flags & 1) != 0,
                             (flags & 2) != 0, cap);
    });
}

int32_t zcb_sweep_stack(zc_engine* e, const double H0p[9], uint32_t n_peak, float* scores, uint32_t* idx, size_t cap,
                        double* info, size_t info_len, zc_shift_result* stack_out, size_t n_out) {
    return guarded(e, "sweep_stack", [&] {
        if (info_len < 16 || !info) return e->fail("sweep_stack: info needs 16 entries");
        zc::SweepGrid gv;
        int G;
        zc::Mat3 Hd;
        e->sweep_settings(gv, G, Hd);
        zc::SweepOut r;
        if (!e->sweep_stack(H0p ? mat(H0p) : Hd, (int)n_peak, r, stack_out, n_out)) return false;
        const size_t n = r.lane_score.size();
        if (scores && idx) {
            if (cap < n) return e->fail("sweep_stack: BufferTooSmall");
            std::copy(r.lane_score.begin(), r.lane_score.end(), scores);
            std::copy(r.lane_idx.begin(), r.lane_idx.end(), idx);
        }
        const double v[16] = {(double)r.cands.size(), r.cell, (double)r.ms, (double)r.G, (double)r.Fx, (double)r.Fy,
                              (double)r.fx0, (double)r.fy0, (double)r.min_n, (double)r.n, (double)r.groups,
                              (double)r.batches, (double)r.launches, r.ox, r.oy, (double)r.peaks.size()};
        std::copy(v, v + 16, info);
        return true;
    });
}

int32_t zcb_tune_sweep(zc_engine* e, double* out, size_t cap, size_t* used) {
    return guarded(e, "tune_sweep", [&] { return e->tune_sweep(out, cap, used); });
}

int32_t zcb_set_dft_stage(zc_engine* e, uint32_t pieces) {
    return guarded(e, "set_dft_stage", [&] { return e->set_dft_stage(pieces); });
}

int32_t zcb_score_static(zc_engine* e, const double* Hs, uint32_t n, double* out) {
    // allocates no device memory: the scratch is a file-scope array (score_static.cu)
    return guarded(e, "score_static", [&] { return e->score_static(Hs, n, out); });
}

}  // extern "C"
