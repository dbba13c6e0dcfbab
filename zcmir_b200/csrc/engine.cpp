// The B200 SMI engine: images, features and the shift-map schedule.
// Host schedule restated from the reference's src/engine.zig (setImageGray 430-434, bake 322-341,
// shiftMapOpts 795-819, shiftMap 822-829) and src/smi.zig (prepare 348-400, shiftMapFrom 552-572).
#include "engine.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

namespace zc {

const char* const kStageNames[kNumStages] = {"canvas", "fwd_rows", "fwd_cols", "inv_cols", "inv_rows_score"};

cudaError_t DevBuf::ensure(size_t bytes) {
    if (bytes <= cap && p) return cudaSuccess;
    release();
    const size_t want = std::max<size_t>(bytes, 256);
    cudaError_t e = cudaMalloc(&p, want);
    if (e != cudaSuccess) {
        p = nullptr;
        cap = 0;
        return e;
    }
    cap = want;
    ++gen;
    return cudaSuccess;
}

void DevBuf::release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
}

// The correlation plan (src/smi.zig:90-158): the real planes kept (15 exact, 5 global; without
// the fourth feature's planes when `three`) and, per correlation slot, its moving and fixed
// plane slots and its number in the full 45-correlation order.
CorrPlanDev corr_plan_dev(bool exact, bool three) {
    int lst_a[45], lst_b[45], nl = 0;
    lst_a[nl] = 0, lst_b[nl++] = 0;
    for (int i = 0; i < 4; ++i) lst_a[nl] = 1 + i, lst_b[nl++] = 0;
    for (int j = 0; j < 4; ++j) lst_a[nl] = 0, lst_b[nl++] = 1 + j;
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) lst_a[nl] = 1 + i, lst_b[nl++] = 1 + j;
    if (exact) {
        for (int k = 0; k < 10; ++k) lst_a[nl] = 5 + k, lst_b[nl++] = 0;
        for (int k = 0; k < 10; ++k) lst_a[nl] = 0, lst_b[nl++] = 5 + k;
    }
    const int n_planes = exact ? 15 : 5;
    int slot[15];
    CorrPlanDev P{};
    for (int pl = 0; pl < n_planes; ++pl) {
        const bool fourth = pl == 4 || pl == 8 || pl == 11 || pl == 13 || pl == 14;
        if (three && fourth) {
            slot[pl] = -1;
            continue;
        }
        slot[pl] = P.n_real;
        P.planes[P.n_real++] = pl;
    }
    for (int c = 0; c < nl; ++c) {
        const int sa = slot[lst_a[c]], sb = slot[lst_b[c]];
        if (sa < 0 || sb < 0) continue;
        P.ca[P.n_corr] = sa;
        P.cb[P.n_corr] = sb;
        P.cnum[P.n_corr] = c;
        P.n_corr++;
    }
    return P;
}

Engine::Engine(int dev) : device(dev) {
    if (const char* v = getenv("ZCMIR_B200_ROW_PASS")) row_pass = v;
    if (const char* v = getenv("ZCMIR_B200_SPECTRA_CACHE")) spectra_cache_ = atoi(v) != 0;
    cudaSetDevice(dev);
    cudaGetDeviceProperties(&prop, dev);
    // priorities: side 1's feature build (st2_) highest, so it is not starved by side 0's passes
    // queued beside it; the engine stream next; the autocorrelation's stream lowest, its blocks
    // fill what the others leave (a lower number is a higher priority)
    cudaDeviceGetStreamPriorityRange(&prio_lo_, &prio_hi_);
    cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, std::min(prio_hi_ + 1, prio_lo_));
}

Engine::~Engine() {
    cudaStreamSynchronize(st);
    if (sweep_exec_) cudaGraphExecDestroy(sweep_exec_);
    for (auto& s : side) {
        s.raw.release();
        s.work.release();
        s.feat.release();
        s.feat4.release();
        s.mag.release();
        s.stack.release();
        s.acf_dev.release();
        if (s.built_ev) cudaEventDestroy(s.built_ev);
        if (s.acf_ev) cudaEventDestroy(s.acf_ev);
        if (s.acf_host) cudaFreeHost(s.acf_host);
    }
    if (up_ev_) cudaEventDestroy(up_ev_);
    for (DevBuf* b : {&fs2_stats_, &fs2_hist_, &fs2_wt_, &fs2_acfpart_, &rank_tmp2_}) b->release();
    if (st2_) {
        cudaStreamSynchronize(st2_);
        cudaStreamDestroy(st2_);
    }
    if (acf_st_) {
        cudaStreamSynchronize(acf_st_);
        cudaStreamDestroy(acf_st_);
    }
    for (DevBuf* b : {&fs_stats_, &fs_hist_, &fs_wt_, &fs_acfpart_, &fs_acf_, &rank_tmp_, &canvas_a_, &canvas_b_,
                      &grid_a_, &grid_b_, &half_a_, &half_b_, &q_, &map_, &res_, &flush_, &pose_hinv_, &pose_sums_,
                      &pose_coef_, &pose_score_, &pose_tsum_, &pose_gens_, &pose_part_, &pose_ticket_, &dft_scratch_, &sw_il_[0], &sw_il_[1], &sw_poses_,
                      &sw_fgrid_, &sw_fhalf_, &sw_grid_, &sw_half_, &sw_q_, &sw_map_, &sw_n0_, &sw_ps_, &sw_pi_})
        b->release();
    for (auto& s : stack_) {
        for (DevBuf* b : {&s.raw, &s.work, &s.feat, &s.feat4, &s.mag, &s.stack, &s.acf_dev}) b->release();
        if (s.built_ev) cudaEventDestroy(s.built_ev);
        if (s.acf_ev) cudaEventDestroy(s.acf_ev);
        if (s.acf_host) cudaFreeHost(s.acf_host);
    }
    stack_res_.release();
    for (DevBuf* b : {&rs_fwd_, &rs_inv_, &rs_map_, &pp_rgba_, &pp_clahe_, &pp_tmp_, &pp_mm_, &ffd_dev_, &ffd_out_,
                      &ffd_pk_, &ffd_cells_, &ffd_coef_})
        b->release();
    pose_in_pin_.release();
    pose_out_pin_.release();
    gn_pin_.release();
    for (DevBuf* b : {&gn_H_, &gn_Htry_, &gn_valid_, &gn_active_, &gn_cur_}) b->release();
    for (auto& kv : tw_) cudaFree(kv.second);
    for (cudaEvent_t e : chunk_ev_)
        if (e) cudaEventDestroy(e);
    if (copy_st_) cudaStreamDestroy(copy_st_);
    if (branch_st_) cudaStreamDestroy(branch_st_);
    for (cudaEvent_t e : {fork_ev_, join_ev_})
        if (e) cudaEventDestroy(e);
    cudaStreamDestroy(st);
}

bool Engine::fail(const std::string& m) {
    if (err.empty()) err = m;
    return false;
}

bool Engine::cuda_ok(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return true;
    return fail(std::string(what) + ": CUDA error: " + cudaGetErrorString(e));
}

// ── images and features ──────────────────────────────────────────────────────────────────────

bool Engine::set_image(int s, const float* data, int w, int h, bool preprocess) {
    // the reference's setImageGray checks (src/engine.zig:430-434)
    if (s < 0 || s > 1 || w < 8 || h < 8 || !data) return fail("set_image_gray: BadImage");
    Side& sd = side[s];
    const size_t n = (size_t)w * h;
    if (!cuda_ok(sd.raw.ensure(n * 4), "set_image_gray")) return false;
    // the upload on the copy stream, so it runs beside the other side's feature build; it waits
    // for this side's previous build (the only reader of `raw`), the build waits for it
    if (!copy_st_ && !cuda_ok(cudaStreamCreateWithFlags(&copy_st_, cudaStreamNonBlocking), "set_image_gray")) return false;
    if (!up_ev_ && !cuda_ok(cudaEventCreateWithFlags(&up_ev_, cudaEventDisableTiming), "set_image_gray")) return false;
    if ((sd.built_ev && !cuda_ok(cudaStreamWaitEvent(copy_st_, sd.built_ev, 0), "set_image_gray")) ||
        !cuda_ok(cudaMemcpyAsync(sd.raw.p, data, n * 4, cudaMemcpyHostToDevice, copy_st_), "set_image_gray") ||
        !cuda_ok(cudaEventRecord(up_ev_, copy_st_), "set_image_gray"))
        return false;
    sd.has = true;
    sd.preprocess = preprocess;
    cudaStream_t bs = st;
    if (!build_stream(s, bs) || !cuda_ok(cudaStreamWaitEvent(bs, up_ev_, 0), "set_image_gray")) return false;
    sd.has = true;
    sd.w = w;
    sd.h = h;
    sd.preprocess = preprocess;
    sd.built = false;
    return build_side(s);
}

bool Engine::set_image_rgba(int s, const unsigned char* rgba, int w, int h) {
    if (s < 0 || s > 1 || w < 8 || h < 8 || !rgba) return fail("set_image_rgba: BadImage");
    Side& sd = side[s];
    const size_t n = (size_t)w * h;
    if (!cuda_ok(pp_rgba_.ensure(n * 4), "set_image_rgba") || !cuda_ok(sd.raw.ensure(n * 4), "set_image_rgba") ||
        !cuda_ok(cudaMemcpyAsync(pp_rgba_.p, rgba, n * 4, cudaMemcpyHostToDevice, st), "set_image_rgba") ||
        !cuda_ok(rgba_to_gray(pp_rgba_.as<unsigned char>(), (int)n, sd.raw.as<float>(), st), "set_image_rgba"))
        return false;
    counts[0] += 1;
    sd.has = true;
    sd.w = w;
    sd.h = h;
    sd.preprocess = true;
    sd.built = false;
    return build_side(s);
}

std::string Engine::bake_key() const {
    char b[160];
    snprintf(b, sizeof b, "%d %u %u %d %.17g %.17g %d %d", set.b("clahe"), set.u("clahe_grid"), set.u("clahe_bins"),
             set.b("band"), set.f("bp_fine"), set.f("bp_coarse"), set.b("invert"), set.b("half"));
    return b;
}

bool Engine::bake(int s, cudaStream_t bs) {
    Side& sd = side[s];
    const int n = sd.w * sd.h;
    const bool half = set.b("half");
    float* work = sd.work.as<float>();
    sd.bake = sd.preprocess ? bake_key() : std::string();
    if (!sd.preprocess) return cuda_ok(cudaMemcpyAsync(work, sd.raw.p, (size_t)n * 4, cudaMemcpyDeviceToDevice, bs), "features");
    // CLAHE (clip limit 40, the settings' grid and bins) from the f32 image, else its texels
    if (set.b("clahe")) {
        if (!cuda_ok(pp_clahe_.ensure(clahe_scratch_bytes((int)set.u("clahe_grid"), (int)set.u("clahe_bins"))), "clahe") ||
            !cuda_ok(clahe(sd.raw.as<float>(), sd.w, sd.h, 40.0, (int)set.u("clahe_bins"), (int)set.u("clahe_grid"), half,
                           pp_clahe_.p, work, st),
                     "clahe"))
            return false;
        counts[0] += 3;
    } else {
        if (!cuda_ok(cudaMemcpyAsync(work, sd.raw.p, (size_t)n * 4, cudaMemcpyDeviceToDevice, st), "features")) return false;
        if (half && !cuda_ok(round_texels(work, n, st), "features")) return false;
    }
    if (set.b("band")) {
        // difference of Gaussians: fine = blur^f, coarse = blur^(c − f) of fine (src/gls.zig:531-557)
        const double fp = set.f("bp_fine") > 0 ? set.f("bp_fine") : 1.0;
        const double cp = set.f("bp_coarse") > 0 ? set.f("bp_coarse") : 6.0;
        const int fine_n = (int)std::max(1.0, std::min(16.0, std::round(fp * fp)));
        const int coarse_n = std::max(fine_n + 1, (int)std::min(64.0, std::round(cp * cp)));
        if (!cuda_ok(pp_tmp_.ensure((size_t)n * 4 * 5), "band") || !cuda_ok(pp_mm_.ensure(8), "band")) return false;
        float* t = pp_tmp_.as<float>();
        float *mid = t, *ping = t + n, *fine = t + 2 * (size_t)n, *coarse = t + 3 * (size_t)n, *d = t + 4 * (size_t)n;
        auto passes = [&](const float* src, float* dst, int k) {
            const float* from = src;
            for (int i = 0; i < k; ++i) {
                float* to = (i == k - 1) ? dst : ping;
                if (to == from) to = (from == ping) ? d : ping;
                if (!cuda_ok(gauss_blur(from, sd.w, sd.h, half, mid, to, st), "band")) return false;
                counts[0] += 2;
                from = to;
            }
            if (from != dst) return cuda_ok(cudaMemcpyAsync(dst, from, (size_t)n * 4, cudaMemcpyDeviceToDevice, st), "band");
            return true;
        };
        if (!passes(work, fine, fine_n) || !passes(fine, coarse, coarse_n - fine_n) ||
            !cuda_ok(dog_rescale(fine, coarse, n, half, d, pp_mm_.as<unsigned>(), work, st), "band"))
            return false;
        counts[0] += 2;
    }
    if (set.b("invert")) {
        if (!cuda_ok(invert_texels(work, n, half, st), "invert")) return false;
        counts[0] += 1;
    }
    return true;
}

// The stream a side's features build on: side 1 without preprocessing on a stream of its own
// with its own scratch, so its build runs beside side 0's (the preprocessing scratch is shared,
// so preprocessed sides build in order on the engine stream). Safe because every call that reads
// a side's buffers waits for its work before returning: when a build starts, the only pending
// work is other builds.
bool Engine::build_stream(int s, cudaStream_t& bs) {
    bs = st;
    if (s != 1 || side[s].preprocess) return true;
    if (!st2_ && !cuda_ok(cudaStreamCreateWithPriority(&st2_, cudaStreamNonBlocking, prio_hi_), "features")) return false;
    bs = st2_;
    return true;
}

bool Engine::build_side(int s) {
    Side& sd = side[s];
    sd.ver = ++build_counter_;
    const size_t n = (size_t)sd.w * sd.h;
    cudaStream_t bs = st;
    if (!build_stream(s, bs)) return false;
    const bool own = bs != st;
    DevBuf &stats = own ? fs2_stats_ : fs_stats_, &hist = own ? fs2_hist_ : fs_hist_, &wt = own ? fs2_wt_ : fs_wt_;
    DevBuf &part = own ? fs2_acfpart_ : fs_acfpart_, &rtmp = own ? rank_tmp2_ : rank_tmp_;
    FeatScratch& fsc = own ? fs2_ : fs_;
    const std::string& fm = set.e("smi_features");
    const int mode = fm == "laplacian" ? 0 : (fm == "three" ? 1 : 2);
    const bool half = set.b("half");
    const int ntiles = ((sd.w + 31) / 32) * ((sd.h + 31) / 32);
    bool ok = cuda_ok(sd.work.ensure(n * 4), "features") && cuda_ok(sd.feat.ensure(n * 16), "features") &&
              cuda_ok(sd.feat4.ensure(n * 16), "features") &&
              cuda_ok(sd.mag.ensure(n * 4), "features") && cuda_ok(sd.stack.ensure(n * 20), "features") &&
              cuda_ok(rtmp.ensure(n * 4), "features") && cuda_ok(stats.ensure(22 * 8), "features") &&
              cuda_ok(hist.ensure(256 * 4), "features") && cuda_ok(wt.ensure(20 * 4), "features") &&
              cuda_ok(part.ensure((size_t)ntiles * 1156 * 4), "features") &&
              cuda_ok(sd.acf_dev.ensure(1156 * 8), "features");
    if (!ok) return false;
    fsc.stats = stats.as<double>();
    fsc.hist = hist.as<unsigned>();
    fsc.wt = wt.as<float>();
    fsc.acf_part = part.as<float>();
    fsc.acf_part_cap = part.cap / 4;
    fsc.acf = sd.acf_dev.as<double>();
    // the side's previous autocorrelation (on acf_st_) reads the features this build rewrites
    if (sd.acf_ev && !cuda_ok(cudaStreamWaitEvent(bs, sd.acf_ev, 0), "features")) return false;
    if (!bake(s, bs)) return false;
    if (!cuda_ok(build_features(sd.work.as<float>(), sd.w, sd.h, mode, half, rtmp.as<float>(), sd.feat.as<float>(),
                                sd.mag.as<float>(), sd.stack.as<float>(), fsc, bs),
                 "features") ||
        !cuda_ok(interleave_features(sd.feat.as<float>(), (int)n, sd.feat4.as<float4>(), bs), "features"))
        return false;
    counts[0] += 12;
    if (!sd.built_ev && !cuda_ok(cudaEventCreateWithFlags(&sd.built_ev, cudaEventDisableTiming), "features")) return false;
    if (!cuda_ok(cudaEventRecord(sd.built_ev, bs), "features")) return false;
    // the autocorrelation (only the calibrated score's correlation area needs it) runs on a
    // stream of its own at low priority, beside the passes that use the features, and its sums
    // go back to the host there; finish_acf waits for that copy alone when the area is needed
    if (!acf_st_ && !cuda_ok(cudaStreamCreateWithPriority(&acf_st_, cudaStreamNonBlocking, prio_lo_), "features"))
        return false;
    if (!sd.acf_host && !cuda_ok(cudaMallocHost(&sd.acf_host, 1156 * sizeof(double)), "features")) return false;
    if (!sd.acf_ev && !cuda_ok(cudaEventCreateWithFlags(&sd.acf_ev, cudaEventDisableTiming), "features")) return false;
    if (!cuda_ok(cudaStreamWaitEvent(acf_st_, sd.built_ev, 0), "features") ||
        !cuda_ok(autocorrelation(sd.feat.as<float>(), sd.w, sd.h, fsc, acf_st_), "features") ||
        !cuda_ok(cudaMemcpyAsync(sd.acf_host, sd.acf_dev.p, 1156 * sizeof(double), cudaMemcpyDeviceToHost, acf_st_),
                 "features") ||
        !cuda_ok(cudaEventRecord(sd.acf_ev, acf_st_), "features"))
        return false;
    counts[0] += 2;
    counts[2]++;
    // the engine stream's later work (maps, scores) waits for a build on the side stream when it
    // first needs the side (join_side), so a map's passes over side 0 may start before it
    sd.join_pending = own;
    sd.acf_pending = true;
    sd.built = true;
    sd.mode = mode;
    sd.half = half;
    return true;
}

bool Engine::need_built(bool join) {
    if (!side[0].has || !side[1].has) return fail("NoImages");
    const std::string& fm = set.e("smi_features");
    const int mode = fm == "laplacian" ? 0 : (fm == "three" ? 1 : 2);
    for (int s = 0; s < 2; ++s) {
        Side& sd = side[s];
        if (!sd.built || sd.mode != mode || sd.half != set.b("half") || (sd.preprocess && sd.bake != bake_key()))
            if (!build_side(s)) return false;
    }
    return !join || (join_side(0) && join_side(1));
}

bool Engine::join_side(int s) {
    Side& sd = side[s];
    if (!sd.join_pending) return true;
    if (!cuda_ok(cudaStreamWaitEvent(st, sd.built_ev, 0), "features")) return false;
    sd.join_pending = false;
    return true;
}

bool Engine::need_images() { return need_built() && finish_acf(); }

bool Engine::finish_acf() {
    for (int s = 0; s < 2; ++s) {
        Side& sd = side[s];
        if (!sd.acf_pending) continue;
        if (!cuda_ok(cudaEventSynchronize(sd.acf_ev), "features")) return false;
        counts[3]++;
        // normalise by the zero lag (smi.wgsl:1572-1578)
        const double* raw = sd.acf_host;
        for (int k = 0; k < 1156; ++k) sd.acf[k] = raw[k] / std::max(raw[144 * 4 + (k & 3)], 1e-12);
        sd.acf_pending = false;
    }
    return true;
}

double Engine::pair_area() const {
    // Bartlett correlation area (smi.wgsl:1580-1595)
    double s = 0;
    for (int k = 0; k < 289; ++k) {
        double ra = 0, rb = 0;
        for (int i = 0; i < 4; ++i) {
            ra += side[0].acf[k * 4 + i];
            rb += side[1].acf[k * 4 + i];
        }
        s += ra * rb;
    }
    return std::max(1.0, s / 16.0);
}

bool Engine::features(int s, float* out, size_t len) {
    if (s < 0 || s > 1 || !side[s].has) return fail("features: NoImage");
    if (!need_images()) return false;
    const size_t n = 4 * (size_t)side[s].w * side[s].h;
    if (len < n) return fail("features: BufferTooSmall");
    if (!cuda_ok(cudaMemcpyAsync(out, side[s].feat.p, n * 4, cudaMemcpyDeviceToHost, st), "features")) return false;
    counts[2]++;
    counts[3]++;
    return cuda_ok(cudaStreamSynchronize(st), "features");
}

bool Engine::work_image(int s, float* out, size_t len) {
    if (s < 0 || s > 1 || !side[s].has) return fail("work_image: NoImage");
    Side& sd = side[s];
    if ((!sd.built && !build_side(s)) || !join_side(s)) return false;
    const size_t n = (size_t)sd.w * sd.h;
    if (len < n) return fail("work_image: BufferTooSmall");
    if (!cuda_ok(cudaMemcpyAsync(out, sd.work.p, n * 4, cudaMemcpyDeviceToHost, st), "work_image")) return false;
    counts[2]++;
    counts[3]++;
    return cuda_ok(cudaStreamSynchronize(st), "work_image");
}

// ── FFT plans ─────────────────────────────────────────────────────────────────────────────────

const float2* Engine::twiddles(int n) {
    auto it = tw_.find(n);
    if (it != tw_.end()) return it->second;
    // e^{−2πi t/n}, t < n, then the compile-time lines' per-stage tables (fft.cuh stage_tw_off)
    const int ns = mix_stages(n), extra = stage_tw_off(n, ns);
    std::vector<float2> h((size_t)n + extra);
    for (int t = 0; t < n; ++t) {
        const double a = -2.0 * M_PI * (double)t / (double)n;
        h[t] = make_float2((float)std::cos(a), (float)std::sin(a));
    }
    for (int s = 1, NS = mix_radix(n, 0); s < ns; NS *= mix_radix(n, s), ++s) {
        const int R = mix_radix(n, s), off = n + stage_tw_off(n, s);
        for (int r = 1; r < R; ++r)
            for (int k = 0; k < NS; ++k) {
                const double a = -2.0 * M_PI * (double)(r * k) / (double)(NS * R);
                h[(size_t)off + (size_t)(r - 1) * NS + k] = make_float2((float)std::cos(a), (float)std::sin(a));
            }
    }
    float2* d = nullptr;
    if (cudaMalloc(&d, h.size() * sizeof(float2)) != cudaSuccess) return nullptr;
    // stream-ordered before every kernel that reads it (pageable source: staged before return)
    if (cudaMemcpyAsync(d, h.data(), h.size() * sizeof(float2), cudaMemcpyHostToDevice, st) != cudaSuccess) {
        cudaFree(d);
        return nullptr;
    }
    tw_[n] = d;
    return d;
}

bool Engine::line_plan(int n, LinePlan& p) {
    if (n < 2 || n > kMaxLine) return fail("FFT length " + std::to_string(n) + " is outside 2..8192");
    int a = 0, b = 0, m = n;
    while (m % 2 == 0) m /= 2, ++a;
    while (m % 3 == 0) m /= 3, ++b;
    if (m != 1) return fail("FFT length " + std::to_string(n) + " is not 2^a·3^b (fft_sizes=ladder lengths only)");
    p = LinePlan{};
    p.n = n;
    // power of two: ⌈a/4⌉ stages of radix 16/8/4/2 with balanced bit counts; then the 3s
    const int s2 = (a + 3) / 4;
    for (int i = 0; i < s2; ++i) {
        const int bits = a / s2 + (i < a % s2 ? 1 : 0);
        p.radix[p.nst++] = 1 << bits;
    }
    for (int i = 0; i < b; ++i) p.radix[p.nst++] = 3;
    int tl = (n + 15) / 16;
    tl = ((tl + 31) / 32) * 32;
    p.tl = tl;
    // every stage's butterflies must fit in its threads (BM·tl ≥ n/R)
    for (int s = 0; s < p.nst; ++s) {
        const int R = p.radix[s];
        const int bm = R == 3 ? 6 : 16 / R;
        if (n / R > bm * tl) return fail("internal: FFT plan does not fit its threads");
    }
    p.tw = twiddles(n);
    if (!p.tw) return fail("twiddles: out of device memory");
    return true;
}

// ── shift map ─────────────────────────────────────────────────────────────────────────────────

bool Engine::plan_map(const Mat3& Hm, bool exact, bool calibrated, unsigned cap, double min_overlap, MapJob& job) {
    // the features only enqueued, side 1's build not yet joined: run_map queues side 0's passes
    // first and joins side 1 before its own; the correlation area the calibrated score needs is
    // read when the row pass is launched, so the host does not wait for the builds here
    if (!need_built(false)) return false;
    if (!metric_ok("shift_map")) return false;
    const bool ladder = set.e("fft_sizes") == "ladder";
    if (!ladder) return fail("shift_map: fft_sizes=\"compact\" is not supported by this build (use \"ladder\")");
    job.exact = exact;
    job.calibrated = exact && calibrated;
    job.fr = reg_frame(Hm, side[0].w, side[0].h, side[1].w, side[1].h);
    job.Hc = canvas_H(Hm, job.fr.ox, job.fr.oy);
    MapPlan mp;
    if (cap == 0) {
        mp = auto_shift_plan(job.fr.w, job.fr.h);
    } else {
        // capN (src/smi.zig:414-422) with this build's longest line, 8192
        const unsigned c = largest_smooth(std::min<unsigned>(cap, kMaxLine), ladder);
        mp = linear_corr_plan_rect(job.fr.w, job.fr.h, c, ladder);
    }
    MapGeom& g = job.g;
    g.W = job.fr.w;
    g.Hh = job.fr.h;
    g.ox = job.fr.ox;
    g.oy = job.fr.oy;
    g.cw = mp.cw;
    g.ch = mp.ch;
    g.nx = mp.nx;
    g.ny = mp.ny;
    g.WP = ((g.nx / 2 + 1) + 7) / 8 * 8;
    job.identity_grid = (g.cw == g.W && g.ch == g.Hh);
    const bool three = side[0].mode == 1;
    job.plan = corr_plan_dev(exact, three);
    const CorrPlanDev& P = job.plan;
    if (!line_plan(g.nx, job.row) || !line_plan(g.ny, job.col)) return false;
    job.S = row_split(g.nx, P.n_corr);
    if (job.S == 0) return fail("shift_map: row of " + std::to_string(g.nx) + " does not split to fit shared memory");
    if (!line_plan(g.nx / job.S, job.line)) return false;
    const unsigned floor_n = min_overlap > 0 ? (unsigned)std::floor(min_overlap * (double)g.cw * (double)g.ch) : 0u;
    const double gcell = (double)g.W / (double)g.cw;
    CombineParams& cp = job.cp;
    cp.exact = exact ? 1 : 0;
    cp.calib = job.calibrated ? 1 : 0;
    cp.nf = three ? 3 : 4;
    cp.min_n = (float)std::max(12u, floor_n);
    cp.area = 0.0;  // set by run_map
    job.gcell = gcell;
    cp.ridge = 1e-4;
    cp.inv_nn = 1.0 / ((double)g.nx * (double)g.ny);
    return true;
}

bool Engine::map_buffers(const MapJob& job) {
    const MapGeom& g = job.g;
    const size_t cn = (size_t)g.W * g.Hh, gn = (size_t)g.cw * g.ch;
    const size_t hs = (size_t)job.plan.n_real * g.ny * g.WP * sizeof(float2);
    const size_t qs = (size_t)job.plan.n_corr * g.ny * g.WP * sizeof(float2);
    bool ok = cuda_ok(canvas_a_.ensure(cn * 20), "shift_map") && cuda_ok(canvas_b_.ensure(cn * 20), "shift_map") &&
              cuda_ok(half_a_.ensure(hs), "shift_map") && cuda_ok(half_b_.ensure(hs), "shift_map") &&
              cuda_ok(q_.ensure(qs), "shift_map") && cuda_ok(map_.ensure((size_t)g.nx * g.ny * 4), "shift_map") &&
              cuda_ok(res_.ensure(64), "shift_map");
    if (ok && !job.identity_grid)
        ok = cuda_ok(grid_a_.ensure(gn * 20), "shift_map") && cuda_ok(grid_b_.ensure(gn * 20), "shift_map");
    if (ok && dft_pieces_) ok = cuda_ok(dft_scratch_.ensure(hs), "dft stage");
    return ok;
}

bool Engine::run_map(MapJob& job, cudaEvent_t* ev, float* host_map) {
    const MapGeom& g = job.g;
    const size_t hs = (size_t)job.plan.n_real * g.ny * g.WP * sizeof(float2);
    if (!map_buffers(job)) return false;
    auto rec = [&](int i) {
        if (ev) cudaEventRecord(ev[i], st);
    };
    const Side &A = side[0], &B = side[1];
    const Mat3 hi = inv3_plain(job.Hc);
    float hif[9];
    for (int i = 0; i < 9; ++i) hif[i] = (float)hi[i];
    const bool okdet = std::fabs(det3(job.Hc)) >= 1e-12;
    char* res = res_.as<char>();
    unsigned long long* best = reinterpret_cast<unsigned long long*>(res);
    float* zero = reinterpret_cast<float*>(res + 8);
    double* n00 = reinterpret_cast<double*>(res + 16);
    // a side's canvas (moving warped, fixed pasted) and, when cells exceed a pixel, its grid
    auto canvas_side = [&](int s, const float*& grid) {
        float* canvas = (s == 0 ? canvas_a_ : canvas_b_).as<float>();
        const cudaError_t e = s == 0 ? warp_stack(A.stack.as<float>(), A.w, A.h, hif, okdet, g.W, g.Hh, canvas, st)
                                     : paste_stack(B.stack.as<float>(), B.w, B.h, g.ox, g.oy, g.W, g.Hh, canvas, st);
        if (!cuda_ok(e, "canvas")) return false;
        grid = canvas;
        if (!job.identity_grid) {
            float* gd = (s == 0 ? grid_a_ : grid_b_).as<float>();
            if (!cuda_ok(resample_grid(canvas, g.W, g.Hh, g.cw, g.ch, gd, st), "resample")) return false;
            grid = gd;
        }
        return true;
    };
    unsigned* fault = reinterpret_cast<unsigned*>(res + 24);  // the inverse columns' fault word
    auto lag0 = [&](const float* ga, const float* gb) {
        return cuda_ok(lag0_count(ga, gb, g.cw, g.ch, n00, st), "lag0") &&
               cuda_ok(cudaMemsetAsync(best, 0, 8, st), "shift_map") &&
               cuda_ok(cudaMemsetAsync(fault, 0, 4, st), "shift_map");
    };
    auto rows_of = [&](int s, const float* grid) {
        return cuda_ok(forward_rows(grid, g, job.plan, job.row, (s == 0 ? half_a_ : half_b_).as<float2>(), st),
                       "forward rows");
    };
    unsigned* fault_tc = reinterpret_cast<unsigned*>(res + 28);  // the tensor-core stage's fault word
    if (dft_pieces_ && !cuda_ok(cudaMemsetAsync(fault_tc, 0, 4, st), "shift_map")) return false;
    auto cols_of = [&](int s) {
        float2* half = (s == 0 ? half_a_ : half_b_).as<float2>();
        if (dft_pieces_) {
            if (job.col.radix[0] != 16 || (g.ny / 16) % 4 != 0)
                return fail("dft stage: the column length " + std::to_string(g.ny) + " does not start with radix 16");
            return cuda_ok(dft_scratch_.ensure(hs), "dft stage") &&
                   cuda_ok(forward_cols_tc(half, dft_scratch_.as<float2>(), g, job.plan, job.col, dft_pieces_, fault_tc,
                                           st),
                           "forward columns (tensor-core stage)");
        }
        return cuda_ok(forward_cols(half, g, job.plan, job.col, st), "forward columns");
    };
    // Each side's canvas, grid and half spectra depend on its feature build, the canvas frame and
    // plan, the buffers they live in and, for the moving side, the canvas pose: with the same key
    // as the last map that built them, they are still in the buffers and are reused.
    auto side_key = [&](int s) {
        std::vector<uint64_t> k;
        const DevBuf &cv = s == 0 ? canvas_a_ : canvas_b_, &gd = s == 0 ? grid_a_ : grid_b_,
                     &hf = s == 0 ? half_a_ : half_b_;
        for (const DevBuf* b : {&cv, &gd, &hf}) k.push_back((uint64_t)(uintptr_t)b->p), k.push_back(b->gen);
        for (int v : {s, side[s].mode, (int)side[s].half, g.W, g.Hh, g.ox, g.oy, g.cw, g.ch, g.nx, g.ny, g.WP,
                      (int)job.identity_grid, job.plan.n_real})
            k.push_back((uint64_t)(int64_t)v);
        k.push_back(side[s].ver);
        for (int i = 0; i < job.plan.n_real; ++i) k.push_back((uint64_t)job.plan.planes[i]);
        if (s == 0) {
            for (int i = 0; i < 9; ++i) {
                uint64_t u;
                memcpy(&u, &job.Hc[i], 8);
                k.push_back(u);
            }
            k.push_back(okdet ? 1 : 0);
        }
        return k;
    };
    const bool use_cache = spectra_cache_ && !spectra_cache_off_;
    std::vector<uint64_t> key[2] = {side_key(0), side_key(1)};
    const bool have[2] = {use_cache && key[0] == spec_key_[0], use_cache && key[1] == spec_key_[1]};
    // a kept side still needs its grid for the zero-lag overlap (its canvas is still in place)
    auto kept_grid = [&](int s, const float*& grid) {
        grid = (s == 0 ? canvas_a_ : canvas_b_).as<float>();
        if (!job.identity_grid) grid = (s == 0 ? grid_a_ : grid_b_).as<float>();
        return true;
    };
    auto side_canvas = [&](int s, const float*& grid) { return have[s] ? kept_grid(s, grid) : canvas_side(s, grid); };
    auto side_rows = [&](int s, const float* grid) { return have[s] || rows_of(s, grid); };
    auto side_cols = [&](int s) {
        if (have[s]) return true;
        if (!cols_of(s)) return false;
        spec_key_[s] = key[s];
        return true;
    };
    for (int s = 0; s < 2; ++s)
        if (!have[s]) spec_key_[s].clear();  // until this side's passes are queued
    const float *ga = nullptr, *gb = nullptr;
    if (!join_side(0)) return false;
    if (ev) {
        // in stage order, so each stage's events bracket its own passes
        if (!join_side(1)) return false;
        rec(0);
        if (!side_canvas(0, ga) || !side_canvas(1, gb) || !lag0(ga, gb)) return false;
        rec(1);
        if (!side_rows(0, ga) || !side_rows(1, gb)) return false;
        rec(2);
        if (!side_cols(0) || !side_cols(1)) return false;
        rec(3);
    } else {
        // side 0's passes first: they need only its own build, so they run while side 1's build
        // (on a stream of its own) may still be going; then the wait for it and side 1's passes
        if (!side_canvas(0, ga) || !side_rows(0, ga) || !side_cols(0) || !join_side(1) || !side_canvas(1, gb) ||
            !lag0(ga, gb) || !side_rows(1, gb) || !side_cols(1))
            return false;
    }
    if (!cuda_ok(inverse_columns(half_a_.as<float2>(), half_b_.as<float2>(), g, job.plan, job.col, q_.as<float2>(), st,
                                 1, 0, 0, 0, fault),
                 "inverse columns"))
        return false;
    rec(4);
    // the correlation area (from both sides' autocorrelations) enters the row pass's score
    if (!finish_acf()) return false;
    job.cp.area = std::max(1.0, pair_area() * (1.0 / (job.gcell * job.gcell)));
    const bool tmem = row_pass != "split" && rows_tmem_supported(g.nx, job.plan.n_corr);
    if (tmem && host_map) {
        // the map's rows in chunks of whole waves (one block per SM per row), each chunk copied to
        // the host on the copy stream while the next chunk runs; the last chunk is the smallest,
        // so little copy is left after the last kernel
        if (!copy_st_ && !cuda_ok(cudaStreamCreateWithFlags(&copy_st_, cudaStreamNonBlocking), "shift_map")) return false;
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        const int big = 4 * sms;
        int y0 = 0, c = 0;
        while (y0 < g.ny) {
            const int rows = (g.ny - y0 > big + sms) ? big : g.ny - y0;
            if (!cuda_ok(inverse_rows_score_tmem(q_.as<float2>(), g, job.plan, twiddles(g.nx), job.cp, n00,
                                                 map_.as<float>(), best, zero, st, y0, rows),
                         "inverse rows (tensor memory)"))
                return false;
            if (!chunk_ev_[c] && !cuda_ok(cudaEventCreateWithFlags(&chunk_ev_[c], cudaEventDisableTiming), "shift_map"))
                return false;
            const size_t off = (size_t)y0 * g.nx;
            if (!cuda_ok(cudaEventRecord(chunk_ev_[c], st), "shift_map") ||
                !cuda_ok(cudaStreamWaitEvent(copy_st_, chunk_ev_[c], 0), "shift_map") ||
                !cuda_ok(cudaMemcpyAsync(host_map + off, map_.as<float>() + off, (size_t)rows * g.nx * 4,
                                         cudaMemcpyDeviceToHost, copy_st_),
                         "shift_map"))
                return false;
            y0 += rows;
            c = (c + 1) % kChunkEvents;
        }
        counts[2]++;
    } else if (tmem) {
        if (!cuda_ok(inverse_rows_score_tmem(q_.as<float2>(), g, job.plan, twiddles(g.nx), job.cp, n00, map_.as<float>(),
                                             best, zero, st),
                     "inverse rows (tensor memory)"))
            return false;
    } else if (!cuda_ok(inverse_rows_score(q_.as<float2>(), g, job.plan, job.line, job.S, twiddles(g.nx), job.cp, n00,
                                           map_.as<float>(), best, zero, st),
                        "inverse rows"))
        return false;
    rec(5);
    counts[0] += (job.identity_grid ? 10 : 12) - (have[0] ? (job.identity_grid ? 3 : 4) : 0) -
                 (have[1] ? (job.identity_grid ? 3 : 4) : 0);
    return true;
}

bool Engine::shift_map(const Mat3& Hm, bool exact, bool calibrated, unsigned cap, double min_overlap,
                       zc_shift_result* out, float* map, size_t map_len) {
    MapJob job;
    if (!plan_map(Hm, exact, calibrated, cap, min_overlap, job)) return false;
    const size_t nn = (size_t)job.g.nx * job.g.ny;
    if (map && map_len < nn) return fail("shift_map: MapTooSmall");
    cudaEvent_t ev[kNumStages + 1];
    if (profiling)
        for (auto& e : ev) cudaEventCreate(&e);
    // with the tensor-memory row pass the map leaves in row chunks during the pass (copy_st_)
    const bool chunked = map && row_pass != "split" && rows_tmem_supported(job.g.nx, job.plan.n_corr);
    if (!run_map(job, profiling ? ev : nullptr, chunked ? map : nullptr)) return false;
    unsigned char host[32];
    if (!cuda_ok(cudaMemcpyAsync(host, res_.p, 32, cudaMemcpyDeviceToHost, st), "shift_map")) return false;
    counts[2]++;
    if (map && !chunked) {
        if (!cuda_ok(cudaMemcpyAsync(map, map_.p, nn * 4, cudaMemcpyDeviceToHost, st), "shift_map")) return false;
        counts[2]++;
    }
    if (!cuda_ok(cudaStreamSynchronize(st), "shift_map") ||
        (chunked && !cuda_ok(cudaStreamSynchronize(copy_st_), "shift_map")))
        return false;
    counts[1]++;
    counts[3]++;
    if (profiling) {
        for (int i = 0; i < kNumStages; ++i) {
            float ms = 0;
            cudaEventElapsedTime(&ms, ev[i], ev[i + 1]);
            auto& p = prof[kStageNames[i]];
            p.first += ms;
            p.second++;
        }
        for (auto& e : ev) cudaEventDestroy(e);
    }
    unsigned long long best;
    float zero;
    unsigned fault;
    memcpy(&best, host, 8);
    memcpy(&zero, host + 8, 4);
    memcpy(&fault, host + 24, 4);
    if (fault)
        return fail("shift_map: the inverse column pass gave up waiting for its operand copies (fault " +
                    std::to_string(fault) + "); the map is not valid");
    memcpy(&fault, host + 28, 4);
    if (dft_pieces_ && fault)
        return fail("shift_map: the tensor-core column stage gave up waiting for its products; the map is not valid");
    map_result(job, best, zero, pair_area(), out);
    return true;
}

void Engine::map_result(const MapJob& job, unsigned long long best, float zero, double area, zc_shift_result* out) {
    const MapGeom& g = job.g;
    const size_t nn = (size_t)g.nx * g.ny;
    zc_shift_result r{};
    r.n = g.nx;
    r.n_y = g.ny;
    r.cw = g.cw;
    r.ch = g.ch;
    r.canvas_w = g.W;
    r.canvas_h = g.Hh;
    r.ox = g.ox;
    r.oy = g.oy;
    r.peak = key_float((uint32_t)(best >> 32));
    r.zero = zero;
    r.corr_area_px = area;
    r.exact = job.exact;
    r.calibrated = job.calibrated;
    const uint32_t idx = 0xffffffffu - (uint32_t)(best & 0xffffffffu);
    if (best != 0 && idx < nn) {
        const int64_t py = idx / g.nx, px = idx % g.nx;
        const int64_t lx = px <= g.nx / 2 ? px : px - g.nx;
        const int64_t ly = py <= g.ny / 2 ? py : py - g.ny;
        r.peak_index = idx;
        r.dx = (double)lx * ((double)g.W / (double)g.cw);
        r.dy = (double)ly * ((double)g.Hh / (double)g.ch);
    }
    *out = r;
}

bool Engine::set_dft_stage(unsigned pieces) {
    if (pieces > 3) return fail("set_dft_stage: pieces must be 0 (FP32), 1, 2 or 3");
    if ((int)pieces != dft_pieces_) forget_spectra();  // kept spectra were made with the other stage
    dft_pieces_ = (int)pieces;
    if (!pieces) dft_scratch_.release();
    return true;
}

bool Engine::shift_map_settings(const Mat3& Hm, zc_shift_result* out, float* map, size_t map_len) {
    if (!metric_ok("shift_map")) return false;
    if (set.e("metric") == "ncc") return ncc_shift_map(Hm, out, map, map_len);
    // mapOpts (src/engine.zig:287-293)
    return shift_map(Hm, set.b("exact"), set.b("calibrated"), set.u("map_res"), set.f("min_overlap"), out, map, map_len);
}

double Engine::graph_maps(MapJob& job, unsigned warmup, unsigned steps, size_t flush_bytes) {
    // the capture may not wait on the host or on work recorded outside it: join both builds and
    // read the autocorrelations first (run_map then finds nothing pending)
    if (!join_side(0) || !join_side(1) || !finish_acf() || !cuda_ok(cudaStreamSynchronize(st), "bench_maps"))
        return -1.0;
    const std::string err_before = err;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    const uint32_t launches0 = counts[0];
    bool ok = cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed) == cudaSuccess;
    if (ok) {
        const bool ran = run_map(job, nullptr);
        const cudaError_t ce = cudaStreamEndCapture(st, &graph);
        ok = ran && ce == cudaSuccess && graph && cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
    }
    // the capture launched nothing; each replay launches the map's kernels
    const uint32_t per_map = counts[0] - launches0;
    counts[0] = launches0;
    double ms_sum = 0.0;
    if (ok) {
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        ok = cudaEventCreate(&e0) == cudaSuccess && cudaEventCreate(&e1) == cudaSuccess;
        for (unsigned i = 0; ok && i < warmup; ++i) ok = cudaGraphLaunch(exec, st) == cudaSuccess;
        for (unsigned i = 0; ok && i < steps; ++i) {
            float ms = 0.f;
            ok = cudaMemsetAsync(flush_.p, (int)(i & 0xff), flush_bytes, st) == cudaSuccess &&
                 cudaEventRecord(e0, st) == cudaSuccess && cudaGraphLaunch(exec, st) == cudaSuccess &&
                 cudaEventRecord(e1, st) == cudaSuccess && cudaEventSynchronize(e1) == cudaSuccess &&
                 cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess;
            ms_sum += ms;
        }
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        counts[0] += per_map * (warmup + steps);
    }
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (!ok) {
        cudaGetLastError();  // a refused capture is not this call's error
        err = err_before;
        log_event("bench_maps: graph replay unavailable; the instrumented maps' time is reported");
        return -1.0;
    }
    return ms_sum / std::max(steps, 1u);
}

bool Engine::bench_maps(const Mat3& Hm, unsigned flags, unsigned cap, unsigned warmup, unsigned steps, double* out,
                        size_t out_len) {
    if (out_len < 16) return fail("bench_maps: output needs 16 doubles");
    // every timed map builds both sides' spectra: the benchmark times whole maps
    struct NoReuse {
        bool& f;
        explicit NoReuse(bool& x) : f(x) { f = true; }
        ~NoReuse() { f = false; }
    } no_reuse(spectra_cache_off_);
    MapJob job;
    if (!plan_map(Hm, (flags & 1) != 0, (flags & 2) != 0, cap, 0.0, job)) return false;
    // an L2 flush between timed maps: write a buffer larger than the 126 MB L2
    const size_t flush_bytes = (size_t)256 << 20;
    if (!cuda_ok(flush_.ensure(flush_bytes), "bench_maps")) return false;
    std::vector<cudaEvent_t> ev((size_t)(kNumStages + 1) * std::max(steps, 1u));
    for (auto& e : ev) cudaEventCreate(&e);
    for (unsigned i = 0; i < warmup; ++i)
        if (!run_map(job, nullptr)) return false;
    for (unsigned i = 0; i < steps; ++i) {
        cudaMemsetAsync(flush_.p, (int)(i & 0xff), flush_bytes, st);
        if (!run_map(job, &ev[(size_t)i * (kNumStages + 1)])) return false;
    }
    if (!cuda_ok(cudaStreamSynchronize(st), "bench_maps")) return false;
    double stage[kNumStages] = {0}, total = 0;
    for (unsigned i = 0; i < steps; ++i) {
        cudaEvent_t* e = &ev[(size_t)i * (kNumStages + 1)];
        float ms = 0;
        cudaEventElapsedTime(&ms, e[0], e[kNumStages]);
        total += ms;
        for (int s = 0; s < kNumStages; ++s) {
            cudaEventElapsedTime(&ms, e[s], e[s + 1]);
            stage[s] += ms;
        }
    }
    for (auto& e : ev) cudaEventDestroy(e);
    const double instrumented = total / std::max(steps, 1u);
    // whole maps replayed from one CUDA graph of the map's passes (no launch gaps between them),
    // each timed by events around the replay with the same L2 flush before it; the stage times
    // above come from the event-instrumented maps. A capture the driver refuses leaves the
    // instrumented time.
    const double graphed = graph_maps(job, warmup, steps, flush_bytes);
    for (size_t i = 0; i < out_len; ++i) out[i] = 0;
    out[0] = graphed > 0 ? graphed : instrumented;
    out[6] = instrumented;
    for (int s = 0; s < kNumStages; ++s) out[1 + s] = stage[s] / std::max(steps, 1u);
    out[8] = job.g.nx;
    out[9] = job.g.ny;
    out[10] = job.g.cw;
    out[11] = job.g.ch;
    out[12] = job.plan.n_real;
    out[13] = job.plan.n_corr;
    out[14] = job.S;
    out[7] = job.g.Hh;
    out[15] = job.g.W;
    return true;
}

}  // namespace zc
