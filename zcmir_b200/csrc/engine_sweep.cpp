// The rotation × scale sweep and the search built on it, restated from the reference's
// src/search.zig (Sweep.sweep 300-494, gnBatch 539-614, runSweep 663-820).
//
// Every candidate pose's translation map on a coarse G×G canvas: candidates are grouped by plane
// size; per group the fixed window's spectra are formed once, then batches of candidates run
// pack → forward rows → forward columns → products + inverse columns → inverse rows with the
// per-shift score → peaks, all on the engine's stream, with only the peaks read back at the end.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "engine.hpp"
#include "lie.hpp"

namespace zc {

namespace {

constexpr size_t kSweepBudget = 1ull << 30;  // device bytes of one batch's work buffers
constexpr int kSweepMaxBatch = 128;
constexpr size_t kTuneBudget = 8ull << 30;  // device bytes of one batch's work buffers while tuning
constexpr int kMom = 45, kCoef = 102, kGrad = 44;  // per pose: moment sums, coefficients, tangent sums

size_t pitch_of(int nx) { return (size_t)((nx / 2 + 1) + 7) / 8 * 8; }

}  // namespace

bool Engine::sweep_setup(const Mat3& H0, const SweepGrid& gv, int G, SweepOut& out) {
    if (!need_images()) return false;
    if (gv.count() == 0) return fail("sweep: empty candidate grid");
    const Side &A = side[0], &B = side[1];
    const double fw = B.w, fh = B.h, mw = A.w, mh = A.h;
    const bool ladder = set.e("fft_sizes") != "compact";
    out = SweepOut{};
    // the G×G canvas is a square centred on the fixed image, wide enough to hold the moving image
    // under the candidate with the biggest singular value, but never over twice the fixed image
    const auto cm = map_pt(H0, (mw + 1) / 2, (mh + 1) / 2);
    double s_max = -INFINITY;
    for (double s : gv.sigmas)
        for (double k : gv.shears)
            for (double a : gv.anisos) s_max = std::max(s_max, sv2(cand_linear(0, s, k, a))[0]);
    const double D = std::min(2 * std::max(fw, fh), std::max(std::max(fw, fh), s_max * std::hypot(mw, mh)));
    const double cell = D / G, ox = (fw + 1) / 2 - D / 2, oy = (fh + 1) / 2 - D / 2;
    const auto fcx = sweep_cells(0.5, fw + 0.5, ox, cell, G), fcy = sweep_cells(0.5, fh + 0.5, oy, cell, G);
    const int Fx = fcx[1] - fcx[0], Fy = fcy[1] - fcy[0];
    out.cell = cell, out.ox = ox, out.oy = oy, out.G = G, out.fx0 = fcx[0], out.fy0 = fcy[0], out.Fx = Fx, out.Fy = Fy;
    // candidates (θ-major), their footprints, plane sizes and taps
    const double s0r = std::sqrt(std::fabs(H0[0] * H0[4] - H0[1] * H0[3]));
    const double s0 = (s0r == 0 || std::isnan(s0r)) ? 1 : s0r;
    const int nc = (int)gv.count();
    out.cands.reserve(nc);
    for (size_t i = 0; i < gv.thetas.size(); ++i)
        for (size_t j = 0; j < gv.sigmas.size(); ++j)
            for (size_t ik = 0; ik < gv.shears.size(); ++ik)
                for (size_t ia = 0; ia < gv.anisos.size(); ++ia) {
                    const double th = gv.thetas[i], s = gv.sigmas[j];
                    const Lin2 L = cand_linear(th, s, gv.shears[ik], gv.anisos[ia]);
                    const Mat3 H = mul3(about_c(cm, L), H0);
                    double x0 = INFINITY, x1 = -INFINITY, y0 = INFINITY, y1 = -INFINITY;
                    const double q[4][2] = {{0.5, 0.5}, {mw + 0.5, 0.5}, {mw + 0.5, mh + 0.5}, {0.5, mh + 0.5}};
                    for (const auto& p : q) {
                        const auto m = map_pt(H, p[0], p[1]);
                        x0 = std::min(x0, m[0]), x1 = std::max(x1, m[0]);
                        y0 = std::min(y0, m[1]), y1 = std::max(y1, m[1]);
                    }
                    const bool ok = std::isfinite(x0 + x1 + y0 + y1);
                    const auto mcx = ok ? sweep_cells(x0, x1, ox, cell, G) : std::array<int, 2>{0, G};
                    const auto mcy = ok ? sweep_cells(y0, y1, oy, cell, G) : std::array<int, 2>{0, G};
                    SweepCand c;
                    c.it = (int)i, c.is = (int)j, c.ik = (int)ik, c.ia = (int)ia, c.th = th, c.s = s, c.H = H;
                    c.gx0 = mcx[0], c.gy0 = mcy[0];
                    c.nx = (int)sweep_plane_len((unsigned)(mcx[1] - mcx[0] + Fx - 1), ladder);
                    c.ny = (int)sweep_plane_len((unsigned)(mcy[1] - mcy[0] + Fy - 1), ladder);
                    // taps per cell side: enough that the box filter samples the moving image at its finest
                    // (the candidate's smaller singular value)
                    c.taps = (float)std::min(6.0, std::max(1.0, std::ceil(cell / (sv2(L)[1] * s0) - 1e-3)));
                    out.cands.push_back(c);
                }
    // slots: candidates grouped by plane size (stable)
    std::vector<int>& perm = out.perm;
    perm.resize(nc);
    for (int k = 0; k < nc; ++k) perm[k] = k;
    std::stable_sort(perm.begin(), perm.end(), [&](int a, int b) {
        const uint64_t ka = ((uint64_t)out.cands[a].nx << 32) | (uint64_t)out.cands[a].ny;
        const uint64_t kb = ((uint64_t)out.cands[b].nx << 32) | (uint64_t)out.cands[b].ny;
        return ka < kb;
    });
    return true;
}

bool Engine::sweep_maps(const Mat3& H0, const SweepGrid& gv, int G, bool exact, int n_peak, double min_overlap,
                        SweepOut& out, int batch, int shard, int nshard) {
    if (n_peak < 1 || n_peak > 16) return fail("sweep: n_peak must be 1..16");
    if (nshard < 1 || shard < 0 || shard >= nshard) return fail("sweep: shard must be 0..nshard-1");
    if (!sweep_setup(H0, gv, G, out)) return false;
    const bool three = side[0].mode == 1;
    const CorrPlanDev plan = corr_plan_dev(exact, three);
    const Side &A = side[0], &B = side[1];
    const double fw = B.w, fh = B.h;
    const double cell = out.cell, ox = out.ox, oy = out.oy;
    const std::array<int, 2> fcx{out.fx0, out.fx0 + out.Fx}, fcy{out.fy0, out.fy0 + out.Fy};
    const int Fx = out.Fx, Fy = out.Fy;
    const int nc = (int)out.cands.size();
    // this shard's candidates in slot order: slots s ≡ shard (mod nshard), so every shard gets
    // candidates of every plane size
    std::vector<int> perm;
    for (int s = shard; s < nc; s += nshard) perm.push_back(out.perm[s]);
    const int nm = (int)perm.size();
    std::vector<float> poses((size_t)(nm + 1) * 12, 0.f);
    for (int k = 0; k < nm; ++k) {
        const SweepCand& c = out.cands[perm[k]];
        const Mat3 Hi = inv3(c.H);
        for (int q = 0; q < 9; ++q) poses[(size_t)k * 12 + q] = (float)Hi[q];
        poses[(size_t)k * 12 + 9] = c.taps;
        poses[(size_t)k * 12 + 10] = (float)c.gx0;
        poses[(size_t)k * 12 + 11] = (float)c.gy0;
    }
    // the fixed window's pose: identity, taps from the cell, its first cell
    float* fp = poses.data() + (size_t)nm * 12;
    fp[0] = fp[4] = fp[8] = 1.f;
    fp[9] = (float)std::min(6.0, std::max(1.0, std::ceil(cell - 1e-3)));
    fp[10] = (float)fcx[0];
    fp[11] = (float)fcy[0];
    // plane classes in slot order: [k0, k1) of the slots share one plane size
    struct Cls {
        int k0, k1, nx, ny, b, S;
        LinePlan row, col, line;
        const float2* tw;
    };
    std::vector<Cls> cls;
    for (int k0 = 0; k0 < nm;) {
        const int nx = out.cands[perm[k0]].nx, ny = out.cands[perm[k0]].ny;
        int k1 = k0;
        while (k1 < nm && out.cands[perm[k1]].nx == nx && out.cands[perm[k1]].ny == ny) ++k1;
        cls.push_back(Cls{k0, k1, nx, ny, 0, 0, {}, {}, {}, nullptr});
        k0 = k1;
    }
    auto per_item = [&](int nx, int ny) {
        const size_t pstride = (size_t)ny * pitch_of(nx);
        return (size_t)5 * (nx - Fx + 1) * (ny - Fy + 1) * 4 + (size_t)(plan.n_real + plan.n_corr) * pstride * 8 +
               (size_t)nx * ny * 4;
    };
    // batch per class: the caller's, else the tuned one, else the environment's, else as many as
    // the budget holds (at most kSweepMaxBatch)
    int env_b = 0;
    if (const char* v = getenv("ZCMIR_B200_SWEEP_BATCH")) env_b = std::max(0, atoi(v));
    size_t grid_max = 0, half_max = 0, q_max = 0, map_max = 0, fhalf_max = 0;
    int bmax = 1;
    for (Cls& c : cls) {
        int b = batch;
        if (!sweep_force_.empty()) {
            const auto it = sweep_force_.find({c.nx, c.ny});
            b = it != sweep_force_.end() ? it->second : b;
        }
        if (b <= 0) {
            const auto it = sweep_tuned_.find({c.nx, c.ny, plan.n_corr, exact ? 1 : 0});
            b = it != sweep_tuned_.end() ? it->second : 0;
        }
        if (b <= 0) b = env_b;
        if (b <= 0) b = (int)std::max<size_t>(1, std::min<size_t>(kSweepMaxBatch, kSweepBudget / per_item(c.nx, c.ny)));
        c.b = std::min(b, c.k1 - c.k0);
        bmax = std::max(bmax, c.b);
        const size_t pstride = (size_t)c.ny * pitch_of(c.nx);
        grid_max = std::max(grid_max, (size_t)5 * (c.nx - Fx + 1) * (c.ny - Fy + 1) * c.b);
        half_max = std::max(half_max, (size_t)plan.n_real * pstride * c.b);
        q_max = std::max(q_max, (size_t)plan.n_corr * pstride * c.b);
        map_max = std::max(map_max, (size_t)c.nx * c.ny * c.b);
        fhalf_max = std::max(fhalf_max, (size_t)plan.n_real * pstride);
        out.n = std::max({out.n, c.nx, c.ny});
        // line plans and twiddles now: nothing may allocate while the launches are captured
        if (!line_plan(c.nx, c.row) || !line_plan(c.ny, c.col)) return false;
        c.S = row_split(c.nx, plan.n_corr);
        if (c.S == 0) return fail("sweep: a plane row of " + std::to_string(c.nx) + " does not fit the row pass");
        if (!line_plan(c.nx / c.S, c.line)) return false;
        c.tw = twiddles(c.nx);
        if (!c.tw) return fail("sweep: twiddles: out of device memory");
    }
    const size_t fgrid = (size_t)5 * Fx * Fy;
    const size_t na = (size_t)A.w * A.h, nb = (size_t)B.w * B.h;
    bool ok = cuda_ok(sw_il_[0].ensure(na * 20), "sweep") && cuda_ok(sw_il_[1].ensure(nb * 20), "sweep") &&
              cuda_ok(sw_poses_.ensure(poses.size() * 4), "sweep") && cuda_ok(sw_fgrid_.ensure(fgrid * 4), "sweep") &&
              cuda_ok(sw_fhalf_.ensure(fhalf_max * 8), "sweep") && cuda_ok(sw_grid_.ensure(grid_max * 4), "sweep") &&
              cuda_ok(sw_half_.ensure(half_max * 8), "sweep") && cuda_ok(sw_q_.ensure(q_max * 8), "sweep") &&
              cuda_ok(sw_map_.ensure(map_max * 4), "sweep") && cuda_ok(sw_n0_.ensure((size_t)bmax * 8), "sweep") &&
              cuda_ok(sw_ps_.ensure((size_t)std::max(nm, 1) * n_peak * 4), "sweep") &&
              cuda_ok(sw_pi_.ensure((size_t)std::max(nm, 1) * n_peak * 4), "sweep");
    if (!ok) return false;
    if (!cuda_ok(cudaMemcpyAsync(sw_poses_.p, poses.data(), poses.size() * 4, cudaMemcpyHostToDevice, st), "sweep"))
        return false;
    const SweepCanvas cv{(float)ox, (float)oy, (float)cell, G};
    const float4* ila = sw_il_[0].as<float4>();
    const float4* ilb = sw_il_[1].as<float4>();
    out.min_n = (unsigned)std::max(12.0, std::floor(min_overlap * (fw * fh) / (cell * cell) + 0.5));
    CombineParams cp{};
    cp.exact = exact ? 1 : 0;
    cp.calib = 0;
    cp.nf = three ? 3 : 4;
    cp.min_n = (float)out.min_n;
    cp.area = 1.0;
    cp.ridge = 1e-4;
    // per-class events (stream-ordered runs only: they time each plane class)
    const bool use_graph = sweep_with_stack_ || (sweep_force_.empty() && (!getenv("ZCMIR_B200_SWEEP_GRAPH") ||
                                                                         atoi(getenv("ZCMIR_B200_SWEEP_GRAPH")) != 0));
    std::vector<cudaEvent_t> cev;
    if (!use_graph) {
        cev.resize(cls.size() + 1);
        for (auto& e : cev) cudaEventCreate(&e);
    }
    auto free_cev = [&] {
        for (auto& e : cev) cudaEventDestroy(e);
        cev.clear();
    };
    // every launch of the sweep's maps, in order; returns the launch count (−1 on an error)
    auto enqueue = [&]() -> int {
        int launches = 0;
        if (!cuda_ok(sweep_interleave(A.stack.as<float>(), (int)na, sw_il_[0].as<float4>(), st), "sweep") ||
            !cuda_ok(sweep_interleave(B.stack.as<float>(), (int)nb, sw_il_[1].as<float4>(), st), "sweep") ||
            !cuda_ok(sweep_pack(ilb, B.w, B.h, sw_poses_.as<float>(), nm, 1, Fx, Fy, cv, nullptr, 0, 0, 0, 0,
                                sw_fgrid_.as<float>(), nullptr, st),
                     "sweep"))
            return -1;
        launches += 3;
        for (size_t ci = 0; ci < cls.size(); ++ci) {
            const Cls& c = cls[ci];
            if (!cev.empty()) cudaEventRecord(cev[ci], st);
            MapGeom gm{};
            gm.nx = c.nx, gm.ny = c.ny, gm.WP = (int)pitch_of(c.nx);
            gm.cw = c.nx - Fx + 1, gm.ch = c.ny - Fy + 1;
            gm.W = gm.cw, gm.Hh = gm.ch;
            MapGeom gf = gm;
            gf.cw = Fx, gf.ch = Fy;
            CombineParams cpc = cp;
            cpc.inv_nn = 1.0 / ((double)c.nx * (double)c.ny);
            const size_t pstride = (size_t)c.ny * gm.WP;
            const size_t wn = (size_t)gm.cw * gm.ch;
            // the fixed window's spectra for this plane size
            if (!cuda_ok(forward_rows(sw_fgrid_.as<float>(), gf, plan, c.row, sw_fhalf_.as<float2>(), st), "sweep") ||
                !cuda_ok(forward_cols(sw_fhalf_.as<float2>(), gf, plan, c.col, st), "sweep"))
                return -1;
            launches += 2;
            for (int c0 = c.k0; c0 < c.k1; c0 += c.b) {
                const int b = std::min(c.b, c.k1 - c0);
                const size_t hs = (size_t)plan.n_real * pstride, qs = (size_t)plan.n_corr * pstride;
                if (!cuda_ok(sweep_pack(ila, A.w, A.h, sw_poses_.as<float>(), c0, b, gm.cw, gm.ch, cv,
                                        sw_fgrid_.as<float>(), fcx[0], fcy[0], Fx, Fy, sw_grid_.as<float>(),
                                        sw_n0_.as<double>(), st),
                             "sweep") ||
                    !cuda_ok(forward_rows(sw_grid_.as<float>(), gm, plan, c.row, sw_half_.as<float2>(), st, b, 5 * wn, hs),
                             "sweep") ||
                    !cuda_ok(forward_cols(sw_half_.as<float2>(), gm, plan, c.col, st, b), "sweep") ||
                    !cuda_ok(inverse_columns(sw_half_.as<float2>(), sw_fhalf_.as<float2>(), gm, plan, c.col,
                                             sw_q_.as<float2>(), st, b, hs, 0, qs),
                             "sweep") ||
                    !cuda_ok(inverse_rows_score(sw_q_.as<float2>(), gm, plan, c.line, c.S, c.tw, cpc,
                                                sw_n0_.as<double>(), sw_map_.as<float>(), nullptr, nullptr, st, b, qs,
                                                (size_t)c.nx * c.ny),
                             "sweep") ||
                    !cuda_ok(sweep_peaks(sw_map_.as<float>(), c.nx, c.ny, (size_t)c.nx * c.ny, b, n_peak, c0,
                                         sw_ps_.as<float>(), sw_pi_.as<uint32_t>(), st),
                             "sweep"))
                    return -1;
                launches += 6;
            }
        }
        if (!cev.empty()) cudaEventRecord(cev.back(), st);
        return launches;
    };
    out.groups = (int)cls.size();
    out.batches = 0;
    for (const Cls& c : cls) out.batches += (c.k1 - c.k0 + c.b - 1) / c.b;
    // the signature of everything the launches read from the host: pointers, sizes, the schedule
    std::vector<uint64_t> sig;
    if (use_graph) {
        auto put = [&](uint64_t v) { sig.push_back(v); };
        auto putd = [&](double v) {
            uint64_t u;
            std::memcpy(&u, &v, 8);
            sig.push_back(u);
        };
        const void* ptrs[] = {A.stack.p, B.stack.p, sw_il_[0].p, sw_il_[1].p, sw_poses_.p, sw_fgrid_.p, sw_fhalf_.p,
                              sw_grid_.p, sw_half_.p, sw_q_.p, sw_map_.p, sw_n0_.p, sw_ps_.p, sw_pi_.p};
        for (const void* q : ptrs) put((uint64_t)(uintptr_t)q);
        for (int v : {A.w, A.h, B.w, B.h, nm, n_peak, Fx, Fy, fcx[0], fcy[0], G, plan.n_real, plan.n_corr, exact ? 1 : 0,
                      three ? 1 : 0, (int)out.min_n})
            put((uint64_t)(int64_t)v);
        putd(ox), putd(oy), putd(cell);
        for (const Cls& c : cls)
            for (uint64_t v : {(uint64_t)c.k0, (uint64_t)c.k1, (uint64_t)c.nx, (uint64_t)c.ny, (uint64_t)c.b,
                               (uint64_t)c.S, (uint64_t)(uintptr_t)c.tw, (uint64_t)(uintptr_t)c.row.tw,
                               (uint64_t)(uintptr_t)c.col.tw, (uint64_t)(uintptr_t)c.line.tw})
                put(v);
        // with the stack's branch: the loaded stack and every buffer its maps use
        put(sweep_with_stack_ ? stack_gen_ : 0);
        if (sweep_with_stack_)
            for (const DevBuf* b : {&canvas_a_, &canvas_b_, &grid_a_, &grid_b_, &half_a_, &half_b_, &q_, &map_, &res_,
                                    &stack_res_, &dft_scratch_})
                put((uint64_t)(uintptr_t)b->p), put(b->gen);
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    auto done = [&](bool r) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        free_cev();
        return r;
    };
    int launches = 0;
    out.graph = false;
    if (use_graph) {
        if (!sweep_exec_ || sig != sweep_sig_) {
            // capture the launches once (nothing runs), instantiate, keep while the signature holds
            if (sweep_exec_) {
                cudaGraphExecDestroy(sweep_exec_);
                sweep_exec_ = nullptr;
            }
            sweep_sig_.clear();
            cudaGraph_t graph = nullptr;
            const std::string err_before = err;
            bool cap_ok = cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed) == cudaSuccess;
            int n = -1;
            if (cap_ok) {
                int ns = 0;
                if (sweep_with_stack_) {
                    // the stack's maps on a second branch (their own buffers), forked from and
                    // joined back into the capture, so the two run side by side in one launch
                    cap_ok = cudaEventRecord(fork_ev_, st) == cudaSuccess &&
                             cudaStreamWaitEvent(branch_st_, fork_ev_, 0) == cudaSuccess;
                    std::swap(st, branch_st_);
                    ns = cap_ok ? stack_enqueue() : -1;
                    std::swap(st, branch_st_);
                    if (ns > 0) counts[0] -= (uint32_t)ns;  // captured, not launched: counted per replay
                }
                n = enqueue();
                if (sweep_with_stack_)
                    cap_ok = cap_ok && cudaEventRecord(join_ev_, branch_st_) == cudaSuccess &&
                             cudaStreamWaitEvent(st, join_ev_, 0) == cudaSuccess;
                n = (n < 0 || ns < 0 || !cap_ok) ? -1 : n + ns;
                const cudaError_t ce = cudaStreamEndCapture(st, &graph);
                cap_ok = n >= 0 && ce == cudaSuccess && graph &&
                         cudaGraphInstantiate(&sweep_exec_, graph, 0) == cudaSuccess;
            }
            if (graph) cudaGraphDestroy(graph);
            if (cap_ok) {
                sweep_sig_ = sig;
                sweep_launches_ = n;
            } else if (sweep_with_stack_) {
                cudaGetLastError();
                if (sweep_exec_) cudaGraphExecDestroy(sweep_exec_);
                sweep_exec_ = nullptr;
                return done(fail("sweep_stack: the combined graph could not be captured" +
                                 (err.empty() ? std::string() : ": " + err)));
            } else {
                cudaGetLastError();  // a refused capture is not this call's error: run stream-ordered
                err = err_before;
                if (sweep_exec_) cudaGraphExecDestroy(sweep_exec_);
                sweep_exec_ = nullptr;
            }
        }
        if (sweep_exec_) {
            cudaEventRecord(e0, st);
            if (!cuda_ok(cudaGraphLaunch(sweep_exec_, st), "sweep")) return done(false);
            launches = sweep_launches_;
            out.graph = true;
        }
    }
    if (!out.graph) {
        cudaEventRecord(e0, st);
        launches = enqueue();
        if (launches < 0) return done(false);
    }
    cudaEventRecord(e1, st);
    std::vector<float> ps((size_t)nm * n_peak);
    std::vector<uint32_t> pi((size_t)nm * n_peak);
    if (!cuda_ok(cudaMemcpyAsync(ps.data(), sw_ps_.p, ps.size() * 4, cudaMemcpyDeviceToHost, st), "sweep") ||
        !cuda_ok(cudaMemcpyAsync(pi.data(), sw_pi_.p, pi.size() * 4, cudaMemcpyDeviceToHost, st), "sweep") ||
        !cuda_ok(cudaStreamSynchronize(st), "sweep"))
        return done(false);
    cudaEventElapsedTime(&out.ms, e0, e1);
    out.classes.clear();
    for (size_t ci = 0; ci < cls.size(); ++ci) {
        float cms = -1.f;
        if (!cev.empty()) cudaEventElapsedTime(&cms, cev[ci], cev[ci + 1]);
        out.classes.push_back({(double)cls[ci].nx, (double)cls[ci].ny, (double)(cls[ci].k1 - cls[ci].k0),
                               (double)cls[ci].b, (double)cms});
    }
    out.launches = launches;
    counts[0] += launches;
    counts[1]++;
    counts[2] += 2;
    counts[3]++;
    // each candidate's lane maxima, scores in fixed pixels (n counts cells); other shards' stay empty
    const double c2 = cell * cell;
    out.lane_score.assign((size_t)nc * n_peak, 0.f);
    out.lane_idx.assign((size_t)nc * n_peak, 0xffffffffu);
    for (int j = 0; j < nm; ++j)
        for (int k = 0; k < n_peak; ++k) {
            out.lane_score[(size_t)perm[j] * n_peak + k] = (float)((double)ps[(size_t)j * n_peak + k] * c2);
            out.lane_idx[(size_t)perm[j] * n_peak + k] = pi[(size_t)j * n_peak + k];
        }
    sweep_make_peaks(out, n_peak);
    return done(true);
}

// Peaks → poses (src/search.zig:460-493) from the lane maxima, slot by slot (the reference's order).
void Engine::sweep_make_peaks(SweepOut& out, int n_peak) {
    const int nc = (int)out.cands.size();
    out.peaks.clear();
    out.best.assign(nc, 0.f);
    for (int slot = 0; slot < nc; ++slot) {
        const int ci = out.perm[slot];
        const SweepCand& cd = out.cands[ci];
        for (int k = 0; k < n_peak; ++k) {
            const double v = out.lane_score[(size_t)ci * n_peak + k];
            const uint32_t t = out.lane_idx[(size_t)ci * n_peak + k];
            if (!(v > 0) || (uint64_t)t >= (uint64_t)cd.nx * cd.ny) continue;
            if (k == 0) out.best[ci] = (float)v;
            // the map index gives a lag between the moving and fixed windows, from −(F − 1) up to
            // the moving window's width − 1; adding the windows' first cells turns it into the
            // moving image's displacement on the canvas in cells, and the pose is corrected by T(−d)
            const int py = (int)(t / (uint32_t)cd.nx), px = (int)(t - (uint32_t)py * (uint32_t)cd.nx);
            const int wx = cd.nx - out.Fx + 1, wy = cd.ny - out.Fy + 1;
            const int lx = px < wx ? px : px - cd.nx, ly = py < wy ? py : py - cd.ny;
            SweepPeak p;
            p.score = v;
            p.cand = ci, p.it = cd.it, p.is = cd.is, p.ik = cd.ik, p.ia = cd.ia, p.th = cd.th, p.s = cd.s;
            p.sx = cd.gx0 + lx - out.fx0;
            p.sy = cd.gy0 + ly - out.fy0;
            p.H = mul3(translate(-p.sx * out.cell, -p.sy * out.cell), cd.H);
            out.peaks.push_back(p);
        }
    }
}

// gn_batch with the loop on the device: per iteration the poses' inverse maps, their moments,
// coefficients and tangent sums (masked to the poses still moving), then one warp per pose builds
// the candidates (k_gn_propose), the candidates are scored, and k_gn_select keeps the first that
// beats each pose's score. The host reads the moved flags once per kGnBatch iterations, to stop
// when no pose moves; the iterations past the last move only launch masked-out kernels.
bool Engine::gn_batch_dev(const std::vector<Mat3>& Hs, unsigned iters, const std::vector<double>& amps,
                          std::vector<ScoredPose>& out) {
    out.clear();
    if (Hs.empty()) return true;
    if (!need_images() || !metric_ok("score")) return false;
    const bool homog = set.e("group") == "homography", sym = set.b("symmetric"), exact = set.b("exact");
    const Side &A = side[0], &B = side[1];
    GnAmps ga{};
    ga.n = (int)amps.size();
    for (int k = 0; k < ga.n; ++k) ga.v[k] = amps[k];
    const int n = (int)Hs.size(), nd = sym ? 2 : 1;
    const GnDims d{n, ga.n + 5, n_keys(homog), homog ? 1 : 0, sym ? 1 : 0, A.w, A.h, B.w, B.h};
    const size_t nt = (size_t)n * d.T, mt = (size_t)nd * nt, m = (size_t)nd * n;
    const size_t act_b = (size_t)(n + 15) / 16 * 16;
    bool ok = cuda_ok(gn_H_.ensure((size_t)n * 9 * 8), "refine") && cuda_ok(gn_Htry_.ensure(nt * 9 * 8), "refine") &&
              cuda_ok(gn_valid_.ensure(nt), "refine") && cuda_ok(gn_active_.ensure(act_b), "refine") &&
              cuda_ok(gn_cur_.ensure((size_t)n * 8), "refine") && cuda_ok(pose_hinv_.ensure(mt * 9 * 4), "refine") &&
              cuda_ok(pose_sums_.ensure(mt * kMom * 8), "refine") &&
              cuda_ok(pose_coef_.ensure(mt * kCoef * 4), "refine") && cuda_ok(pose_score_.ensure(mt * 8), "refine") &&
              cuda_ok(pose_tsum_.ensure(m * kGrad * 8), "refine") && cuda_ok(pose_gens_.ensure(2 * 72 * 4), "refine") &&
              cuda_ok(gn_pin_.ensure((size_t)n * 9 * 8 + (size_t)n * 8 + act_b + 2 * 72 * 4), "refine");
    if (!ok) return false;
    // page-locked staging: poses (f64), scores (f64), moved flags, generators (f32)
    double* hH = gn_pin_.as<double>();
    double* hcur = hH + (size_t)n * 9;
    unsigned char* hact = reinterpret_cast<unsigned char*>(hcur + n);
    float* hgens = reinterpret_cast<float*>(hact + act_b);
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < 9; ++k) hH[(size_t)i * 9 + k] = Hs[i][k];
    const auto gf = generators(homog, B.w, B.h), gi = generators(homog, A.w, A.h);
    for (int k = 0; k < 8; ++k)
        for (int e = 0; e < 9; ++e) {
            hgens[k * 9 + e] = (float)gf[k][e];
            hgens[72 + k * 9 + e] = (float)gi[k][e];
        }
    double* H = gn_H_.as<double>();
    double* Ht = gn_Htry_.as<double>();
    double* cur = gn_cur_.as<double>();
    unsigned char* act = gn_active_.as<unsigned char>();
    unsigned char* valid = gn_valid_.as<unsigned char>();
    float* dh = pose_hinv_.as<float>();
    float* dg = pose_gens_.as<float>();
    double* sums = pose_sums_.as<double>();
    double* tsum = pose_tsum_.as<double>();
    double* score = pose_score_.as<double>();
    float* coef = pose_coef_.as<float>();
    std::vector<double> ninf((size_t)n, -INFINITY);
    if (!cuda_ok(cudaMemcpyAsync(H, hH, (size_t)n * 9 * 8, cudaMemcpyHostToDevice, st), "refine") ||
        !cuda_ok(cudaMemcpyAsync(dg, hgens, 2 * 72 * 4, cudaMemcpyHostToDevice, st), "refine") ||
        !cuda_ok(cudaMemsetAsync(act, 1, (size_t)n, st), "refine"))
        return false;
    std::copy(ninf.begin(), ninf.end(), hcur);
    if (!cuda_ok(cudaMemcpyAsync(cur, hcur, (size_t)n * 8, cudaMemcpyHostToDevice, st), "refine")) return false;
    counts[2] += 3;
    const PoseSide pa{A.feat.as<float>(), A.feat4.as<float4>(), A.w, A.h},
        pb{B.feat.as<float>(), B.feat4.as<float4>(), B.w, B.h};
    PoseRed rd;
    if (!pose_red((int)nt, rd)) return false;
    constexpr unsigned kGnBatch = 4;
    for (unsigned it = 0; it < iters && !cancel; ++it) {
        // the poses: moments, coefficients, gradient and Gauss–Newton sums
        ok = cuda_ok(gn_hinv(H, n, d.sym, dh, st), "refine") &&
             cuda_ok(pose_moments(pa, pb, dh, n, sums, st, {}, act, rd), "refine") &&
             (!sym || cuda_ok(pose_moments(pb, pa, dh + (size_t)n * 9, n, sums + (size_t)n * kMom, st, {}, act, rd), "refine")) &&
             cuda_ok(pose_coefs(sums, (int)m, exact, coef, score, st), "refine") &&
             cuda_ok(pose_tangent(pa, pb, dh, coef, dg, n, true, tsum, st, {}, act, rd), "refine") &&
             (!sym || cuda_ok(pose_tangent(pb, pa, dh + (size_t)n * 9, coef + (size_t)n * kCoef, dg + 72, n, true,
                                           tsum + (size_t)n * kGrad, st, {}, act, rd),
                              "refine")) &&
             // the candidates, then their scores
             cuda_ok(gn_propose(d, ga, H, sums, score, tsum, act, cur, Ht, valid, st), "refine") &&
             cuda_ok(gn_hinv(Ht, (int)nt, d.sym, dh, st), "refine") &&
             cuda_ok(pose_moments(pa, pb, dh, (int)nt, sums, st, {}, valid, rd), "refine") &&
             (!sym ||
              cuda_ok(pose_moments(pb, pa, dh + nt * 9, (int)nt, sums + nt * kMom, st, {}, valid, rd), "refine")) &&
             cuda_ok(pose_coefs(sums, (int)mt, exact, coef, score, st), "refine") &&
             cuda_ok(gn_select(d, score, valid, Ht, H, cur, act, st), "refine");
        if (!ok) return false;
        counts[0] += 5 + 2 * nd + 2 + nd + 2;
        if ((it + 1) % kGnBatch != 0 || it + 1 == iters) continue;
        // stop once no pose moved in the last iteration
        if (!cuda_ok(cudaMemcpyAsync(hact, act, (size_t)n, cudaMemcpyDeviceToHost, st), "refine") ||
            !cuda_ok(cudaStreamSynchronize(st), "refine"))
            return false;
        counts[2]++, counts[3]++;
        if (std::none_of(hact, hact + n, [](unsigned char a) { return a != 0; })) break;
    }
    if (!cuda_ok(cudaMemcpyAsync(hH, H, (size_t)n * 9 * 8, cudaMemcpyDeviceToHost, st), "refine") ||
        !cuda_ok(cudaMemcpyAsync(hcur, cur, (size_t)n * 8, cudaMemcpyDeviceToHost, st), "refine") ||
        !cuda_ok(cudaStreamSynchronize(st), "refine"))
        return false;
    counts[1]++, counts[2] += 2, counts[3]++;
    out.resize(n);
    for (int i = 0; i < n; ++i) {
        for (int k = 0; k < 9; ++k) out[i].H[k] = hH[(size_t)i * 9 + k];
        out[i].score = hcur[i];
    }
    return true;
}

bool Engine::gn_batch(const std::vector<Mat3>& Hs, unsigned iters, const std::vector<double>& amps,
                      std::vector<ScoredPose>& cur) {
    // the device loop, unless a live spline moves the samples (its directions are per pose on the
    // host) or ZCMIR_B200_GN=host asks for the host loop
    const char* gv = std::getenv("ZCMIR_B200_GN");
    if (!(gv && std::string(gv) == "host") && !ffd_live() && amps.size() <= 16) return gn_batch_dev(Hs, iters, amps, cur);
    const bool homog = set.e("group") == "homography";
    const int nk = n_keys(homog);
    const double rw = side[1].w, rh = side[1].h;
    cur.clear();
    for (const Mat3& H : Hs) cur.push_back({H, -INFINITY});
    static const double mults[5] = {0.5, 1, 2, 4, 8};
    auto beats = [](double nw, double old) { return nw > old + std::max(1e-6 * std::fabs(old), 1e-12); };
    auto move = [&](const Mat3& H, const double* v, double a) {
        Coords x{};
        for (int k = 0; k < nk; ++k) x[k] = a * v[k];
        return composeN(H, x, homog, rw, rh);
    };
    std::vector<size_t> act(Hs.size());
    for (size_t i = 0; i < act.size(); ++i) act[i] = i;
    struct Try {
        size_t i;
        Mat3 H;
    };
    for (unsigned it = 0; it < iters && !cancel && !act.empty(); ++it) {
        std::vector<Mat3> hs;
        for (size_t i : act) hs.push_back(cur[i].H);
        std::vector<PoseEval> ev;
        if (!eval_poses(hs, true, true, ev)) return false;
        std::vector<Try> tries;
        for (size_t k = 0; k < act.size(); ++k) {
            const size_t i = act[k];
            const PoseEval& g = ev[k];
            cur[i].score = g.mean;
            if (!amps.empty()) {
                // the unit ascent direction (src/lie.zig unitAscent)
                double d[8] = {0}, n = 0;
                for (int q = 0; q < nk; ++q) d[q] = g.grad[q], n += d[q] * d[q];
                n = std::sqrt(n);
                if (n >= 1e-18)
                    for (int q = 0; q < nk; ++q) d[q] /= n;
                double dn = 0;
                for (int q = 0; q < nk; ++q) dn += d[q] * d[q];
                if (std::sqrt(dn) > 1e-12)
                    for (double a : amps) tries.push_back({i, move(cur[i].H, d, a)});
            }
            double Am[64], half[8], step[8];
            for (int q = 0; q < nk * nk; ++q) Am[q] = g.hess[q];
            for (int q = 0; q < nk; ++q) Am[q * nk + q] += 1e-4 * std::max(Am[q * nk + q], 1e-12);
            for (int q = 0; q < nk; ++q) half[q] = 0.5 * g.grad[q];
            if (!solve_linear(Am, half, nk, step)) continue;
            double nrm = 0;
            for (int q = 0; q < nk; ++q) nrm += step[q] * step[q];
            nrm = std::sqrt(nrm);
            for (double m : mults) {
                const double s = m * (nrm * m > 0.25 ? 0.25 / (nrm * m) : 1.0);
                tries.push_back({i, move(cur[i].H, step, s)});
            }
        }
        if (tries.empty()) break;
        std::vector<Mat3> th;
        for (const Try& t : tries) th.push_back(t.H);
        std::vector<PoseEval> sc;
        if (!eval_poses(th, false, false, sc)) return false;
        std::vector<char> moved(Hs.size(), 0);
        for (size_t k = 0; k < tries.size(); ++k)
            if (beats(sc[k].mean, cur[tries[k].i].score)) {
                cur[tries[k].i] = {tries[k].H, sc[k].mean};
                moved[tries[k].i] = 1;
            }
        std::vector<size_t> next;
        for (size_t i : act)
            if (moved[i]) next.push_back(i);
        act.swap(next);
    }
    return true;
}

void Engine::sweep_settings(SweepGrid& gv, int& G, Mat3& H0) {
    auto clampf = [](double x, double lo, double hi) { return std::min(hi, std::max(lo, x)); };
    const unsigned g = set.u("sw_grid");
    G = (g == 32 || g == 64 || g == 128 || g == 256) ? (int)g : 128;
    const double rot_deg = clampf(set.f("sw_rot"), 0, 180);
    // a span past 360° is clamped to one turn; an upper end below the lower one wraps through
    // ±180° (e.g. 170 to −170 covers 20° about 180°)
    const bool range = set.b("sw_rot_range");
    const double rot_lo = range ? clampf(set.f("sw_rot_lo"), -360, 360) : -rot_deg;
    double rot_hi = range ? clampf(set.f("sw_rot_hi"), -360, 360) : rot_deg;
    if (rot_hi < rot_lo) rot_hi += 360;
    rot_hi = std::min(rot_hi, rot_lo + 360);
    SweepGridOpts o;
    o.rot_lo = rot_lo, o.rot_hi = rot_hi;
    o.n_theta = std::clamp(set.u("sw_nth"), 1u, 720u);
    o.s_min = clampf(set.f("sw_smin"), 0.05, 1);
    o.s_max = clampf(set.f("sw_smax"), 1, 20);
    o.n_sigma = std::clamp(set.u("sw_ns"), 1u, 129u);
    o.shear_max = set.b("sw_shear") ? clampf(set.f("sw_shear_max"), 0, 1) : 0;
    o.n_shear = std::clamp(set.u("sw_nshear"), 1u, 15u);
    o.aniso_max = set.b("sw_aniso") ? clampf(set.f("sw_aniso_max"), 0, 1) : 0;
    o.n_aniso = std::clamp(set.u("sw_naniso"), 1u, 15u);
    gv = sweep_grid(o);
    const double lw = side[0].w, lh = side[0].h, rw = side[1].w, rh = side[1].h;
    H0 = set.b("sw_rel") ? H : translate((rw - lw) / 2, (rh - lh) / 2);
}

bool Engine::sweep_stack(const Mat3& H0, int n_peak, SweepOut& sw, zc_shift_result* stack_out, size_t n_out) {
    if (stack_jobs_.empty()) return fail("sweep_stack: load a stack first (zcb_stack_load)");
    if (!stack_out || n_out < stack_jobs_.size())
        return fail("sweep_stack: the stack's results need " + std::to_string(stack_jobs_.size()) + " entries");
    if (!branch_st_ && !cuda_ok(cudaStreamCreateWithFlags(&branch_st_, cudaStreamNonBlocking), "sweep_stack")) return false;
    for (cudaEvent_t* e : {&fork_ev_, &join_ev_})
        if (!*e && !cuda_ok(cudaEventCreateWithFlags(e, cudaEventDisableTiming), "sweep_stack")) return false;
    // the engine pair's builds joined and autocorrelations read: the capture may not wait on them
    if (!need_images() || !join_side(0) || !join_side(1) || !finish_acf()) return false;
    SweepGrid gv;
    int G;
    Mat3 Hd;
    sweep_settings(gv, G, Hd);
    (void)Hd;
    const double min_ov = std::min(0.5, std::max(0.0, set.f("min_overlap")));
    struct Flag {
        bool& f;
        explicit Flag(bool& x) : f(x) { f = true; }
        ~Flag() { f = false; }
    } with_stack(sweep_with_stack_);
    const bool ran = sweep_maps(H0, gv, G, set.b("exact"), n_peak, min_ov, sw, 0, 0, 1);
    forget_spectra();  // the stack's branch wrote the map path's canvas and spectrum buffers
    return ran && stack_collect(stack_out);
}

bool Engine::tune_sweep(double* out, size_t cap, size_t* used) {
    if (!search_check()) return false;
    SweepGrid gv;
    int G;
    Mat3 H0;
    sweep_settings(gv, G, H0);
    const bool exact = set.b("exact");
    const double min_ov = std::min(0.5, std::max(0.0, set.f("min_overlap")));
    const CorrPlanDev plan = corr_plan_dev(exact, side[0].mode == 1);
    SweepOut probe;
    if (!sweep_setup(H0, gv, G, probe)) return false;
    // the plane classes and what one candidate's work buffers take
    std::map<std::array<int, 2>, int> members;
    for (const SweepCand& c : probe.cands) members[{c.nx, c.ny}]++;
    auto per_item = [&](int nx, int ny) {
        const size_t pstride = (size_t)ny * pitch_of(nx);
        return (size_t)5 * (nx - probe.Fx + 1) * (ny - probe.Fy + 1) * 4 +
               (size_t)(plan.n_real + plan.n_corr) * pstride * 8 + (size_t)nx * ny * 4;
    };
    static const int kOptions[] = {16, 32, 64, 128, 256, 512, 1024, 2048};
    std::map<std::array<int, 2>, std::vector<std::pair<int, double>>> timed;  // class → (batch, ms per map)
    struct Restore {
        std::map<std::array<int, 2>, int>& f;
        ~Restore() { f.clear(); }
    } restore{sweep_force_};
    for (int b : kOptions) {
        sweep_force_.clear();
        bool any = false;
        for (const auto& kv : members) {
            const size_t cap_b = std::max<size_t>(1, kTuneBudget / per_item(kv.first[0], kv.first[1]));
            const int eb = (int)std::min<size_t>({(size_t)b, cap_b, (size_t)kv.second});
            sweep_force_[kv.first] = eb;
            const auto& seen = timed[kv.first];
            if (std::none_of(seen.begin(), seen.end(), [&](const std::pair<int, double>& p) { return p.first == eb; }))
                any = true;
        }
        if (!any) continue;
        SweepOut r;
        // one untimed run (buffers, caches), then the timed one
        if (!sweep_maps(H0, gv, G, exact, 4, min_ov, r) || !sweep_maps(H0, gv, G, exact, 4, min_ov, r)) return false;
        for (const auto& c : r.classes) {
            const std::array<int, 2> key{(int)c[0], (int)c[1]};
            auto& seen = timed[key];
            if (std::none_of(seen.begin(), seen.end(), [&](const std::pair<int, double>& p) { return p.first == (int)c[3]; }))
                seen.push_back({(int)c[3], c[4] / std::max(1.0, c[2])});
        }
    }
    size_t n = 0;
    auto put = [&](double v) {
        if (out && n < cap) out[n] = v;
        ++n;
    };
    std::string msg = "tune_sweep";
    for (const auto& kv : timed) {
        if (kv.second.empty()) continue;
        const auto best = *std::min_element(kv.second.begin(), kv.second.end(),
                                            [](const std::pair<int, double>& a, const std::pair<int, double>& b) {
                                                return a.second < b.second;
                                            });
        sweep_tuned_[{kv.first[0], kv.first[1], plan.n_corr, exact ? 1 : 0}] = best.first;
        put(kv.first[0]), put(kv.first[1]), put(members[kv.first]), put(best.first), put(best.second);
        put((double)kv.second.size());
        for (const auto& p : kv.second) put(p.first), put(p.second);
        char b[96];
        snprintf(b, sizeof b, "  %d×%d: batch %d (%.4f ms per map)", kv.first[0], kv.first[1], best.first, best.second);
        msg += b;
    }
    log_event(msg);
    if (used) *used = n;
    return true;
}

bool Engine::search_check() {
    if (!need_images()) return false;
    if (set.e("search_mode") != "sweep")
        return fail("search: search_mode \"" + set.e("search_mode") + "\" is not part of this build (search_mode=\"sweep\" is)");
    if (set.e("metric") == "ncc") return fail("search: SweepNeedsMomentScore (the sweep scores SMI moments; metric \"ncc\" has none)");
    if (!metric_ok("search")) return false;
    return true;
}

bool Engine::search(zc_search_result* out) {
    if (!search_check()) return false;
    SweepGrid gv;
    int G;
    Mat3 H0;
    sweep_settings(gv, G, H0);
    const double min_ov = std::min(0.5, std::max(0.0, set.f("min_overlap")));
    SweepOut res;
    if (!sweep_maps(H0, gv, G, set.b("exact"), 4, min_ov, res)) return false;
    return search_finish(res, gv, H0, out);
}

bool Engine::match_by_sweep(zc_match_result* out) {
    if (!need_images()) return false;
    // a keypoint fit has no prior: start from the images' centres aligned
    const double lw = side[0].w, lh = side[0].h, rw = side[1].w, rh = side[1].h;
    H = translate((rw - lw) / 2, (rh - lh) / 2);
    const std::string mode = set.e("search_mode");
    std::string err;
    if (mode != "sweep") {
        const char* js = "{\"search_mode\":\"sweep\"}";
        set.apply(js, strlen(js), err);
    }
    log_event("match  no keypoint matcher in this build: the SMI sweep search fits the pose");
    zc_search_result r{};
    const bool ok = search(&r);
    if (mode != "sweep") {
        const std::string back = "{\"search_mode\":\"" + mode + "\"}";  // an enum tag: no escaping
        set.apply(back.c_str(), back.size(), err);
    }
    if (!ok) return false;
    zc_match_result m{};
    std::memcpy(m.H, H.data(), sizeof m.H);
    *out = m;
    return true;
}

bool Engine::search_lanes(const float* scores, const uint32_t* idx, size_t n, zc_search_result* out) {
    if (!search_check()) return false;
    SweepGrid gv;
    int G;
    Mat3 H0;
    sweep_settings(gv, G, H0);
    SweepOut res;
    if (!sweep_setup(H0, gv, G, res)) return false;
    const size_t need = res.cands.size() * 4;
    if (n != need || !scores || !idx)
        return fail("search_lanes: " + std::to_string(n) + " lane entries for " + std::to_string(res.cands.size()) +
                    " candidates × 4 (the sweep settings must match the sweep's)");
    res.lane_score.assign(scores, scores + n);
    res.lane_idx.assign(idx, idx + n);
    sweep_make_peaks(res, 4);
    return search_finish(res, gv, H0, out);
}

bool Engine::search_finish(const SweepOut& res, const SweepGrid& gv, const Mat3& H0, zc_search_result* out) {
    cancel = false;
    const int G = res.G;
    const unsigned kk = set.u("sw_k");
    const unsigned K = (kk == 8 || kk == 16 || kk == 32) ? kk : 32;
    const unsigned n_fin = std::clamp(set.u("sw_fin"), 1u, 16u);
    const Mat3 Hcur = H;
    const double c_mov[2] = {(side[0].w + 1) / 2.0, (side[0].h + 1) / 2.0};
    std::vector<PoseEval> e0;
    if (!eval_poses({Hcur}, false, false, e0)) return false;  // with the live spline
    const double s_cur = e0[0].mean;
    // the spline is off while the sweep's peaks climb (src/search.zig:703-705, 806-810)
    const bool ffd_was = set.b("ffd");
    struct Suspend {
        bool& f;
        explicit Suspend(bool& x) : f(x) { f = true; }
        ~Suspend() { f = false; }
    } suspend(ffd_suspended_);
    const bool exact = set.b("exact");
    const std::vector<SweepPeak> top = nms4(res.peaks, (unsigned)gv.thetas.size(), K, gv.wrap);
    char buf[320];
    snprintf(buf, sizeof buf, "search  %zuθ × %zuσ%s  %d maps  %d² grid (%.1f px, FFT ≤ %d²)  %s  %zu peaks  (%.2f ms)",
             gv.thetas.size(), gv.sigmas.size(), gv.shears.size() * gv.anisos.size() > 1 ? " × shear × stretch" : "",
             (int)res.cands.size(), G, res.cell, res.n, exact ? "exact" : "global", top.size(), res.ms);
    log_event(buf);
    zc_search_result r{};
    std::memcpy(r.H, Hcur.data(), sizeof r.H);
    r.score = s_cur;
    r.prev = s_cur;
    r.count_a = (uint32_t)top.size();
    if (top.empty()) {
        log_event("search  no peak above the overlap floor");
        *out = r;
        return true;
    }
    const std::vector<double> amps =
        geo_amps(set.f("g_a0"), set.f("g_decay"), set.u("g_steps") > 0 ? set.u("g_steps") : 7);
    std::vector<Mat3> starts;
    for (const SweepPeak& p : top) starts.push_back(p.H);
    std::vector<ScoredPose> screened;
    if (!gn_batch(starts, 4, amps, screened)) return false;
    // finalists: the best after the short climb, plus the best coarse peaks
    std::vector<size_t> order(screened.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return screened[a].score > screened[b].score; });
    std::vector<size_t> fin;
    for (size_t k = 0; k < std::min<size_t>(n_fin, order.size()); ++k)
        if (std::find(fin.begin(), fin.end(), order[k]) == fin.end()) fin.push_back(order[k]);
    for (size_t i = 0; i < std::min<size_t>(n_fin, top.size()); ++i)
        if (std::find(fin.begin(), fin.end(), i) == fin.end()) fin.push_back(i);
    std::vector<Mat3> fin_h;
    for (size_t i : fin) fin_h.push_back(screened[i].H);
    std::vector<ScoredPose> finals;
    if (!gn_batch(fin_h, 25, amps, finals)) return false;
    size_t bi = 0;
    for (size_t i = 0; i < finals.size(); ++i)
        if (finals[i].score > finals[bi].score) bi = i;
    const ScoredPose best = finals[bi];
    const auto rs = sim_of(best.H, H0, c_mov[0], c_mov[1]);
    snprintf(buf, sizeof buf, "search  screen %zu × 4 steps, climb %zu × ≤25 Gauss–Newton  best nS %.1f", top.size(),
             finals.size(), best.score);
    log_event(buf);
    r.count_b = (uint32_t)finals.size();
    auto beats = [](double nw, double old) { return nw > old + std::max(1e-6 * std::fabs(old), 1e-12); };
    if (beats(best.score, s_cur)) {
        H = best.H;
        std::memcpy(r.H, best.H.data(), sizeof r.H);
        r.score = best.score;
        r.improved = 1;
        if (ffd_was) std::fill(ffd_cps_.begin(), ffd_cps_.end(), 0.f);  // the spline starts over at the new pose
        snprintf(buf, sizeof buf, "search done  nS %.1f (was %.1f)  θ %.1f° σ %.3f%s", best.score, s_cur,
                 rs[0] * 180 / M_PI, rs[1], ffd_was ? "  spline reset" : "");
    } else {
        snprintf(buf, sizeof buf, "search done  kept the current pose (nS %.1f ≥ %.1f)", s_cur, best.score);
    }
    log_event(buf);
    *out = r;
    return true;
}

}  // namespace zc
