// Shift maps along a stack of slices (serial sections, time series).
//
// The reference's register_stack (python/zcmir/api.py:522-580) registers slice pair by slice pair,
// each call uploading both images again and rebuilding their features. Here the slices' features
// are built once each on the device, then one shift map per consecutive pair — slice k moving,
// slice k − 1 fixed, at a prior pose — runs on the engine's stream with its result key copied
// device to device, and all results are read back once at the end.
//
// In parts (stack_load, stack_enqueue, stack_collect) the maps can also be captured into a CUDA
// graph beside the sweep's (Engine::sweep_stack): stack_load leaves nothing pending — every build
// joined, every autocorrelation read, every buffer the maps use allocated — so stack_enqueue
// only queues kernels and device copies.
#include <algorithm>
#include <cstring>
#include <utility>

#include "engine.hpp"

namespace zc {

bool Engine::stack_load(int n, const float* const* images, const int* ws, const int* hs, const Mat3* priors,
                        bool exact, bool calibrated, unsigned cap) {
    stack_jobs_.clear();
    stack_areas_.clear();
    ++stack_gen_;
    if (n < 2) return fail("stack_maps: a stack needs at least 2 slices");
    if (!images || !ws || !hs) return fail("stack_maps: null argument");
    for (int i = 0; i < n; ++i)
        if (!images[i] || ws[i] < 8 || hs[i] < 8) return fail("stack_maps: BadImage (slice " + std::to_string(i) + ")");
    if ((int)stack_.size() < n) stack_.resize(n);
    if (!cuda_ok(stack_res_.ensure((size_t)(n - 1) * 24), "stack_maps")) return false;
    // every slice's features, once (the current settings: feature mode, f16 input)
    for (int i = 0; i < n; ++i) {
        SideSwap sw(side[0], stack_[i]);
        if (!set_image(0, images[i], ws[i], hs[i], false)) return false;
    }
    std::vector<MapJob> jobs(n - 1);
    std::vector<double> areas(n - 1);
    for (int k = 1; k < n; ++k) {
        SideSwap mv(side[0], stack_[k]);
        SideSwap fx(side[1], stack_[k - 1]);
        // both slices built and their autocorrelations read (the correlation area of the pair)
        if (!join_side(0) || !join_side(1) || !finish_acf()) return false;
        // default prior: the slices' centres aligned
        const Mat3 H = priors ? priors[k - 1] : translate((ws[k - 1] - ws[k]) / 2.0, (hs[k - 1] - hs[k]) / 2.0);
        MapJob& job = jobs[k - 1];
        if (!plan_map(H, exact, calibrated, cap == 0 ? kMapCap : cap, 0.0, job) || !map_buffers(job)) return false;
        areas[k - 1] = pair_area();
    }
    stack_jobs_ = std::move(jobs);
    stack_areas_ = std::move(areas);
    return true;
}

int Engine::stack_enqueue() {
    if (stack_jobs_.empty()) {
        fail("stack_maps: no stack loaded");
        return -1;
    }
    const uint32_t launches0 = counts[0];
    // the slices' spectra are never kept across pairs (each pair's fixed slice was the moving
    // one of the pair before, in the other buffers)
    const bool cache_off = spectra_cache_off_;
    spectra_cache_off_ = true;
    bool ok = true;
    for (size_t k = 1; ok && k <= stack_jobs_.size(); ++k) {
        SideSwap mv(side[0], stack_[k]);
        SideSwap fx(side[1], stack_[k - 1]);
        ok = run_map(stack_jobs_[k - 1], nullptr) &&
             cuda_ok(cudaMemcpyAsync(stack_res_.as<unsigned char>() + (k - 1) * 24, res_.p, 24, cudaMemcpyDeviceToDevice,
                                     st),
                     "stack_maps");
    }
    spectra_cache_off_ = cache_off;
    forget_spectra();  // the map buffers now hold the last pair's spectra, not the engine pair's
    return ok ? (int)(counts[0] - launches0) : -1;
}

bool Engine::stack_collect(zc_shift_result* out) {
    const size_t m = stack_jobs_.size();
    std::vector<unsigned char> host(m * 24);
    if (!cuda_ok(cudaMemcpyAsync(host.data(), stack_res_.p, host.size(), cudaMemcpyDeviceToHost, st), "stack_maps") ||
        !cuda_ok(cudaStreamSynchronize(st), "stack_maps"))
        return false;
    counts[1]++;
    counts[2]++;
    counts[3]++;
    for (size_t k = 0; k < m; ++k) {
        unsigned long long best;
        float zero;
        std::memcpy(&best, host.data() + k * 24, 8);
        std::memcpy(&zero, host.data() + k * 24 + 8, 4);
        map_result(stack_jobs_[k], best, zero, stack_areas_[k], &out[k]);
    }
    return true;
}

bool Engine::stack_maps(int n, const float* const* images, const int* ws, const int* hs, const Mat3* priors,
                        bool exact, bool calibrated, unsigned cap, zc_shift_result* out, float* ms) {
    if (!out) return fail("stack_maps: null argument");
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    auto done = [&](bool r) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        return r;
    };
    cudaEventRecord(e0, st);
    if (!stack_load(n, images, ws, hs, priors, exact, calibrated, cap) || stack_enqueue() < 0) return done(false);
    cudaEventRecord(e1, st);
    if (!stack_collect(out)) return done(false);
    if (ms) cudaEventElapsedTime(ms, e0, e1);
    return done(true);
}

}  // namespace zc
