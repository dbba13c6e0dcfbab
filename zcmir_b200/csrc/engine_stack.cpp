// Shift maps along a stack of slices (serial sections, time series).
//
// The reference's register_stack (python/zcmir/api.py:522-580) registers slice pair by slice pair,
// each call uploading both images again and rebuilding their features. Here the slices' features
// are built once each on the device, then one shift map per consecutive pair — slice k moving,
// slice k − 1 fixed, at a prior pose — runs on the engine's stream with its result key copied
// device to device, and all results are read back once at the end.
#include <algorithm>
#include <cstring>
#include <utility>

#include "engine.hpp"

namespace zc {

bool Engine::stack_maps(int n, const float* const* images, const int* ws, const int* hs, const Mat3* priors,
                        bool exact, bool calibrated, unsigned cap, zc_shift_result* out, float* ms) {
    if (n < 2) return fail("stack_maps: a stack needs at least 2 slices");
    if (!images || !ws || !hs || !out) return fail("stack_maps: null argument");
    for (int i = 0; i < n; ++i)
        if (!images[i] || ws[i] < 8 || hs[i] < 8) return fail("stack_maps: BadImage (slice " + std::to_string(i) + ")");
    if ((int)stack_.size() < n) stack_.resize(n);
    if (!cuda_ok(stack_res_.ensure((size_t)(n - 1) * 24), "stack_maps")) return false;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    auto done = [&](bool r) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        return r;
    };
    cudaEventRecord(e0, st);
    // every slice's features, once (the current settings: feature mode, f16 input)
    for (int i = 0; i < n; ++i) {
        SideSwap sw(side[0], stack_[i]);
        if (!set_image(0, images[i], ws[i], hs[i], false)) return done(false);
    }
    std::vector<MapJob> jobs(n - 1);
    std::vector<double> areas(n - 1);
    for (int k = 1; k < n; ++k) {
        SideSwap mv(side[0], stack_[k]);
        SideSwap fx(side[1], stack_[k - 1]);
        // default prior: the slices' centres aligned
        const Mat3 H = priors ? priors[k - 1] : translate((ws[k - 1] - ws[k]) / 2.0, (hs[k - 1] - hs[k]) / 2.0);
        MapJob& job = jobs[k - 1];
        if (!plan_map(H, exact, calibrated, cap == 0 ? kMapCap : cap, 0.0, job)) return done(false);
        if (!run_map(job, nullptr)) return done(false);
        if (!cuda_ok(cudaMemcpyAsync(stack_res_.as<unsigned char>() + (size_t)(k - 1) * 24, res_.p, 24,
                                     cudaMemcpyDeviceToDevice, st),
                     "stack_maps"))
            return done(false);
        areas[k - 1] = pair_area();
    }
    cudaEventRecord(e1, st);
    std::vector<unsigned char> host((size_t)(n - 1) * 24);
    if (!cuda_ok(cudaMemcpyAsync(host.data(), stack_res_.p, host.size(), cudaMemcpyDeviceToHost, st), "stack_maps") ||
        !cuda_ok(cudaStreamSynchronize(st), "stack_maps"))
        return done(false);
    counts[1]++;
    counts[2]++;
    counts[3]++;
    if (ms) cudaEventElapsedTime(ms, e0, e1);
    for (int k = 0; k < n - 1; ++k) {
        unsigned long long best;
        float zero;
        std::memcpy(&best, host.data() + (size_t)k * 24, 8);
        std::memcpy(&zero, host.data() + (size_t)k * 24 + 8, 4);
        map_result(jobs[k], best, zero, areas[k], &out[k]);
    }
    return done(true);
}

}  // namespace zc
