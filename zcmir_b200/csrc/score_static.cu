// Pose scores without device allocation: zcb_score_static.
//
// The same kernels as zc_score (the overlap moments of pose.cu, then the float64 score per
// direction), but every device buffer of the call lives in one file-scope array, so a call
// allocates no device memory. zc_score grows its pose buffers with cudaMalloc (and frees the old
// ones) on its first call and whenever a call scores more poses than any before it. Callers that
// cannot allow that:
//   - a host that scores poses while its other streams keep the GPU busy: cudaFree waits for the
//     whole device, so a growth step would stall every stream of the process;
//   - a host that hands the GPU's free memory to its own pool at start-up: an allocation in the
//     middle of a run can then fail.
//
// Limits: at most kMaxPoses = 64 poses per call; the array holds 103,936 bytes of device memory
// for the life of the process. The array is shared by every engine on a device, so calls that
// overlap in time (two threads, or two engines) race on it, and it keeps the last call's
// contents. The feature planes must already be built for the current settings (zc_score,
// zc_features and zc_set_image_gray build them); building them allocates, so this call refuses
// rather than build.
//
// Set-up: the array's device address is looked up with cudaGetSymbolAddress, with the device
// current, once per device. zc_create does this for its device, so the first call of an engine
// made there needs no set-up; only an engine whose device was never set up (its look-up at
// creation failed) does it on its first call, which should then come before any stream capture
// begins. With lazy module loading (the CUDA 12 default) the look-up is what loads the module that
// holds the array, and so what reserves its 103,936 bytes on the device: at creation, not in a
// call.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "engine.hpp"
#include "kernels.hpp"

namespace {

constexpr int kMaxPoses = 64;
constexpr int kRows = 2 * kMaxPoses;  // both directions when the score is symmetric
constexpr int kMom = 45, kCoef = 102;

constexpr size_t align256(size_t b) { return (b + 255) & ~size_t(255); }
constexpr size_t kHinvOff = 0;                                                       // f32 [rows][9]
constexpr size_t kSumsOff = kHinvOff + align256(kRows * 9 * sizeof(float));          // f64 [rows][45]
constexpr size_t kCoefOff = kSumsOff + align256(kRows * kMom * sizeof(double));       // f32 [rows][102]
constexpr size_t kScoreOff = kCoefOff + align256(kRows * kCoef * sizeof(float));      // f64 [rows]
constexpr size_t kScratchBytes = kScoreOff + align256(kRows * sizeof(double));
static_assert(kScratchBytes == 103936, "the stated size of the scratch array");

}  // namespace

static __device__ __align__(256) unsigned char g_score_scratch[kScratchBytes];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
unsigned char* g_scratch_ptr[kMaxDevices];

// The array's address on device `dev`, looked up on the first call for that device.
cudaError_t scratch_on(int dev, unsigned char** out) {
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_ptr[dev]) {
        int cur = -1;
        cudaError_t e = cudaGetDevice(&cur);
        if (e != cudaSuccess) return e;
        if (cur != dev && (e = cudaSetDevice(dev)) != cudaSuccess) return e;
        unsigned char* ptr = nullptr;
        e = cudaGetSymbolAddress((void**)&ptr, g_score_scratch);
        if (cur != dev) cudaSetDevice(cur);
        if (e != cudaSuccess) return e;
        g_scratch_ptr[dev] = ptr;
    }
    *out = g_scratch_ptr[dev];
    return cudaSuccess;
}

}  // namespace

namespace zc {

// Called by zc_create for the engine's device: looks the array up (and so loads its module)
// before any call needs it. A failure here is not fatal; the first call retries and reports it.
void static_scratch_setup(int dev) {
    unsigned char* p = nullptr;
    (void)scratch_on(dev, &p);
}

bool Engine::score_static(const double* Hs, uint32_t n_poses, double* out3) {
    if (n_poses > (uint32_t)kMaxPoses)
        return fail("score_static: " + std::to_string(n_poses) + " poses exceed the static scratch's maximum of " +
                    std::to_string(kMaxPoses) + " per call; score them in chunks of at most " +
                    std::to_string(kMaxPoses));
    const int n = (int)n_poses;
    if (n > 0 && (!Hs || !out3)) return fail("score_static: null poses or output");
    if (!side[0].has || !side[1].has) return fail("NoImages");
    if (set.e("metric") != "smi")
        return fail("score_static: metric \"" + set.e("metric") + "\" is not part of this build's SMI path");
    if (ffd_live()) return fail("score_static: the spline is live; its scores come from zc_score");
    const std::string& fm = set.e("smi_features");
    const int mode = fm == "laplacian" ? 0 : (fm == "three" ? 1 : 2);
    for (const Side& sd : side)
        if (!sd.built || sd.mode != mode || sd.half != set.b("half") || (sd.preprocess && sd.bake != bake_key()))
            return fail(
                "score_static: the feature planes are not built for the current settings; building them "
                "allocates device memory, so call zc_score or zc_features once first");
    // A side whose build ran on a stream of its own (side 1 after zc_set_image_gray) may still be
    // writing its planes: the engine stream waits for that build's event. Only stream waits are
    // issued here, nothing is allocated.
    if (!join_side(0) || !join_side(1)) return false;
    if (n == 0) return true;
    unsigned char* base = nullptr;
    if (!cuda_ok(scratch_on(device, &base), "score_static: scratch set-up")) return false;
    float* hinv = reinterpret_cast<float*>(base + kHinvOff);
    double* sums = reinterpret_cast<double*>(base + kSumsOff);
    float* coef = reinterpret_cast<float*>(base + kCoefOff);
    double* score = reinterpret_cast<double*>(base + kScoreOff);

    const bool sym = set.b("symmetric"), exact = set.b("exact");
    const int m = (sym ? 2 : 1) * n;
    // inverse poses: the forward direction samples the moving image at H⁻¹x, the inverse
    // direction (pose H⁻¹) the fixed image at Hx
    float hh[kRows * 9];
    for (int i = 0; i < n; ++i) {
        Mat3 H;
        for (int k = 0; k < 9; ++k) H[k] = Hs[(size_t)i * 9 + k];
        const Mat3 Hi = inv3(H);
        for (int k = 0; k < 9; ++k) hh[i * 9 + k] = (float)Hi[k];
        if (sym) {
            const Mat3 Hii = inv3(Hi);
            for (int k = 0; k < 9; ++k) hh[(n + i) * 9 + k] = (float)Hii[k];
        }
    }
    if (!cuda_ok(cudaMemcpyAsync(hinv, hh, (size_t)m * 9 * sizeof(float), cudaMemcpyHostToDevice, st), "score_static"))
        return false;
    const PoseSide pa{side[0].feat.as<float>(), side[0].feat4.as<float4>(), side[0].w, side[0].h},
        pb{side[1].feat.as<float>(), side[1].feat4.as<float4>(), side[1].w, side[1].h};
    // The moment sums accumulate with atomics and are the only part of the array that must
    // start at zero: pose_moments clears its n × 45 sums on the stream before accumulating. The
    // inverse poses, coefficients and scores are written in full before they are read.
    if (!cuda_ok(pose_moments(pa, pb, hinv, n, sums, st), "score_static")) return false;
    if (sym && !cuda_ok(pose_moments(pb, pa, hinv + (size_t)n * 9, n, sums + (size_t)n * kMom, st), "score_static"))
        return false;
    if (!cuda_ok(pose_coefs(sums, m, exact, coef, score, st), "score_static")) return false;
    double sc[kRows];
    if (!cuda_ok(cudaMemcpyAsync(sc, score, (size_t)m * sizeof(double), cudaMemcpyDeviceToHost, st), "score_static") ||
        !cuda_ok(cudaStreamSynchronize(st), "score_static"))
        return false;
    counts[0] += (sym ? 2 : 1) + 1;  // launches, submits, reads, waits
    counts[1]++;
    counts[2]++;
    counts[3]++;
    // per pose as zc_score writes it: the mean, the forward score and the inverse one (NaN when
    // the score is not symmetric)
    auto fin = [](double v) { return std::isfinite(v) ? v : 0.0; };
    for (int i = 0; i < n; ++i) {
        const double fwd = fin(sc[i]), inv = sym ? fin(sc[n + i]) : 0.0;
        out3[(size_t)i * 3 + 0] = sym ? 0.5 * (fwd + inv) : fwd;
        out3[(size_t)i * 3 + 1] = fwd;
        out3[(size_t)i * 3 + 2] = sym ? inv : std::nan("");
    }
    return true;
}

}  // namespace zc
