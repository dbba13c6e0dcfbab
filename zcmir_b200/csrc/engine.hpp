// The B200 SMI engine behind the zc_* C ABI: two images with their resident features, the pose,
// the settings, and the shift-map schedule on one CUDA stream.
#pragma once

#include <cuda_runtime.h>

#include <array>
#include <deque>
#include <map>
#include <string>
#include <utility>
#include <vector>

#include "../../include/zcmir.h"
#include "geom.hpp"
#include "kernels.hpp"
#include "settings.hpp"
#include "sweep.hpp"

namespace zc {

// A device allocation that grows on demand (never shrinks until release).
struct DevBuf {
    void* p = nullptr;
    size_t cap = 0;
    uint64_t gen = 0;  // bumped by every (re)allocation: contents from before it are gone
    cudaError_t ensure(size_t bytes);
    void release();
    template <class T>
    T* as() const {
        return static_cast<T*>(p);
    }
};

// Page-locked host memory that grows on demand, for copies the copy engines run straight from
// or into host memory (no staging pass). Regrown only while no copy into it is pending.
struct PinnedBuf {
    void* p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t bytes) {
        if (bytes <= cap) return cudaSuccess;
        release();
        const cudaError_t e = cudaMallocHost(&p, bytes);
        if (e == cudaSuccess) cap = bytes;
        else p = nullptr;
        return e;
    }
    void release() {
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
    }
    template <class T>
    T* as() const {
        return static_cast<T*>(p);
    }
};

struct Side {
    bool has = false;
    int w = 0, h = 0;
    bool preprocess = false;
    DevBuf raw;    // the image as uploaded (f32 gray)
    DevBuf work;   // the work image the features are built from (f16-quantised when half)
    DevBuf feat;   // 4 whitened planes, plane-major
    DevBuf feat4;  // the same, interleaved: one float4 per pixel (the pose kernels' bilinear taps)
    DevBuf mag;    // Sobel magnitude of the rank
    DevBuf stack;  // [1, f0..f3]
    std::array<double, 1156> acf{};  // normalised autocorrelation, 289 lags × 4 planes
    DevBuf acf_dev;                  // its raw sums on the device
    double* acf_host = nullptr;      // pinned copy of those sums, made on the build's stream
    cudaEvent_t acf_ev = nullptr;    // recorded after that copy
    bool acf_pending = false;        // acf_host holds (or will hold) sums that acf does not yet
    cudaEvent_t built_ev = nullptr;  // recorded after the last build, which read `raw`
    bool join_pending = false;       // built on a stream of its own; the engine stream has not yet waited
    bool built = false;
    int mode = -1;
    bool half = false;
    std::string bake;  // the preprocessing settings the work image was made with
    uint64_t ver = 0;  // which build the feature planes come from (unique per engine)
};

// Scores (and optionally the symmetric gradient and Gauss–Newton matrix) at one pose.
struct PoseEval {
    double fwd = 0, inv = 0, mean = 0, n = 0;  // scores; n: the forward overlap
    bool has_inv = false, has_grad = false, has_hess = false;
    std::array<double, 45> sums{};             // the forward direction's moment sums
    std::array<double, 8> grad{};              // over the group's tangent coordinates
    std::array<double, 64> hess{};             // nk × nk
};

// One map's plan and device-side description.
struct MapJob {
    Frame fr;
    Mat3 Hc;
    MapGeom g;
    CorrPlanDev plan;
    LinePlan row, col, line;
    int S;
    CombineParams cp;  // cp.area set when the row pass is launched
    double gcell = 1.0;  // canvas pixels per grid cell
    bool identity_grid;
    bool exact, calibrated;
};

// One candidate of the sweep with its window on the sweep canvas (src/search.zig:340-366).
struct SweepCand {
    int it, is, ik, ia;
    double th, s;
    Mat3 H;
    int gx0, gy0, nx, ny;  // first window cell, plane size
    float taps;
};

// The sweep's batched maps reduced to peaks (src/search.zig SweepOut).
struct SweepOut {
    std::vector<SweepCand> cands;       // θ-major, then σ, shear, stretch
    std::vector<SweepPeak> peaks;       // slot order (by plane size), then rank
    std::vector<float> best;            // each candidate's top score, fixed pixels
    std::vector<int> perm;              // slot order: candidates by plane size (stable)
    std::vector<float> lane_score;      // [nc][n_peak] lane maxima per candidate, fixed pixels
    std::vector<uint32_t> lane_idx;     // their map indices (0xffffffff: none)
    double cell = 0, ox = 0, oy = 0;
    int G = 0, fx0 = 0, fy0 = 0, Fx = 0, Fy = 0, n = 0;
    unsigned min_n = 0;
    int groups = 0, batches = 0, launches = 0;
    float ms = 0;                       // device time of the maps (CUDA events)
    // per plane class (slot order): nx, ny, candidates, batch, device ms (stream-ordered runs only)
    std::vector<std::array<double, 5>> classes;
    bool graph = false;                 // the maps were one replay of a captured CUDA graph
};

// A pose and its score (the batched Gauss–Newton screen).
struct ScoredPose {
    Mat3 H;
    double score;
};

// The correlation plan for exact (15 planes) or global (5) scores, without the fourth feature's
// planes when `three` (src/smi.zig:90-158).
CorrPlanDev corr_plan_dev(bool exact, bool three);

// One direction's roto-scale map plan (src/smi.zig RsPlan).
struct RsPlan {
    int n = 0, n_th = 0, n_lam = 0;
    double log0 = 0, span = 0, dlam = 0, dth = 0, r0 = 0, r1 = 0, cx = 0, cy = 0;
};

// Swaps two sides for the life of the object (the map code works on side[0], side[1]).
struct SideSwap {
    Side& a;
    Side& b;
    SideSwap(Side& x, Side& y) : a(x), b(y) { std::swap(a, b); }
    ~SideSwap() { std::swap(a, b); }
};

// Stages of a map timed by the profiler / the benchmark entry point.
enum Stage { kCanvas = 0, kFwdRows, kFwdCols, kInvCols, kInvRows, kNumStages };
extern const char* const kStageNames[kNumStages];

// Looks up zcb_score_static's file-scope device array on device dev (score_static.cu); zc_create
// calls it once per engine, so the calls themselves reserve nothing.
void static_scratch_setup(int dev);

class Engine {
  public:
    explicit Engine(int device);
    ~Engine();

    Settings set;
    Mat3 H = mat_identity();
    Side side[2];
    std::string err;
    bool cancel = false;
    std::deque<std::string> events;

    int device = 0;
    cudaDeviceProp prop{};
    cudaStream_t st = nullptr;
    cudaStream_t copy_st_ = nullptr;  // copies that overlap kernels: image uploads, map row chunks
    cudaEvent_t up_ev_ = nullptr;     // an image upload done
    static constexpr int kChunkEvents = 16;
    cudaEvent_t chunk_ev_[kChunkEvents] = {};

    // counters since the last zc_gpu_counts: launches, submits, reads, waits
    uint32_t counts[4] = {0, 0, 0, 0};
    bool profiling = false;
    // the last pass: "tmem" (sums in tensor memory, whole rows) or "split" (rows split S ways,
    // sums in shared memory); from ZCMIR_B200_ROW_PASS at creation, "tmem" by default
    std::string row_pass = "tmem";
    std::map<std::string, std::pair<double, uint32_t>> prof;  // name → (ms, count)

    bool fail(const std::string& m);
    bool cuda_ok(cudaError_t e, const char* what);

    // images and features
    bool set_image(int s, const float* data, int w, int h, bool preprocess);
    // RGBA8 → gray (0.299 R + 0.587 G + 0.114 B), always preprocessed (src/engine.zig:422-426)
    bool set_image_rgba(int s, const unsigned char* rgba, int w, int h);
    bool need_images();
    // both sides present and their features built (enqueued) for the current settings; with
    // join, the engine stream also waits for the builds made on a stream of their own
    bool need_built(bool join = true);
    // the engine stream waits for side s's build, if it ran on a stream of its own
    bool join_side(int s);
    // the sides' autocorrelations as their builds copied them back (a wait on each pending
    // side's copy only), normalised
    bool finish_acf();
    bool features(int s, float* out, size_t len);
    bool work_image(int s, float* out, size_t len);
    double pair_area() const;

    // maps
    bool plan_map(const Mat3& H, bool exact, bool calibrated, unsigned cap, double min_overlap, MapJob& job);
    // host_map (nullable): with the tensor-memory row pass, the map is copied there in row
    // chunks on the copy stream during the pass (the caller synchronises copy_st_)
    bool run_map(MapJob& job, cudaEvent_t* ev /* kNumStages+1 events or null */, float* host_map = nullptr);
    bool shift_map(const Mat3& H, bool exact, bool calibrated, unsigned cap, double min_overlap, zc_shift_result* out,
                   float* map, size_t map_len);
    bool shift_map_settings(const Mat3& H, zc_shift_result* out, float* map, size_t map_len);
    // a map's result from its best key (score bits, inverted index), zero-lag score and the
    // pair's correlation area
    void map_result(const MapJob& job, unsigned long long best, float zero, double area, zc_shift_result* out);
    // roto-scale map (engine_rs.cpp): pose H about c (fixed pixels, 1-based; null: the moving
    // image's centroid under H); symmetric: with the inverse-frame map. Optional host outputs
    // (len ≥ n²): the finished map, the raw forward and inverse maps.
    bool rs_map(const Mat3& H, const double* c, bool symmetric, zc_rs_result* out, float* map, float* fwd, float* inv,
                size_t len);
    // the one-sided roto-scale map's peak at H about c as the rotation (rad) and log scale
    // that correct the pose (the climb's roto-scale hop)
    bool rs_peak(const Mat3& H, const double c[2], double* dth, double* dsg);
    // the moving image's centroid under H: the mean of its four mapped corners (src/lie.zig
    // movingCentroid), the roto-scale map's default centre
    void rs_center(const Mat3& H, double c[2]) const;
    bool rs_map_one(const Mat3& H, const double c[2], double r0, double r1, bool exact, bool calibrated, unsigned cap,
                    DevBuf& dst, RsPlan& p);
    // the NCC overlay metric (engine_ncc.cpp): the zero-lag NCC of the pair's union canvas at H,
    // and the NCC of every shift as a map; zc_score and zc_shift_map return these when the
    // settings' metric is "ncc"
    bool ncc_score(const Mat3& H, double* out);
    bool ncc_shift_map(const Mat3& H, zc_shift_result* out, float* map, size_t map_len);
    // fails unless the settings' metric is one this build has: "smi", or "ncc" (whose pose
    // gradients, climb, sweep-free maps and roto-scale maps are SMI's, as in the reference)
    bool metric_ok(const char* what);
    // maps along a stack (engine_stack.cpp): each slice's features once, then slice k (moving)
    // against slice k − 1 (fixed) at priors[k − 1] for k = 1..n−1; ms: device time of it all
    bool stack_maps(int n, const float* const* images, const int* ws, const int* hs, const Mat3* priors, bool exact,
                    bool calibrated, unsigned cap, zc_shift_result* out, float* ms);
    // the stack in parts: stack_load uploads the slices, builds their features and plans the
    // n − 1 maps (every buffer the maps use allocated, every build and autocorrelation finished,
    // so the maps can be captured); stack_enqueue queues the maps on `st` with each result key
    // copied into stack_res_ (returns the launches, −1 on an error); stack_collect reads the
    // keys back into out[0 .. n − 2]
    bool stack_load(int n, const float* const* images, const int* ws, const int* hs, const Mat3* priors, bool exact,
                    bool calibrated, unsigned cap);
    int stack_enqueue();
    bool stack_collect(zc_shift_result* out);
    // the buffers run_map uses for a job, allocated now
    bool map_buffers(const MapJob& job);
    std::vector<MapJob> stack_jobs_;
    std::vector<double> stack_areas_;
    uint64_t stack_gen_ = 0;  // bumped by every stack_load (the combined graph's signature)
    // the sweep of the current pair and the loaded stack's maps as two branches of one CUDA graph,
    // launched once (engine_sweep.cpp)
    bool sweep_stack(const Mat3& H0, int n_peak, SweepOut& sw, zc_shift_result* stack_out, size_t n_out);
    bool sweep_with_stack_ = false;  // set while sweep_stack runs sweep_maps
    cudaStream_t branch_st_ = nullptr;  // the stack's branch while the combined graph is captured
    cudaEvent_t fork_ev_ = nullptr, join_ev_ = nullptr;
    // benchmark: warmup + steps maps at H (device-resident inputs), per-step CUDA-event times
    // ms per map of `steps` replays of one captured CUDA graph of job's passes (an L2 flush
    // before each); -1 when the capture or its replay is refused
    double graph_maps(MapJob& job, unsigned warmup, unsigned steps, size_t flush_bytes);
    bool bench_maps(const Mat3& H, unsigned flags, unsigned cap, unsigned warmup, unsigned steps, double* out,
                    size_t out_len);

    // poses (engine_pose.cpp): both directions (or the forward one) of many poses in one pass
    // pose_cps: one spline per pose (n × 2·g·g, the engine's lattice; the inverse direction
    // negated on the other image) instead of the engine's live one
    bool eval_poses(const std::vector<Mat3>& Hs, bool grad, bool hess, std::vector<PoseEval>& out,
                    bool forward_only = false, const float* pose_cps = nullptr);
    bool moments(const Mat3& H, double* out45);
    bool score3(const Mat3& H, double* out3);
    // scores of n ≤ 64 poses with every device buffer in a file-scope array (score_static.cu)
    bool score_static(const double* Hs, uint32_t n, double* out3);
    bool gradient(const Mat3& H, bool hess, zc_grad_result* out);
    bool climb(zc_climb_result* out);

    // the B-spline on top of the pose (engine_ffd.cpp; src/pair.zig:17-37 Ffd): g = ffd_grid
    // clamped to 2..16 (a new g zeroes the control points), 2·g·g control points in half-image
    // units of the lattice's image (the fixed one, or the moving one with ffd_source)
    unsigned ffd_grid();
    bool ffd_live();
    bool set_ffd(const float* cps, size_t n);
    size_t get_ffd(float* cps, size_t cap);
    // score and ∇ over the control points at H (src/pair.zig:387-410 ffdGrad)
    bool ffd_gradient(const Mat3& H, double* score, double* grad, size_t len);
    // the composed warp at the engine's pose (and spline, when on) over the fixed image: per
    // 0-based fixed pixel x_moving − x_fixed (src/export.zig:64-106), rw × rh × 2 floats
    bool displacement(float* out, size_t len);
    // the forward and inverse directions' device splines for the pose passes (none unless live)
    bool ffd_dirs(PoseFfd& fwd, PoseFfd& inv);
    // per-pose splines for n poses (n × 2·g·g floats) as the two directions' device packs
    bool ffd_pose_dirs(const float* cps, int n, PoseFfd& fwd, PoseFfd& inv);
    // the climb's spline stage (src/gclimb.zig:206-246 splineStage): both directions' per-cell
    // Gauss–Newton terms at H, the banded step under the bending energy, the candidates along it
    // picked by score less bending penalty; lam: the penalty weight, set at the climb's first
    // spline step (< 0 until then)
    bool spline_stage(const Mat3& H, double& lam, bool& moved, double& score);
    void log_event(const std::string& text);

    // the rotation × scale sweep (engine_sweep.cpp): every candidate's map reduced to n_peak
    // peaks; batch 0 picks the batch from a memory budget
    // Sweep batch sizes chosen by tune_sweep, per plane class: (nx, ny, correlations, exact).
    std::map<std::array<int, 4>, int> sweep_tuned_;
    // The sweep's launches captured as one CUDA graph, replayed while their parameters (the
    // signature) are unchanged.
    cudaGraphExec_t sweep_exec_ = nullptr;
    std::vector<uint64_t> sweep_sig_;
    int sweep_launches_ = 0;  // kernels one replay of sweep_exec_ launches
    // What the map's canvas / grid / half-spectrum buffers of each side hold (empty: nothing
    // known): a map whose side has the same key reuses them instead of rebuilding that side's
    // canvas and forward transforms. Cleared by every other user of those buffers.
    std::array<std::vector<uint64_t>, 2> spec_key_;
    bool spectra_cache_ = true;     // ZCMIR_B200_SPECTRA_CACHE=0 at creation: always rebuild
    bool spectra_cache_off_ = false;  // set while a benchmark times whole maps
    uint64_t build_counter_ = 0;
    void forget_spectra() {
        spec_key_[0].clear();
        spec_key_[1].clear();
    }
    // the batched Gauss–Newton refine's device state (gn_batch_dev)
    DevBuf gn_H_, gn_Htry_, gn_valid_, gn_active_, gn_cur_;
    PinnedBuf gn_pin_;
    // while tuning: batch per plane class (nx, ny), stream-ordered launches timed per class
    std::map<std::array<int, 2>, int> sweep_force_;
    // time each candidate batch size per plane class of the current sweep settings, keep the
    // fastest (rows of out: nx, ny, candidates, chosen batch, its ms per candidate, options,
    // then (batch, ms per candidate) per option)
    bool tune_sweep(double* out, size_t cap, size_t* used);
    // the forward column FFTs' first stage on the tensor cores in `pieces` BF16 parts (0: FP32)
    bool set_dft_stage(unsigned pieces);
    int dft_pieces_ = 0;
    DevBuf dft_scratch_;
    bool sweep_maps(const Mat3& H0, const SweepGrid& gv, int G, bool exact, int n_peak, double min_overlap,
                    SweepOut& out, int batch = 0, int shard = 0, int nshard = 1);
    // the host half of a sweep: canvas, candidates, footprints, plane sizes and slot order
    bool sweep_setup(const Mat3& H0, const SweepGrid& gv, int G, SweepOut& out);
    // the peaks and their poses from the lane maxima (slot order)
    void sweep_make_peaks(SweepOut& out, int n_peak);
    // the search from a sweep's peaks: NMS, batched Gauss–Newton screen, finalists, the pose
    bool search_finish(const SweepOut& res, const SweepGrid& gv, const Mat3& H0, zc_search_result* out);
    // the search from every candidate's 4 lane maxima gathered from sharded sweeps
    bool search_lanes(const float* scores, const uint32_t* idx, size_t n, zc_search_result* out);
    bool search_check();
    // Gauss–Newton on many poses at once (src/search.zig gnBatch)
    // gn_batch run on the device (gn_device.cu): no host round trip inside a batch of
    // iterations; one read of the poses' moved flags per batch (ZCMIR_B200_GN=host: the host loop)
    bool gn_batch_dev(const std::vector<Mat3>& Hs, unsigned iters, const std::vector<double>& amps,
                      std::vector<ScoredPose>& out);
    bool gn_batch(const std::vector<Mat3>& Hs, unsigned iters, const std::vector<double>& amps,
                  std::vector<ScoredPose>& out);
    // zc_match without keypoints: the SMI sweep search from the images' centres aligned gives
    // the fit, which becomes the pose (keypoint counts 0)
    bool match_by_sweep(zc_match_result* out);
    // sweep → NMS → batched Gauss–Newton screen → finalists (src/search.zig runSweep)
    bool search(zc_search_result* out);
    // the sweep grid, canvas size and prior pose the settings ask for
    void sweep_settings(SweepGrid& gv, int& G, Mat3& H0);

  private:
    bool build_side(int s);
    // the work image of side s from its raw image: CLAHE, band pass, invert as set (preprocessed
    // sides), else the raw image as is
    bool bake(int s, cudaStream_t bs);
    bool build_stream(int s, cudaStream_t& bs);
    std::string bake_key() const;
    bool line_plan(int n, LinePlan& p);
    const float2* twiddles(int n);

    FeatScratch fs_;
    DevBuf fs_stats_, fs_hist_, fs_wt_, fs_acfpart_, fs_acf_, rank_tmp_;
    FeatScratch fs2_;  // side 1's own scratch when it builds on st2_
    DevBuf fs2_stats_, fs2_hist_, fs2_wt_, fs2_acfpart_, rank_tmp2_;
    cudaStream_t st2_ = nullptr;
    cudaStream_t acf_st_ = nullptr;     // the features' autocorrelations, lowest priority
    int prio_lo_ = 0, prio_hi_ = 0;     // the device's stream priority range
    DevBuf canvas_a_, canvas_b_, grid_a_, grid_b_, half_a_, half_b_, q_, map_, res_, flush_;
    DevBuf pose_hinv_, pose_sums_, pose_coef_, pose_score_, pose_tsum_, pose_gens_;
    // the pose kernels' per-block totals and per-pose tickets (their sums added in block order)
    DevBuf pose_part_, pose_ticket_;
    bool pose_red(int n, PoseRed& r);
    DevBuf rs_fwd_, rs_inv_, rs_map_;
    DevBuf pp_rgba_, pp_clahe_, pp_tmp_, pp_mm_;
    std::vector<Side> stack_;
    DevBuf stack_res_;
    DevBuf sw_il_[2], sw_poses_, sw_fgrid_, sw_fhalf_, sw_grid_, sw_half_, sw_q_, sw_map_, sw_n0_, sw_ps_, sw_pi_;
    PinnedBuf pose_in_pin_, pose_out_pin_;  // eval_poses: inverse poses + generators up, sums back
    std::vector<float> ffd_cps_ = std::vector<float>(2 * 16 * 16, 0.f);
    unsigned ffd_g_ = 4;
    bool ffd_suspended_ = false;  // the search's climbs run without the spline
    DevBuf ffd_dev_, ffd_out_, ffd_pk_, ffd_cells_, ffd_coef_;
    std::map<int, float2*> tw_;
};

}  // namespace zc
