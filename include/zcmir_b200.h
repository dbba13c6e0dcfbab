/* Entry points of the B200 build beyond the reference's zc_* ABI (libzcmir.so). They have no
 * counterpart in the reference: benchmarking and host-logic checks that need no GPU. */
#ifndef ZCMIR_B200_H
#define ZCMIR_B200_H

#include "zcmir.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Time `steps` shift maps at pose H after `warmup` untimed ones, with the images' features
 * resident on the GPU and an L2 flush between timed maps (outside the timed spans). flags: 1
 * exact, 2 calibrated; cap as zc_shift_map (0: 1024). out[16] (out_len ≥ 16): [0] ms per map
 * (CUDA events around replays of one CUDA graph of the map's passes; the instrumented maps' time
 * when the graph cannot be captured), [1..5] per-stage ms of event-instrumented maps (canvas,
 * forward rows, forward columns, inverse columns, inverse rows + score), [6] ms per instrumented
 * map, [7] canvas height, [8..15] nx, ny, cw, ch, real planes, correlations, row split, canvas
 * width. 0 / -1 with zc_error. */
int32_t zcb_bench_maps(zc_engine* e, const double H[9], uint32_t flags, uint32_t cap, uint32_t warmup, uint32_t steps,
                       double* out, size_t out_len);

/* Settings without an engine: apply the JSON object `json` onto the defaults and write the
 * resulting settings JSON to out (the full length is returned through *out_len). 0 on success;
 * -1 with the message in err (its length through *err_len) when the JSON is rejected. */
int32_t zcb_settings_apply(const char* json, size_t len, char* out, size_t cap, size_t* out_len, char* err,
                           size_t err_cap, size_t* err_len);

/* The sweep's batched maps alone (the first stage of zc_search) with the engine's sw_* settings
 * and prior pose H0 (NULL: the pose zc_search would use). For every candidate (θ-major, then σ,
 * shear, stretch) its n_peak (1..16) best lane maxima — score in fixed pixels, map index
 * (0xffffffff: none) — into scores / idx (cap ≥ candidates × n_peak; both NULL: not returned).
 * batch: candidates per launch (0: per plane class the size zcb_tune_sweep chose, else what a
 * 1 GB budget holds, at most 128). The whole sweep's launches are captured once as a CUDA graph and
 * replayed while their parameters are unchanged (ZCMIR_B200_SWEEP_GRAPH=0: stream-ordered
 * launches). shard / nshard: only the candidates in
 * slots ≡ shard (mod nshard) of the plane-size order are mapped (one rank's share of a sweep
 * split across GPUs); the others' entries stay (0, 0xffffffff), so the shards' outputs merge by
 * a sum of scores and a minimum of indices. info[16]: [0] candidates, [1] cell (px),
 * [2] device ms of the maps, [3] grid G, [4..5] fixed window Fx, Fy (cells), [6..7] its first
 * cell, [8] overlap floor (cells), [9] largest plane side, [10] plane-size groups, [11] batches,
 * [12] kernel launches, [13..14] canvas origin (px), [15] peaks. No counterpart in the reference
 * (its sweep is internal to zc_search, src/search.zig:300-494). 0 / -1 with zc_error. */
int32_t zcb_sweep(zc_engine* e, const double H0[9], uint32_t n_peak, uint32_t batch, uint32_t shard, uint32_t nshard,
                  float* scores, uint32_t* idx, size_t cap, double* info, size_t info_len);

/* The sweep's autotuner: for every plane class (nx × ny) of a sweep with the engine's sw_*
 * settings and images, times the whole sweep stream-ordered with candidate batches of 16, 32, …,
 * 2048 (each class capped by its candidates and an 8 GB work-buffer budget) and keeps, per class,
 * the batch with the least device time per candidate map; later sweeps (zcb_sweep batch 0,
 * zc_search) use it. out (nullable, cap doubles; *used: the doubles written or needed), per class:
 * nx, ny, candidates, chosen batch, its ms per candidate, k, then k pairs (batch, ms per
 * candidate). Tuning grows the sweep's work buffers to the largest batch tried. No counterpart in
 * the reference (whose tuning hooks, src/exports.zig:95-121, set workgroup shapes by hand).
 * 0 / -1 with zc_error. */
int32_t zcb_tune_sweep(zc_engine* e, double* out, size_t cap, size_t* used);

/* zc_search from gathered lane maxima: scores / idx hold every candidate's 4 lane maxima (n =
 * candidates × 4, as zcb_sweep with n_peak 4 writes them, merged over shards); the engine's
 * settings must be those of the sweep. Runs the rest of the search (peaks → poses, NMS, batched
 * Gauss–Newton screen, finalists) and sets the pose as zc_search does. No counterpart in the
 * reference (its search is one call, src/search.zig:663-820). 0 / -1 with zc_error. */
int32_t zcb_search_lanes(zc_engine* e, const float* scores, const uint32_t* idx, size_t n, zc_search_result* out);

/* Shift maps along a stack of n ≥ 2 slices (gray f32 images[i], w[i] × h[i]): each slice's
 * features are built once, then slice k (moving) is mapped against slice k − 1 (fixed) for
 * k = 1..n−1 at pose priors[9·(k−1)..] (NULL: the slices' centres aligned), with flags (1 exact,
 * 2 calibrated) and cap as zc_shift_map; out[k−1] gets each map's result, *ms (nullable) the
 * device time of the whole stack (features and maps). The engine's own image pair and pose are
 * left as they were. No counterpart in the reference (its register_stack registers pair by pair
 * through the functional API, python/zcmir/api.py:522-580). 0 / -1 with zc_error. */
int32_t zcb_stack_maps(zc_engine* e, uint32_t n, const float* const* images, const uint32_t* w, const uint32_t* h,
                       const double* priors, uint32_t flags, uint32_t cap, zc_shift_result* out, double* ms);

/* zcb_stack_maps in two parts, for the combined launch. zcb_stack_load takes the same stack
 * (slices, sizes, priors, flags, cap): it builds every slice's features and plans the n − 1 maps,
 * allocating what they need, and runs no map. zcb_sweep_stack then runs the sweep of the engine's
 * image pair (as zcb_sweep with the current sw_* settings, all candidates, the tuned batches;
 * H0 NULL: the settings' start pose) and the loaded stack's maps as two branches of ONE CUDA
 * graph (captured on the first call, kept while the sweep's schedule, the stack and their buffers
 * are unchanged), launched once: scores/idx/cap/info as zcb_sweep (info[2] is the device time of
 * the whole launch, info[12] its kernel count), stack_out[0 .. n − 2] as zcb_stack_maps's out
 * (n_out ≥ n − 1). The stack stays loaded across calls. No counterpart in the reference. 0 / -1
 * with zc_error. */
int32_t zcb_stack_load(zc_engine* e, uint32_t n, const float* const* images, const uint32_t* w, const uint32_t* h,
                       const double* priors, uint32_t flags, uint32_t cap);
int32_t zcb_sweep_stack(zc_engine* e, const double H0[9], uint32_t n_peak, float* scores, uint32_t* idx, size_t cap,
                        double* info, size_t info_len, zc_shift_result* stack_out, size_t n_out);

/* Scores of n poses (Hs: n row-major 3×3 maps, each as zc_score's H) into out[3n], per pose the
 * mean, forward and inverse score exactly as zc_score writes them, allocating no device memory.
 * No counterpart in the reference (whose only pose score is zc_score, src/exports.zig:417). For
 * hosts that cannot let a call allocate: zc_score grows its buffers with cudaMalloc/cudaFree,
 * and cudaFree waits for the whole device (stalling the host's other streams), while a host that
 * gave the GPU's free memory to its own pool can see that allocation fail. The scratch is one
 * file-scope device array of 103,936 bytes: n ≤ 64 (larger n is rejected with an error), and
 * calls that overlap in time (any engines on the same device) race on it; it keeps the last
 * call's contents. zc_create looks up the array's address on its device, which (with lazy module
 * loading) loads the module holding it and so reserves its bytes then, not in a call; only if that
 * look-up failed does the first call on the device retry it (make that call before any stream
 * capture begins). The feature planes must already be built for the current settings (by
 * zc_set_image_gray, zc_score or zc_features), else -1 with zc_error; a side still building on a
 * stream of its own is waited for on the engine's stream. 0 / -1. */
int32_t zcb_score_static(zc_engine* e, const double* Hs, uint32_t n, double* out);

/* Precision study of the FFT's small-radix stage (no counterpart in the reference): with pieces 1,
 * 2 or 3, the shift maps' forward column FFTs (zc_shift_map and the settings map) run their first
 * stage — radix 16, which the column length must start with — on the tensor cores, every FP32
 * input and DFT coefficient split into `pieces` BF16 parts and the stage summed from their
 * products (1, 3 or 6) in FP32; the other stages stay FP32. The stage needs one more buffer as
 * large as a side's half spectra and an extra pass, so it is slower than the default; 0 (the
 * default) puts the FP32 stage back. Other values: −1 with zc_error. 0 / −1. */
int32_t zcb_set_dft_stage(zc_engine* e, uint32_t pieces);

/* Gauss–Newton from each of n poses (Hs, row-major 3×3 each) at once for `iters` steps of the
 * search's batched screen (src/search.zig gnBatch: a step only where it raises the pair score),
 * the final poses into Hout and their scores into scores: the seeds of a search that starts from
 * poses of its own (the learned proposal's). 0 / −1. */
int32_t zcb_refine_poses(zc_engine* e, const double* Hs, uint32_t n, uint32_t iters, double* Hout, double* scores);

/* The learned pose proposal's network (no counterpart in the reference): a circular 1-D CNN over
 * a coarse sweep landscape x [n][6][36] (per rotation 10·i° from −180°, for each of 3 scales: the
 * best and second-best map peak over the landscape's maximum), logits [n][3240] over the plain
 * sweep's 360 × 9 rotation × scale grid (index 90·i + 9·dθ + s: rotation 10·i − 5 + dθ degrees
 * from −180°, scale s). params: zcb_prop_nparams() float32 (conv 6→32 k5, conv 32→32 k5, conv
 * 32→90 k3, each weights then bias). The calls allocate and free their own device memory; 0 / −1
 * with the message from zcb_prop_error. */
size_t zcb_prop_nparams(void);
size_t zcb_prop_error(char* buf, size_t cap);
int32_t zcb_prop_forward(const float* params, size_t np, const float* x, uint32_t n, float* logits);
/* per-sample softmax cross-entropy loss[n] over labels (0..3239) and the mean loss's gradient */
int32_t zcb_prop_grad(const float* params, size_t np, const float* x, const int32_t* labels, uint32_t n, float* loss,
                      float* grad);
/* Adam (β 0.9 / 0.999) over seeded shuffled minibatches of `batch` for `epochs`; params in/out;
 * epoch_loss[epochs] (nullable) the mean training loss of each epoch */
int32_t zcb_prop_train(float* params, size_t np, const float* x, const int32_t* labels, uint32_t n, uint32_t batch,
                       uint32_t epochs, float lr, uint32_t seed, float* epoch_loss);

/* The 2-D convolutional pose proposal on the tensor cores (no counterpart in the reference): input
 * x [n][128][128][8] BF16 bits (uint16; NHWC: 4 feature planes of each image of a pair), four
 * 3×3 stride-2 convolutions 8→32→64→64→128 with ReLU, the mean over the 8×8 positions and a
 * linear layer to logits [n][216] (24 rotation × 9 log-scale bins, index 9·r + s). Weights are
 * used rounded to BF16, activations stored in BF16, every product summed in FP32 (mma.sync
 * m16n8k16). params: zcb_cnn_nparams() float32 (W1 [32][3][3][8], b1, W2 [64][3][3][32], b2,
 * W3 [64][3][3][64], b3, W4 [128][3][3][64], b4, Wfc [216][128], bfc). The calls allocate and
 * free their own device memory; 0 / −1 with the message from zcb_cnn_error. */
size_t zcb_cnn_nparams(void);
size_t zcb_cnn_error(char* buf, size_t cap);
int32_t zcb_cnn_forward(const float* params, size_t np, const uint16_t* x, uint32_t n, float* logits);
/* the mean softmax cross-entropy over labels (0..215) of a batch of n ≤ 4096, and its gradient */
int32_t zcb_cnn_grad(const float* params, size_t np, const uint16_t* x, const int32_t* labels, uint32_t n, float* loss,
                     float* grad);
/* Adam (β 0.9 / 0.999) for `steps` minibatches of `batch` ≤ 1024 drawn with replacement (seeded)
 * from the n samples, all held on the device; params in/out; losses[steps] (nullable) each
 * step's mean loss; ms_per_step (nullable) the device time per step */
int32_t zcb_cnn_train(float* params, size_t np, const uint16_t* x, const int32_t* labels, uint32_t n, uint32_t batch,
                      uint32_t steps, float lr, uint64_t seed, float* losses, float* ms_per_step);

/* The device's measured FP32 rate (TFLOP/s, fused multiply-adds counted as two), the
 * denominator of the maps' FP32 roofline fraction (no counterpart in the reference). 0 / −1. */
int32_t zcb_fp32_peak(double* tflops);

#ifdef __cplusplus
}
#endif

#endif /* ZCMIR_B200_H */
