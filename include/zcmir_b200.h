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
 * (CUDA events), [1..5] per-stage ms (canvas, forward rows, forward columns, inverse columns,
 * inverse rows + score), [7] canvas height, [8..15] nx, ny, cw, ch, real planes, correlations,
 * row split, canvas width. 0 / -1 with zc_error. */
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
 * batch: candidates per launch (0: from a 1 GB budget). info[16]: [0] candidates, [1] cell (px),
 * [2] device ms of the maps, [3] grid G, [4..5] fixed window Fx, Fy (cells), [6..7] its first
 * cell, [8] overlap floor (cells), [9] largest plane side, [10] plane-size groups, [11] batches,
 * [12] kernel launches, [13..14] canvas origin (px), [15] peaks. No counterpart in the reference
 * (its sweep is internal to zc_search, src/search.zig:300-494). 0 / -1 with zc_error. */
int32_t zcb_sweep(zc_engine* e, const double H0[9], uint32_t n_peak, uint32_t batch, float* scores, uint32_t* idx,
                  size_t cap, double* info, size_t info_len);

/* Scores of n poses (Hs: n row-major 3×3 maps, each as zc_score's H) into out[3n], per pose the
 * mean, forward and inverse score exactly as zc_score writes them, allocating no device memory.
 * No counterpart in the reference (whose only pose score is zc_score, src/exports.zig:417). For
 * hosts that cannot let a call allocate: zc_score grows its buffers with cudaMalloc/cudaFree,
 * and cudaFree waits for the whole device (stalling the host's other streams), while a host that
 * gave the GPU's free memory to its own pool can see that allocation fail. The scratch is one
 * file-scope device array of 103,936 bytes: n ≤ 64 (larger n is rejected with an error), and
 * calls that overlap in time (any engines on the same device) race on it; it keeps the last
 * call's contents. The first call on each device looks up the array's address (make it before
 * any stream capture begins). The feature planes must already be built for the current
 * settings (by zc_set_image_gray, zc_score or zc_features); otherwise -1 with zc_error. 0 / -1. */
int32_t zcb_score_static(zc_engine* e, const double* Hs, uint32_t n, double* out);

#ifdef __cplusplus
}
#endif

#endif /* ZCMIR_B200_H */
