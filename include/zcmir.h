/* zcmir C ABI, B200 build (libzcmir.so).
 *
 * The drop-in boundary for zcmir's SMI path: the same `zc_*` entry points, argument meanings,
 * struct layouts and error conventions as the reference's native library, so the reference's
 * own ctypes loader (python/zcmir/_native.py:69-146, `_SIGS` 79-133) binds this library
 * unchanged. Each declaration cites the reference export it replaces (src/exports.zig or
 * src/native_api.zig, by line).
 *
 * Conventions (src/exports.zig:1-16):
 *   - i32 results: 0 = ok, -1 = failure; zc_error() gives the message.
 *   - size_t results that fill a caller buffer return the full length (the caller retries
 *     with a larger buffer when it exceeds cap).
 *   - every output array is caller-allocated, with its length; the engine copies input
 *     images and owns all device memory; an engine is an opaque heap object freed by
 *     zc_destroy.
 *   - one engine = one CUDA context on one GPU; calls are not thread-safe, except zc_cancel.
 *   - every result-returning call is synchronous (it returns after the GPU work and the
 *     copy back have finished).
 * Pose convention: H maps MOVING pixel coordinates to FIXED ones, row-major 3x3 doubles,
 * (1, 1) the centre of the top-left pixel.
 */
#ifndef ZCMIR_H
#define ZCMIR_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct zc_engine zc_engine;

/* Result of a shift map (src/engine.zig:32-53; 88 bytes). The map is n_y rows of n with lag
 * (0, 0) at index 0 and negative lags wrapped; corrected pose = translate(-dx, -dy) * H. */
typedef struct zc_shift_result {
    uint32_t n, cw, ch, canvas_w, canvas_h;
    int32_t ox, oy;
    uint32_t peak_index;
    double dx, dy, peak, zero, corr_area_px;
    uint32_t exact, calibrated, n_y, _pad;
} zc_shift_result;

/* Result of a roto-scale map (src/engine.zig:59-75; 96 bytes). */
typedef struct zc_rs_result {
    uint32_t n, n_th, n_lam, peak_index;
    double dlam, r0, r1, cx, cy, peak, zero, dth, dsg;
    uint32_t symmetric, calibrated;
} zc_rs_result;

/* Pose score and tangent gradient (src/engine.zig:78-87; 616 bytes). */
typedef struct zc_grad_result {
    double score, fwd, inv, n;
    double grad[8];
    double hess[64];
    uint32_t has_hess, nk;
} zc_grad_result;

/* Climb result (src/climb.zig:7-12; 88 bytes). */
typedef struct zc_climb_result {
    double H[9];
    double score;
    uint32_t iterations, moved;
} zc_climb_result;

/* Keypoint detection counts (src/engine.zig:113; 16 bytes). */
typedef struct zc_detect_result {
    uint32_t n1, n2, levels1, levels2;
} zc_detect_result;

/* Match result (src/engine.zig:117-129; 112 bytes). */
typedef struct zc_match_result {
    double H[9];
    uint32_t ninl, n_corr, ninl_aff, pos_n, pos_inl, has_rot;
    double rot_deg;
    uint32_t pos_kept, _pad;
} zc_match_result;

/* Search result (src/search.zig:30-41; 104 bytes). */
typedef struct zc_search_result {
    double H[9];
    double score, prev;
    uint32_t improved, count_a, count_b, _pad;
} zc_search_result;

/* Union canvas of a pose (src/overlay.zig Canvas; 88 bytes). */
typedef struct zc_canvas_info {
    int32_t ox, oy;
    uint32_t ow, oh;
    double Hc[9];
} zc_canvas_info;

/* ── creation and errors ── */
const char* zc_version(void);                                           /* src/native_api.zig:20 */
/* Creates an engine on the current CUDA device. The argument (the reference's wgpu-native
 * path) is accepted and ignored. NULL on failure; zc_create_error says why. */
zc_engine* zc_create(const char* wgpu_path);                            /* src/native_api.zig:26 */
size_t zc_create_error(char* buf, size_t cap);                          /* src/native_api.zig:41 */
void zc_destroy(zc_engine* e);                                          /* src/native_api.zig:47 */
size_t zc_adapter(zc_engine* e, char* buf, size_t cap);                 /* src/exports.zig:22 */
size_t zc_error(zc_engine* e, char* buf, size_t cap);                   /* src/exports.zig:30 */

/* ── settings ── */
int32_t zc_configure(zc_engine* e, const char* json, size_t len);       /* src/exports.zig:35 */
size_t zc_settings(zc_engine* e, char* buf, size_t cap);                /* src/exports.zig:42 */

/* ── images ── */
int32_t zc_set_image(zc_engine* e, uint32_t side, const float* data, uint32_t w, uint32_t h);          /* src/exports.zig:50 */
int32_t zc_set_image_gray(zc_engine* e, uint32_t side, const float* data, uint32_t w, uint32_t h,
                          uint32_t preprocess);                                                          /* src/exports.zig:57 */
int32_t zc_set_image_rgba(zc_engine* e, uint32_t side, const uint8_t* data, uint32_t w, uint32_t h);  /* src/exports.zig:63 */
int32_t zc_work_image(zc_engine* e, uint32_t side, float* out, size_t len);                            /* src/exports.zig:320 */
int32_t zc_features(zc_engine* e, uint32_t side, float* out, size_t len);                              /* src/exports.zig:264 */
void zc_image_size(zc_engine* e, uint32_t side, uint32_t out[2]);                                      /* src/exports.zig:238 */
void zc_swap(zc_engine* e);                                                                            /* src/exports.zig:226 */

/* ── scores and maps ── */
int32_t zc_moments(zc_engine* e, const double H[9], double out[45]);    /* src/exports.zig:276 */
int32_t zc_score(zc_engine* e, const double H[9], double out[3]);       /* src/exports.zig:417 */
int32_t zc_gradient(zc_engine* e, const double H[9], uint32_t hess, zc_grad_result* out);          /* src/exports.zig:424 */
int32_t zc_shift_map(zc_engine* e, const double H[9], uint32_t flags, uint32_t cap, zc_shift_result* out,
                     float* map, size_t map_len);                                                   /* src/exports.zig:436 */
int32_t zc_shift_map_set(zc_engine* e, const double H[9], zc_shift_result* out, float* map,
                         size_t map_len);                                                           /* src/exports.zig:442 */
int32_t zc_rs_map(zc_engine* e, const double H[9], const double* c, uint32_t symmetric, zc_rs_result* out,
                  float* map, float* fwd, float* inv, size_t len);                                  /* src/exports.zig:449 */

/* ── pose and optimisation ── */
void zc_set_pose(zc_engine* e, const double H[9]);                      /* src/exports.zig:388 */
void zc_get_pose(zc_engine* e, double H[9]);                            /* src/exports.zig:392 */
int32_t zc_climb(zc_engine* e, zc_climb_result* out);                   /* src/exports.zig:405 */
int32_t zc_search(zc_engine* e, zc_search_result* out);                 /* src/exports.zig:344 */
void zc_cancel(zc_engine* e);                                           /* src/exports.zig:221 */
size_t zc_events(zc_engine* e, char* buf, size_t cap);                  /* src/exports.zig:412 */

/* ── profiling ── */
int32_t zc_profile(zc_engine* e, uint32_t on);                          /* src/exports.zig:210 */
size_t zc_profile_report(zc_engine* e, char* buf, size_t cap);          /* src/exports.zig:215 */
void zc_gpu_counts(zc_engine* e, uint32_t out[4]);                      /* src/exports.zig:110 */
int32_t zc_bench_moments(zc_engine* e, uint32_t n_poses, uint32_t iters);                /* src/exports.zig:123 */
void zc_tune_parts(uint32_t px_per_thread, uint32_t fill_wg, uint32_t tg_px, uint32_t tg_cap);  /* src/exports.zig:116 */

/* ── outside the SMI path: exported so the reference's loader binds, each returns its
 * failure value with a "not supported" message (keypoints, splines, overlays, export) ── */
int32_t zc_compile_wgsl(zc_engine* e, const char* code, size_t code_len, const char* entry, size_t entry_len,
                        char* msg, size_t cap);                                            /* src/exports.zig:245 */
int32_t zc_pg_info(zc_engine* e, double out[5]);                                           /* src/exports.zig:284 */
int32_t zc_pg_maps(zc_engine* e, uint32_t side, float* out, size_t len);                   /* src/exports.zig:293 */
int32_t zc_pg_descriptors(zc_engine* e, uint32_t side, float* out, size_t len);            /* src/exports.zig:306 */
int32_t zc_match_scores(zc_engine* e, float* out, size_t cap);                             /* src/exports.zig:232 */
int32_t zc_detect(zc_engine* e, zc_detect_result* out);                                    /* src/exports.zig:332 */
int32_t zc_match(zc_engine* e, zc_match_result* out);                                      /* src/exports.zig:338 */
int32_t zc_auto(zc_engine* e, zc_climb_result* out);                                       /* src/exports.zig:350 */
int32_t zc_keypoints(zc_engine* e, uint32_t side, float* out, size_t cap_points);          /* src/exports.zig:356 */
int32_t zc_keypoint_frames(zc_engine* e, uint32_t side, float* out, size_t cap_points);    /* src/exports.zig:364 */
int32_t zc_matches(zc_engine* e, uint32_t* out, size_t cap);                               /* src/exports.zig:376 */
int32_t zc_set_ffd(zc_engine* e, const float* cps, size_t n);                              /* src/exports.zig:382 */
size_t zc_get_ffd(zc_engine* e, float* cps, size_t cap);                                   /* src/exports.zig:397 */
uint32_t zc_fit_check(zc_engine* e, const double H[9]);                                    /* src/exports.zig:371 */
int32_t zc_ffd_gradient(zc_engine* e, const double H[9], double* score, double* grad, size_t len);    /* src/exports.zig:430 */
int32_t zc_canvas(zc_engine* e, const double H[9], uint32_t inverse, zc_canvas_info* out);      /* src/exports.zig:458 */
int32_t zc_overlay(zc_engine* e, const double H[9], uint32_t inverse, zc_canvas_info* out, float* moving, float* fixed,
                   size_t len);                                                             /* src/exports.zig:465 */
int32_t zc_tile_heat(zc_engine* e, const double H[9], uint32_t grid, uint32_t min_n, double* out, float* dest,
                     float* src, size_t len);                                               /* src/exports.zig:471 */
int64_t zc_export_warp(zc_engine* e, const char* stem, size_t stem_len, void* out, size_t cap);       /* src/exports.zig:480 */
int32_t zc_displacement(zc_engine* e, float* out, size_t len);                             /* src/exports.zig:489 */

/* Sizes of ShiftResult, RsResult, GradResult (src/exports.zig:497). */
void zc_result_sizes(uint32_t out[4]);

#ifdef __cplusplus
}
#endif

#endif /* ZCMIR_H */
