// Host-side launchers of the engine's CUDA kernels (features.cu, shiftmap.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "fft.cuh"

namespace zc {

// ── per-image features (features.cu) ──
// Scratch the feature build needs on the device (sizes in bytes are fixed; see features.cu).
struct FeatScratch {
    double* stats = nullptr;     // [0] Σg, [1] Σ(g − mean)², [2..21] whitening moments
    unsigned* hist = nullptr;    // 256 bins
    float* wt = nullptr;         // L⁻¹ (16) and μ (4) of the whitening
    float* acf_part = nullptr;   // per-tile autocorrelation partial sums
    size_t acf_part_cap = 0;     // floats
    double* acf = nullptr;       // 289 × 4 normalised autocorrelation
};

// gray (w×h f32, device) → feat (4 planes), mag (1 plane), stack (5 planes). mode: 0 laplacian,
// 1 three, 2 cubic. `half`: quantise the input to f16 first (in place on `gray`).
cudaError_t build_features(float* gray, int w, int h, int mode, bool half, float* rank_tmp, float* feat,
                           float* mag, float* stack, FeatScratch& s, cudaStream_t st);
// the features' autocorrelation sums at |τ| ≤ 8 (289 lags × 4 planes, device doubles in s.acf;
// per-tile partials in s.acf_part)
cudaError_t autocorrelation(const float* feat, int w, int h, FeatScratch& s, cudaStream_t st);

// ── shift maps (shiftmap.cu) ──
struct MapGeom {
    int W, Hh;       // canvas
    int ox, oy;      // canvas offset (fixed pixel (0,0) at canvas (−ox, −oy))
    int cw, ch;      // correlation grid
    int nx, ny;      // FFT grid
    int WP;          // half-spectrum row pitch (≥ nx/2 + 1)
};

struct CombineParams {
    int exact;       // per-overlap whitening
    int calib;       // Wilson–Hilferty z (exact only)
    int nf;          // features the score runs over (3 or 4); 1: the NCC map (one correlation
                     // over the norm product, which the n00 slot carries)
    float min_n;     // overlap floor (cells)
    double area;     // feature correlation area in cells (calibrated z)
    double ridge;
    double inv_nn;   // 1/(nx·ny): the inverse FFT's scale
    // log-polar maps: each correlation at log-radius lag k (row k, wrapped) is scaled by
    // e^{kΔλ}·Δλ·Δθ so the sums integrate dest area; 0 for shift maps
    double lp_dlam = 0, lp_dth = 0;
};

// Correlation plan on the device: plane numbers per slot, and per correlation slot its
// (moving slot, fixed slot, correlation number).
struct CorrPlanDev {
    int n_real;
    int n_corr;
    int planes[15];
    int ca[45], cb[45], cnum[45];
};

// canvas stacks: moving warped by the canvas pose (hi = its inverse, f32 row-major), fixed pasted
cudaError_t warp_stack(const float* stack, int w, int h, const float hi[9], bool ok, int W, int Hh, float* canvas,
                       cudaStream_t st);
cudaError_t paste_stack(const float* stack, int w, int h, int ox, int oy, int W, int Hh, float* canvas,
                        cudaStream_t st);
cudaError_t resample_grid(const float* canvas, int W, int Hh, int cw, int ch, float* grid, cudaStream_t st);
// Σ grid_a[0]·grid_b[0] (float64) into *out: the overlap count at lag 0
cudaError_t lag0_count(const float* grid_a, const float* grid_b, int cw, int ch, double* out, cudaStream_t st);

// The transforms below run `batch` independent items at once (a sweep's candidates), item b at
// the given strides (in elements) from the first; batch 1 is one map.

// forward transforms of one side: real planes of the grid → row R2C (rows < ch) into the half
// spectra [n_real][ny][WP] complex; then the column FFTs of the half spectra in place (the
// batch's half spectra contiguous: half_stride = n_real·ny·WP)
cudaError_t forward_rows(const float* grid, const MapGeom& g, const CorrPlanDev& plan, const LinePlan& row,
                         float2* half, cudaStream_t st, int batch = 1, size_t grid_stride = 0, size_t half_stride = 0);
cudaError_t forward_cols(float2* half, const MapGeom& g, const CorrPlanDev& plan, const LinePlan& col,
                         cudaStream_t st, int batch = 1);
// the column FFTs on the run-time line plan whatever the length (col.s0: the stage to start at)
cudaError_t forward_cols_generic(float2* half, const MapGeom& g, const CorrPlanDev& plan, const LinePlan& col,
                                 cudaStream_t st);
// The column FFTs with their first stage (radix 16) on the tensor cores (dft_tc.cu): each FP32
// input and each DFT coefficient split into `pieces` (1 to 3) BF16 parts, the stage a sum of
// BF16 products (1, 3 or 6) accumulated in FP32 in tensor memory; then the other
// stages in FP32 (forward_cols_generic from stage 1). scratch: as large as the half spectra;
// the result is copied back into half. fault (device word): 1 or-ed in if a wait on the tensor
// cores gave up. Needs col.radix[0] == 16.
cudaError_t forward_cols_tc(float2* half, float2* scratch, const MapGeom& g, const CorrPlanDev& plan,
                            const LinePlan& col, int pieces, unsigned* fault, cudaStream_t st);
// products and inverse column FFTs: Q[slot][ny][WP] (b_stride 0: one fixed side for every item).
// fault (nullable, device memory): 1 is or-ed into it if the TMA-fed pass (1024- and 2048-point
// square maps, one item) gave up waiting for a copy, 2 if its staging was misaligned; its Q is
// then not valid. ZCMIR_B200_INV_COLS=pipe selects the register-prefetch pass instead.
cudaError_t inverse_columns(const float2* half_a, const float2* half_b, const MapGeom& g, const CorrPlanDev& plan,
                            const LinePlan& col, float2* Q, cudaStream_t st, int batch = 1, size_t a_stride = 0,
                            size_t b_stride = 0, size_t q_stride = 0, unsigned* fault = nullptr);
bool inverse_columns_tma_supported(const MapGeom& g, int batch);
cudaError_t inverse_columns_tma(const float2* half_a, const float2* half_b, const MapGeom& g, const CorrPlanDev& plan,
                                const float2* tw, float2* Q, cudaStream_t st, unsigned* fault);
// inverse row FFTs fused with the per-shift score and the argmax: map (ny × nx f32), best key
// (u64), zero-lag score (best and zero may be null); n00: one zero-lag overlap per item
cudaError_t inverse_rows_score(const float2* Q, const MapGeom& g, const CorrPlanDev& plan, const LinePlan& line,
                               int S, const float2* tw_nx, const CombineParams& cp, const double* n00, float* map,
                               unsigned long long* best, float* zero, cudaStream_t st, int batch = 1,
                               size_t q_stride = 0, size_t map_stride = 0);
// the same pass with the sums in tensor memory: a whole row per block (nx ∈ {512, 1024, 2048})
bool rows_tmem_supported(int nx, int n_corr);
// rows y0 .. y0 + rows − 1 of the map (rows < 0: to the last), so a caller can copy the map out
// in row chunks while the later rows run
cudaError_t inverse_rows_score_tmem(const float2* Q, const MapGeom& g, const CorrPlanDev& plan, const float2* tw_nx,
                                    const CombineParams& cp, const double* n00, float* map, unsigned long long* best,
                                    float* zero, cudaStream_t st, int y0 = 0, int rows = -1);
// the split S of the row pass for nx (smallest divisor keeping its shared memory in budget); 0
// when none fits
int row_split(int nx, int n_corr);
size_t row_pass_smem(int L, int n_corr, int tl);

// ── the rotation × scale sweep (sweep.cu) ──
// The sweep's G×G canvas of cells: cell (cx, cy) spans dest pixels [ox + cx·cell, …) (1-based).
struct SweepCanvas {
    float ox, oy, cell;
    int G;
};
// plane-major 5-plane stack of n pixels → n float4 (w, w f0, w f1, w f2) followed by the fifth
// plane (w f3) as n floats: 20 bytes per pixel
cudaError_t sweep_interleave(const float* stack, int n, float4* il, cudaStream_t st);
// the windows [batch][5][win_y][win_x] of slots slot0.. (poses: 12 floats per slot: dest →
// source map, taps, first window cell); with fw (the fixed window's weights, [Fy][Fx] at cell
// (fx0, fy0)) each item's zero-lag overlap into n0[batch] (cleared here)
cudaError_t sweep_pack(const float4* il, int sw, int sh, const float* poses, int slot0, int batch, int win_x,
                       int win_y, const SweepCanvas& cv, const float* fw, int fx0, int fy0, int Fx, int Fy, float* grid,
                       double* n0, cudaStream_t st);
// the n_peak best lane maxima of each map (map b at maps + b·map_stride) into slots slot0..
cudaError_t sweep_peaks(const float* maps, int nx, int ny, size_t map_stride, int batch, int n_peak, int slot0,
                        float* ps, uint32_t* pi, cudaStream_t st);

// ── preprocessing (preprocess.cu); with `half` every output is rounded to f16 texels ──
cudaError_t rgba_to_gray(const unsigned char* rgba, int n, float* gray, cudaStream_t st);
size_t clahe_scratch_bytes(int grid, int bins);
cudaError_t clahe(const float* src, int w, int h, double clip, int bins, int grid, bool half, void* scratch,
                  float* dst, cudaStream_t st);
// one σ = 1 Gaussian blur (rows then columns) through tmp
cudaError_t gauss_blur(const float* src, int w, int h, bool half, float* tmp, float* dst, cudaStream_t st);
// clamp(fine) − clamp(coarse) rescaled to [0, 1] into out; d (n floats), mm (2 u32) scratch
cudaError_t dog_rescale(const float* fine, const float* coarse, int n, bool half, float* d, unsigned* mm, float* out,
                        cudaStream_t st);
cudaError_t invert_texels(float* a, int n, bool half, cudaStream_t st);
cudaError_t round_texels(float* a, int n, cudaStream_t st);

// ── the roto-scale map (rs.cu) ──
// canvas stack (5 planes, W × Hh) → log-polar grid [5][n_lam][n_th] about (cx, cy), ρ-weighted
cudaError_t rs_logpolar(const float* canvas, int W, int Hh, float cx, float cy, float log0, float span, int n_th,
                        int n_lam, float* grid, cudaStream_t st);
// symmetric average (inv may be null), scale mask, argmax key and lag-0 cell of an n × n map
cudaError_t rs_finish(const float* fwd, const float* inv, bool mirror, int n, float dlam, float lo, float hi,
                      float* out, unsigned long long* best, float* zero, cudaStream_t st);

// ── the NCC overlay metric (ncc.cu); the work images are f32, hi the canvas pose's inverse ──
// both canvas planes of the pair: moving warped (rounded to f16 texels when half), fixed pasted
cudaError_t ncc_canvas(const float* mv, int w, int h, const float hi[9], bool ok, const float* fx, int fw, int fh, int ox,
                       int oy, bool half, int W, int Hh, float* ca, float* cb, cudaStream_t st);
// Σa, Σb, Σa², Σb², Σab over the canvas (float64) into mom[5], the canvas not written
cudaError_t ncc_moments(const float* mv, int w, int h, const float hi[9], bool ok, const float* fx, int fw, int fh,
                        int ox, int oy, bool half, int W, int Hh, double* mom, cudaStream_t st);
// the canvases resampled to cw × ch (plane 0 of ga, gb), made mean-free; sums[4] = Σa, Σb, Σa'²,
// Σb'²; *den = max(‖a'‖‖b'‖, 1e-12)
cudaError_t ncc_grid(const float* ca, const float* cb, int W, int Hh, int cw, int ch, float* ga, float* gb,
                     double* sums, double* den, cudaStream_t st);

// ── pose scores and gradients (pose.cu) ──
struct PoseSide {
    const float* feat;    // 4 whitened planes, plane-major
    const float4* feat4;  // the same planes interleaved, one float4 per pixel
    int w, h;
};
// the 4 plane-major feature planes of n pixels interleaved into one float4 per pixel
cudaError_t interleave_features(const float* feat, int n, float4* out, cudaStream_t st);
// A cubic B-spline on top of the pose: g × g control points (x, y per point, in half-image units
// of the lattice's image), on b (the destination: it moves b's pixel before H⁻¹) or, source, on a
// (it moves the sample after H⁻¹). cps null: no spline.
struct PoseFfd {
    const float* cps = nullptr;
    int g = 0;
    int source = 0;
    int stride = 0;  // floats between poses' control points (0: one set for every pose)
};
// How a pose's blocks add their float64 totals. With part set, each block stores its totals in
// part and the pose's last block to finish adds them in block order, so the sums are the same on
// every run and in every batch; ticket: one counter per pose of the launch, zero before it (each
// is put back to zero). Without part: float64 atomics, in the order the blocks finish.
struct PoseRed {
    double* part = nullptr;
    unsigned* ticket = nullptr;
    size_t cap = 0;      // doubles at part
    size_t tickets = 0;  // counters at ticket
};
// doubles of PoseRed::part any pose kernel needs for n poses onto an image of `pixels` pixels
size_t pose_red_need(size_t pixels, int n);
// the 45 sums of n poses of one direction (a sampled at H⁻¹x for every b pixel x); hinv: n
// inverse poses (f32, row-major); sums: n × 45 float64 (zeroed here)
// The pose kernels' launch shape (zc_tune_parts): pixels per thread, the least and the most
// blocks per pose (0 keeps the current value). It changes the order of the cross-block sums, so
// scores move within their float32 rounding.
void pose_tune(unsigned px_per_thread, unsigned min_blocks, unsigned max_blocks);
// mask (nullable, n bytes): poses with a zero byte are skipped (their sums stay 0)
cudaError_t pose_moments(const PoseSide& a, const PoseSide& b, const float* hinv, int n, double* sums, cudaStream_t st,
                         const PoseFfd& ffd = {}, const unsigned char* mask = nullptr, const PoseRed& red = {});
// score (float64) and the 102 gradient coefficients (f32) of each pose's sums
cudaError_t pose_coefs(const double* sums, int n, bool exact, float* coef, double* score, cudaStream_t st);
// tangent sums per pose: 8 gradient + 36 Gauss–Newton (upper triangle) float64 (zeroed here);
// gens: 8 generators (9 f32 each) in b's pixel coordinates
cudaError_t pose_tangent(const PoseSide& a, const PoseSide& b, const float* hinv, const float* coef, const float* gens,
                         int n, bool hess, double* out, cudaStream_t st, const PoseFfd& ffd = {},
                         const unsigned char* mask = nullptr, const PoseRed& red = {});
// ── the batched Gauss–Newton refine on the device (gn_device.cu) ──
struct GnDims {
    int n;        // poses
    int T;        // candidates per pose: the step ladder's then the 5 Gauss–Newton multiples
    int nk;       // tangent keys (8 homography, 6 affine)
    int homog, sym;
    double mw, mh, fw, fh;  // moving and fixed image sizes
};
struct GnAmps {
    int n;         // unit-ascent step lengths (≤ 16)
    double v[16];
};
// inverse maps of n poses H (n × 9 float64) for the pose kernels: forward rows 0..n−1, the
// inverse direction's n..2n−1 when sym
cudaError_t gn_hinv(const double* H, int n, int sym, float* hinv, cudaStream_t st);
// per active pose: its pair score into cur, its candidates into Htry (n × T × 9) and valid
cudaError_t gn_propose(const GnDims& d, const GnAmps& amps, const double* H, const double* sums, const double* score,
                       const double* tsum, const unsigned char* active, double* cur, double* Htry,
                       unsigned char* valid, cudaStream_t st);
// per active pose: the first candidate (in order) that beats the score so far becomes the pose;
// a pose that did not move becomes inactive. tscore: the candidates' scores (forward, then inverse)
cudaError_t gn_select(const GnDims& d, const double* tscore, const unsigned char* valid, const double* Htry, double* H,
                      double* cur, unsigned char* active, cudaStream_t st);
// ∂score/∂(control points cp0 .. cp0 + 15) of pose 0 of one direction from its coefficients:
// out[32] float64 (x then y per point; zeroed here)
cudaError_t pose_ffd_grad(const PoseSide& a, const PoseSide& b, const float* hinv, const float* coef,
                          const PoseFfd& ffd, int cp0, double* out, cudaStream_t st, const PoseRed& red = {});
// the spline's Gauss–Newton terms per lattice cell of pose 0 of one direction (its coefficients
// with a positive semi-definite Q): per cell and chunk 332 float32 sums (100 symmetric basis
// pairs × K_xx, K_xy, K_yy, then 16 taps × ∇_x, ∇_y); nch chunks per cell
constexpr int kFfdCell = 332;
cudaError_t pose_ffd_cells(const PoseSide& a, const PoseSide& b, const float* hinv, const float* hpose,
                           const float* coef, const PoseFfd& ffd, int nch, float* out, cudaStream_t st);

}  // namespace zc
