// The SMI shift map on the GPU (the reference's Smi.shiftMap, src/smi.zig:540-572, with its
// kernels in shaders/smi.wgsl:626-931, 1597-1706).
//
// Pipeline for one map (nx × ny FFT grid, cw × ch correlation grid, P real planes, C
// correlations):
//   1. canvas: the moving stack warped by the canvas pose, the fixed stack pasted
//      (warp_stack / paste_stack), then resampled to the grid when the map is coarser.
//   2. forward_rows / forward_cols (per side): the P real planes are formed on the fly from the
//      5 stack values, two per complex row, row-FFT'd (rows < ch only), unpacked into P half
//      spectra (columns 0..nx/2), then column-FFT'd (rows ≥ ch are zero).
//   3. inverse_columns: per correlation and column tile, A·conj(B) and the inverse column FFT.
//   4. inverse_rows_score: per row, correlations paired as c1 + i·c2 on the Hermitian full row,
//      inverse row FFT, and the per-shift score in float64 with its argmax, without writing a
//      correlation plane to memory. Rows longer than shared memory holds for all C correlations
//      are split S ways by one decimation-in-frequency step (output shifts x ≡ s mod S).
#include <cstdlib>
#include <string>

#include "passes.cuh"

namespace zc {
namespace {

// ── canvas (smi.wgsl:1655-1706) ──────────────────────────────────────────────────────────────

struct Mat9f {
    float m[9];
};

__global__ void k_warp_stack(const float* __restrict__ stack, int w, int h, Mat9f hi, int ok_det, int W, int Hh,
                             float* __restrict__ canvas) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= Hh) return;
    const size_t n = (size_t)W * Hh, pix = (size_t)y * W + x, sn = (size_t)w * h;
    bool ok = ok_det != 0;
    float fx = 0.f, fy = 0.f;
    if (ok) {
        const float X = (float)x + 1.0f, Y = (float)y + 1.0f;
        const float qx = hi.m[0] * X + hi.m[1] * Y + hi.m[2];
        const float qy = hi.m[3] * X + hi.m[4] * Y + hi.m[5];
        const float qz = hi.m[6] * X + hi.m[7] * Y + hi.m[8];
        ok = fabsf(qz) >= 1e-8f;
        if (ok) {
            fx = qx / qz - 1.0f;
            fy = qy / qz - 1.0f;
            ok = !(fx < 0.f || fy < 0.f || fx > (float)(w - 1) || fy > (float)(h - 1));
        }
    }
    int x0 = 0, y0 = 0, x1 = 0, y1 = 0;
    float tx = 0.f, ty = 0.f;
    if (ok) {
        const float flx = floorf(fx), fly = floorf(fy);
        tx = fx - flx;
        ty = fy - fly;
        x0 = min(max((int)flx, 0), w - 1);
        y0 = min(max((int)fly, 0), h - 1);
        x1 = min(max((int)flx + 1, 0), w - 1);
        y1 = min(max((int)fly + 1, 0), h - 1);
    }
#pragma unroll
    for (int p = 0; p < 5; ++p) {
        float v = 0.f;
        if (ok) {
            const float* s = stack + p * sn;
            const float v00 = s[(size_t)y0 * w + x0], v10 = s[(size_t)y0 * w + x1];
            const float v01 = s[(size_t)y1 * w + x0], v11 = s[(size_t)y1 * w + x1];
            const float a = v00 * (1.f - tx) + v10 * tx, b = v01 * (1.f - tx) + v11 * tx;
            v = a * (1.f - ty) + b * ty;
        }
        canvas[p * n + pix] = v;
    }
}

__global__ void k_paste_stack(const float* __restrict__ stack, int w, int h, int ox, int oy, int W, int Hh,
                              float* __restrict__ canvas) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= Hh) return;
    const size_t n = (size_t)W * Hh, pix = (size_t)y * W + x, sn = (size_t)w * h;
    const int sx = x + ox, sy = y + oy;
    const bool in = sx >= 0 && sy >= 0 && sx < w && sy < h;
#pragma unroll
    for (int p = 0; p < 5; ++p) canvas[p * n + pix] = in ? stack[p * sn + (size_t)sy * w + sx] : 0.f;
}

// k×k box of bilinear taps per cell (smi.wgsl:626-639, 675-705)
__global__ void k_resample(const float* __restrict__ canvas, int W, int Hh, int cw, int ch, float* __restrict__ grid) {
    const int gx = blockIdx.x * blockDim.x + threadIdx.x, gy = blockIdx.y * blockDim.y + threadIdx.y;
    if (gx >= cw || gy >= ch) return;
    const float fx = (float)W / (float)max(cw, 1), fy = (float)Hh / (float)max(ch, 1);
    const int kx = (int)fminf(fmaxf(ceilf(fx - 1e-4f), 1.f), 8.f);
    const int ky = (int)fminf(fmaxf(ceilf(fy - 1e-4f), 1.f), 8.f);
    const size_t n = (size_t)W * Hh, gn = (size_t)cw * ch;
    float s[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
    for (int j = 0; j < ky; ++j) {
        const float py = ((float)gy + ((float)j + 0.5f) / (float)ky) * fy - 0.5f;
        const float fly = floorf(py);
        const float ay = py - fly;
        const int ya = min(max((int)fly, 0), Hh - 1), yb = min(max((int)fly + 1, 0), Hh - 1);
        for (int i = 0; i < kx; ++i) {
            const float px = ((float)gx + ((float)i + 0.5f) / (float)kx) * fx - 0.5f;
            const float flx = floorf(px);
            const float ax = px - flx;
            const int xa = min(max((int)flx, 0), W - 1), xb = min(max((int)flx + 1, 0), W - 1);
#pragma unroll
            for (int p = 0; p < 5; ++p) {
                const float* c = canvas + p * n;
                const float a = c[(size_t)ya * W + xa] * (1.f - ax) + c[(size_t)ya * W + xb] * ax;
                const float b = c[(size_t)yb * W + xa] * (1.f - ax) + c[(size_t)yb * W + xb] * ax;
                s[p] += a * (1.f - ay) + b * ay;
            }
        }
    }
    const float inv = 1.f / (float)(kx * ky);
#pragma unroll
    for (int p = 0; p < 5; ++p) grid[p * gn + (size_t)gy * cw + gx] = s[p] * inv;
}

__global__ void k_lag0(const float* __restrict__ a, const float* __restrict__ b, int n, double* out) {
    __shared__ double sh[32];
    double acc = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        acc += (double)a[i] * (double)b[i];
    acc = block_sum(acc, sh);
    if (threadIdx.x == 0) atomicAdd(out, acc);
}

}  // namespace

// ── launchers ────────────────────────────────────────────────────────────────────────────────

cudaError_t warp_stack(const float* stack, int w, int h, const float hi[9], bool ok, int W, int Hh, float* canvas,
                       cudaStream_t st) {
    Mat9f m;
    for (int i = 0; i < 9; ++i) m.m[i] = hi[i];
    dim3 b(32, 8), g((W + 31) / 32, (Hh + 7) / 8);
    k_warp_stack<<<g, b, 0, st>>>(stack, w, h, m, ok ? 1 : 0, W, Hh, canvas);
    return cudaGetLastError();
}

cudaError_t paste_stack(const float* stack, int w, int h, int ox, int oy, int W, int Hh, float* canvas,
                        cudaStream_t st) {
    dim3 b(32, 8), g((W + 31) / 32, (Hh + 7) / 8);
    k_paste_stack<<<g, b, 0, st>>>(stack, w, h, ox, oy, W, Hh, canvas);
    return cudaGetLastError();
}

cudaError_t resample_grid(const float* canvas, int W, int Hh, int cw, int ch, float* grid, cudaStream_t st) {
    dim3 b(32, 8), g((cw + 31) / 32, (ch + 7) / 8);
    k_resample<<<g, b, 0, st>>>(canvas, W, Hh, cw, ch, grid);
    return cudaGetLastError();
}

cudaError_t lag0_count(const float* a, const float* b, int cw, int ch, double* out, cudaStream_t st) {
    cudaMemsetAsync(out, 0, sizeof(double), st);
    const int n = cw * ch;
    int blocks = (n + 255) / 256;
    if (blocks > 296) blocks = 296;
    k_lag0<<<blocks, 256, 0, st>>>(a, b, n, out);
    return cudaGetLastError();
}

namespace {

// A pass with the line policy of its length: a compile-time line where some unit carries one,
// the runtime mixed-radix plan otherwise.
cudaError_t dispatch_pass(Pass p, const LinePlan& L, const PassArgs& a, cudaStream_t st) {
    cudaError_t e = cudaSuccess;
    if (pass_lines_a(p, L, a, st, &e) || pass_lines_b(p, L, a, st, &e) || pass_lines_c(p, L, a, st, &e)) return e;
    switch (L.n) {
        case 1024: return run_fixed<1024, true>(p, L.tw, a, st);
        case 2048: return run_fixed<2048, true>(p, L.tw, a, st);
        default: break;
    }
    const GenericLine f{L};
    switch (p) {
        case Pass::FwdRows: return run_pass<Pass::FwdRows, GenericLine, true>(f, a, st);
        case Pass::FwdCols: return run_pass<Pass::FwdCols, GenericLine, true>(f, a, st);
        case Pass::InvCols: return run_pass<Pass::InvCols, GenericLine, true>(f, a, st);
        default: return run_pass<Pass::Rows, GenericLine, true>(f, a, st);
    }
}

PassArgs pass_args(const MapGeom& g, const CorrPlanDev& plan, int batch) {
    PassArgs a;
    a.g = g;
    a.plan = &plan;
    a.batch = batch;
    return a;
}

}  // namespace

cudaError_t forward_rows(const float* grid, const MapGeom& g, const CorrPlanDev& plan, const LinePlan& row,
                         float2* half, cudaStream_t st, int batch, size_t grid_stride, size_t half_stride) {
    PassArgs a = pass_args(g, plan, batch);
    a.grid = grid;
    a.grid_stride = grid_stride;
    a.half = half;
    a.half_stride = half_stride;
    return dispatch_pass(Pass::FwdRows, row, a, st);
}

cudaError_t forward_cols(float2* half, const MapGeom& g, const CorrPlanDev& plan, const LinePlan& col,
                         cudaStream_t st, int batch) {
    PassArgs a = pass_args(g, plan, batch);
    a.half = half;
    return dispatch_pass(Pass::FwdCols, col, a, st);
}

cudaError_t forward_cols_generic(float2* half, const MapGeom& g, const CorrPlanDev& plan, const LinePlan& col,
                                 cudaStream_t st) {
    PassArgs a = pass_args(g, plan, 1);
    a.half = half;
    return run_pass<Pass::FwdCols, GenericLine, true>(GenericLine{col}, a, st);
}

cudaError_t inverse_columns(const float2* ha, const float2* hb, const MapGeom& g, const CorrPlanDev& plan,
                            const LinePlan& col, float2* Q, cudaStream_t st, int batch, size_t a_stride,
                            size_t b_stride, size_t q_stride, unsigned* fault) {
    static const bool pipe = [] {
        const char* v = getenv("ZCMIR_B200_INV_COLS");
        return v && std::string(v) == "pipe";
    }();
    if (!pipe && col.n == g.ny && inverse_columns_tma_supported(g, batch))
        return inverse_columns_tma(ha, hb, g, plan, col.tw, Q, st, fault);
    PassArgs a = pass_args(g, plan, batch);
    a.half = const_cast<float2*>(ha);
    a.half_stride = a_stride;
    a.half_b = hb;
    a.b_stride = b_stride;
    a.Q = Q;
    a.q_stride = q_stride;
    return dispatch_pass(Pass::InvCols, col, a, st);
}

size_t row_pass_smem(int L, int n_corr, int tl) {
    return (size_t)split_lines(tl) * padded_len(L) * sizeof(float2) + (size_t)n_corr * L * sizeof(float);
}

int row_split(int nx, int n_corr) {
    for (int S = 1; S <= 64; ++S) {
        if (nx % S) continue;
        const int L = nx / S;
        if (L > kMaxLine) continue;
        const int tl = row_tl(L);
        if (tl > 512) continue;
        const size_t sm = S == 1 ? multi_row_smem(L, n_corr, tl, 1) : row_pass_smem(L, n_corr, tl);
        if (sm <= kRowSmem) return S;
    }
    return 0;
}

cudaError_t inverse_rows_score(const float2* Q, const MapGeom& g, const CorrPlanDev& plan, const LinePlan& line,
                               int S, const float2* tw_nx, const CombineParams& cp, const double* n00, float* map,
                               unsigned long long* best, float* zero, cudaStream_t st, int batch, size_t q_stride,
                               size_t map_stride) {
    PassArgs a = pass_args(g, plan, batch);
    a.Q = const_cast<float2*>(Q);
    a.q_stride = q_stride;
    a.S = S;
    a.tw_nx = tw_nx;
    a.cp = &cp;
    a.n00 = n00;
    a.map = map;
    a.map_stride = map_stride;
    a.best = best;
    a.zero = zero;
    return dispatch_pass(Pass::Rows, line, a, st);
}

}  // namespace zc
