// A 2-D convolutional pose proposal on the tensor cores: BF16 operands, FP32 accumulation.
//
// Network (input: a pair's two 128 × 128 feature stacks, 4 planes each, as 8 channels, NHWC):
//   conv 3×3 stride 2 pad 1, 8 → 32 (64²), ReLU; 32 → 64 (32²), ReLU; 64 → 64 (16²), ReLU;
//   64 → 128 (8²), ReLU; the mean over the 8 × 8 positions; a linear layer 128 → 216 logits
//   (24 rotation bins × 9 log-scale bins, index 9·rotation + scale); softmax cross-entropy.
// Parameters, float32 masters in this order: W1 [32][3][3][8], b1, W2 [64][3][3][32], b2,
// W3 [64][3][3][64], b3, W4 [128][3][3][64], b4, Wfc [216][128], bfc.
//
// Precision: every weight is used rounded to BF16; activations are stored in BF16 after each
// ReLU; the backward pass rounds each layer's pre-activation gradient to BF16 before its two
// products; every product is summed in FP32 by mma.sync m16n8k16 (BF16 in, FP32 accumulate).
// The head (mean, linear layer, softmax) runs in FP32 on the CUDA cores with the BF16-rounded
// weights. Adam keeps float32 masters and moments.
//
// Each convolution, its input gradient and its weight gradient are one implicit GEMM kernel
// (k_gemm) with a different gather: output pixels × output channels over (tap, input channel);
// input pixels × input channels over (tap, output channel) with the stride-2 parity test; output
// channels × (tap, input channel) over pixels, split over blocks and summed with FP32 atomics.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "zcmir_b200.h"

namespace {

using bf16 = __nv_bfloat16;

constexpr int kIn = 128, kC0 = 8, kBins = 216, kFeat = 128;
constexpr int kCh[5] = {8, 32, 64, 64, 128};
constexpr int kSide[5] = {128, 64, 32, 16, 8};  // spatial side of layer l's input (l = 0..3) and the last output

constexpr int wsize(int l) { return kCh[l + 1] * 9 * kCh[l]; }
constexpr int woff(int l) {
    int o = 0;
    for (int i = 0; i < l; ++i) o += wsize(i) + kCh[i + 1];
    return o;
}
constexpr int kFcW = woff(4), kFcB = kFcW + kBins * kFeat, kNParams = kFcB + kBins;

// ── the GEMM: C[M][N] = Σ_k A(m, k) · B(n, k), BF16 operands from gather functors ────────────

constexpr int BM = 64, BN = 64, BK = 32, BKP = BK + 8, kThreads = 128;

__device__ __forceinline__ void mma16816(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Block: 4 warps over a 64 × 64 tile of C, warp w rows 16w..16w+15 × all 64 columns (8 n-tiles).
// K in steps of 32 from blockIdx.z · kspan (split K: each z adds its part through epi).
// Operands are staged 8 BF16 values (16 bytes) at a time from the gather's run8(row, k): 8
// consecutive k (AKF / BKF true: the row's channels of one tap, contiguous in NHWC) or 8
// consecutive rows (false: the output channels of one pixel). So K and kspan are multiples of 8
// when the run is along k, M (or N) a multiple of 8 when it is along the rows.
__device__ __forceinline__ uint4 zero8() { return make_uint4(0u, 0u, 0u, 0u); }

template <bool KF, int R, class L>
__device__ __forceinline__ void stage(bf16 (&S)[R][BKP], const L& l, int r0, int nr, int k0, int ke, int tid) {
    if constexpr (KF) {
#pragma unroll
        for (int i = tid; i < R * BK / 8; i += kThreads) {
            const int r = i / (BK / 8), cg = i % (BK / 8);
            const int row = r0 + r, k = k0 + cg * 8;
            *reinterpret_cast<uint4*>(&S[r][cg * 8]) = (row < nr && k < ke) ? l.run8(row, k) : zero8();
        }
    } else {
#pragma unroll
        for (int i = tid; i < R * BK / 8; i += kThreads) {
            const int c = i / (R / 8), rg = i % (R / 8);
            const int row = r0 + rg * 8, k = k0 + c;
            const uint4 v = (row < nr && k < ke) ? l.run8(row, k) : zero8();
            const bf16* e = reinterpret_cast<const bf16*>(&v);
#pragma unroll
            for (int j = 0; j < 8; ++j) S[rg * 8 + j][c] = e[j];
        }
    }
}
template <bool AKF, bool BKF, class LA, class LB, class EPI>
__global__ void __launch_bounds__(kThreads) k_gemm(int M, int N, int K, int kspan, LA la, LB lb, EPI epi) {
    __shared__ __align__(16) bf16 As[BM][BKP];
    __shared__ __align__(16) bf16 Bs[BN][BKP];
    const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
    const int kb = blockIdx.z * kspan, ke = min(K, kb + kspan);
    float acc[8][4] = {};
    const int g = lane >> 2, q = lane & 3;
    for (int k0 = kb; k0 < ke; k0 += BK) {
        stage<AKF>(As, la, m0, M, k0, ke, tid);
        stage<BKF>(Bs, lb, n0, N, k0, ke, tid);
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < BK; kk += 16) {
            uint32_t a[4];
            const int r = 16 * w + g, c = kk + 2 * q;
            a[0] = *reinterpret_cast<const uint32_t*>(&As[r][c]);
            a[1] = *reinterpret_cast<const uint32_t*>(&As[r + 8][c]);
            a[2] = *reinterpret_cast<const uint32_t*>(&As[r][c + 8]);
            a[3] = *reinterpret_cast<const uint32_t*>(&As[r + 8][c + 8]);
#pragma unroll
            for (int nt = 0; nt < 8; ++nt) {
                const uint32_t b0 = *reinterpret_cast<const uint32_t*>(&Bs[nt * 8 + g][c]);
                const uint32_t b1 = *reinterpret_cast<const uint32_t*>(&Bs[nt * 8 + g][c + 8]);
                mma16816(acc[nt], a, b0, b1);
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int nt = 0; nt < 8; ++nt)
#pragma unroll
        for (int h = 0; h < 4; ++h) {
            const int m = m0 + 16 * w + g + (h >> 1) * 8, n = n0 + nt * 8 + 2 * q + (h & 1);
            if (m < M && n < N) epi(m, n, acc[nt][h]);
        }
}

// ── gathers and epilogues of the three convolution products ────────────────────────────────

struct ConvShape {
    int B, H, W, Ci, Co;  // input B × H × W × Ci; output B × H/2 × W/2 × Co
    __device__ __forceinline__ int OH() const { return H >> 1; }
    __device__ __forceinline__ int OW() const { return W >> 1; }
};

// patch element (output pixel m, column k = tap·Ci + ci) of a stride-2, pad-1 3×3 convolution
// (8 consecutive k from a multiple of 8: 8 channels of one tap, Ci a multiple of 8)
struct Patch {
    const bf16* x;
    ConvShape s;
    __device__ __forceinline__ uint4 run8(int m, int k) const {
        const int ohw = s.OH() * s.OW(), b = m / ohw, p = m - b * ohw, oy = p / s.OW(), ox = p - oy * s.OW();
        const int tap = k / s.Ci, ci = k - tap * s.Ci, ky = tap / 3, kx = tap - ky * 3;
        const int iy = 2 * oy + ky - 1, ix = 2 * ox + kx - 1;
        if (iy < 0 || iy >= s.H || ix < 0 || ix >= s.W) return zero8();
        return *reinterpret_cast<const uint4*>(x + (((size_t)b * s.H + iy) * s.W + ix) * s.Ci + ci);
    }
};
struct RowMajor {  // a[r · ld + k .. + 7], ld a multiple of 8
    const bf16* a;
    int ld;
    __device__ __forceinline__ uint4 run8(int r, int k) const {
        return *reinterpret_cast<const uint4*>(a + (size_t)r * ld + k);
    }
};
// forward epilogue: bias, ReLU, BF16 store
struct FwdEpi {
    const float* bias;
    bf16* y;
    int Co;
    __device__ __forceinline__ void operator()(int m, int n, float v) const {
        y[(size_t)m * Co + n] = __float2bfloat16_rn(fmaxf(v + bias[n], 0.f));
    }
};
// input-gradient gather: (input pixel m, column k = tap·Co + co) of the pre-activation gradient
// dz of the output, where the output pixel (iy + 1 − ky, ix + 1 − kx) / 2 exists
struct DataGather {
    const bf16* dz;
    ConvShape s;
    __device__ __forceinline__ uint4 run8(int m, int k) const {
        const int hw = s.H * s.W, b = m / hw, p = m - b * hw, iy = p / s.W, ix = p - iy * s.W;
        const int tap = k / s.Co, co = k - tap * s.Co, ky = tap / 3, kx = tap - ky * 3;
        const int ty = iy + 1 - ky, tx = ix + 1 - kx;
        if (ty < 0 || tx < 0 || (ty & 1) || (tx & 1)) return zero8();
        const int oy = ty >> 1, ox = tx >> 1;
        if (oy >= s.OH() || ox >= s.OW()) return zero8();
        return *reinterpret_cast<const uint4*>(dz + (((size_t)b * s.OH() + oy) * s.OW() + ox) * s.Co + co);
    }
};
// input-gradient epilogue: through the ReLU that produced the input (mask: input > 0), BF16
struct DataEpi {
    const bf16* x;
    bf16* dzp;
    int Ci;
    __device__ __forceinline__ void operator()(int m, int n, float v) const {
        const size_t i = (size_t)m * Ci + n;
        dzp[i] = __float2bfloat16_rn(__bfloat162float(x[i]) > 0.f ? v : 0.f);
    }
};
// weight-gradient operands, 8 consecutive rows of one pixel: A(co .. co + 7, pixel) =
// dz[pixel][co ..]; B(tap·Ci + ci .. + 7, pixel) = the patch's 8 channels
struct DzT {
    const bf16* dz;
    int Co;
    __device__ __forceinline__ uint4 run8(int co, int px) const {
        return *reinterpret_cast<const uint4*>(dz + (size_t)px * Co + co);
    }
};
struct PatchT {
    Patch p;
    __device__ __forceinline__ uint4 run8(int n, int px) const { return p.run8(px, n); }
};
struct AtomicEpi {
    float* dw;
    int N;
    __device__ __forceinline__ void operator()(int m, int n, float v) const { atomicAdd(&dw[(size_t)m * N + n], v); }
};

// ── small kernels: weights, head, loss, Adam ────────────────────────────────────────────────

int blocks(size_t m) { return (int)((m + 255) / 256); }

// BF16 copies of one layer's weights: wb[co][tap][ci] and the transposed wt[ci][tap][co]
__global__ void k_wcast(const float* __restrict__ w, int Co, int Ci, bf16* __restrict__ wb, bf16* __restrict__ wt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= Co * 9 * Ci) return;
    const int ci = i % Ci, tap = (i / Ci) % 9, co = i / (9 * Ci);
    const bf16 v = __float2bfloat16_rn(w[i]);
    wb[i] = v;
    if (wt) wt[((size_t)ci * 9 + tap) * Co + co] = v;
}

// h[b][c] = mean over the 8 × 8 positions of a4[b][·][·][c]
__global__ void k_gap(const bf16* __restrict__ a4, int B, float* __restrict__ h) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B * kFeat) return;
    const int b = i / kFeat, c = i - b * kFeat;
    float s = 0.f;
    for (int p = 0; p < 64; ++p) s += __bfloat162float(a4[((size_t)b * 64 + p) * kFeat + c]);
    h[i] = s * (1.f / 64.f);
}

// logits[b][o] = bfc[o] + Σ_c bf16(Wfc[o][c]) h[b][c]
__global__ void k_fc(const float* __restrict__ h, const float* __restrict__ W, const float* __restrict__ bias, int B,
                     float* __restrict__ z) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B * kBins) return;
    const int b = i / kBins, o = i - b * kBins;
    float s = bias[o];
    for (int c = 0; c < kFeat; ++c) s = fmaf(__bfloat162float(__float2bfloat16_rn(W[o * kFeat + c])), h[b * kFeat + c], s);
    z[i] = s;
}

// per sample: softmax of its 216 logits; dz = (p − onehot) / B; loss sum (sum of −log p_label / B)
__global__ void k_xent(const float* __restrict__ z, const int* __restrict__ lab, int B, float* __restrict__ dz,
                       float* __restrict__ loss) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    const float* zb = z + (size_t)b * kBins;
    float mx = -3.4e38f;
    for (int o = 0; o < kBins; ++o) mx = fmaxf(mx, zb[o]);
    float s = 0.f;
    for (int o = 0; o < kBins; ++o) s += expf(zb[o] - mx);
    const float ls = logf(s) + mx;
    for (int o = 0; o < kBins; ++o) dz[(size_t)b * kBins + o] = (expf(zb[o] - ls) - (o == lab[b] ? 1.f : 0.f)) / B;
    atomicAdd(loss, (ls - zb[lab[b]]) / B);
}

// head backward: dWfc[o][c] = Σ_b dz[b][o] h[b][c]; dbfc[o] = Σ_b dz[b][o]
__global__ void k_fc_bwd_w(const float* __restrict__ dz, const float* __restrict__ h, int B, float* __restrict__ dW,
                           float* __restrict__ db) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < kBins * kFeat) {
        const int o = i / kFeat, c = i - o * kFeat;
        float s = 0.f;
        for (int b = 0; b < B; ++b) s = fmaf(dz[b * kBins + o], h[b * kFeat + c], s);
        dW[i] = s;
    } else if (i < kBins * kFeat + kBins) {
        const int o = i - kBins * kFeat;
        float s = 0.f;
        for (int b = 0; b < B; ++b) s += dz[b * kBins + o];
        db[o] = s;
    }
}

// dz4[b][p][c] = bf16( [a4 > 0] · (Σ_o dz[b][o] bf16(Wfc[o][c])) / 64 )
__global__ void k_head_bwd(const float* __restrict__ dz, const float* __restrict__ W, const bf16* __restrict__ a4,
                           int B, bf16* __restrict__ dz4) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B * 64 * kFeat) return;
    const int c = i % kFeat, b = i / (64 * kFeat);
    float s = 0.f;
    for (int o = 0; o < kBins; ++o) s = fmaf(dz[b * kBins + o], __bfloat162float(__float2bfloat16_rn(W[o * kFeat + c])), s);
    dz4[i] = __float2bfloat16_rn(__bfloat162float(a4[i]) > 0.f ? s * (1.f / 64.f) : 0.f);
}

// db[co] = Σ over pixels of dz[px][co]
__global__ void k_bias_grad(const bf16* __restrict__ dz, size_t npx, int Co, float* __restrict__ db) {
    const int co = blockIdx.x;
    float s = 0.f;
    for (size_t p = threadIdx.x; p < npx; p += blockDim.x) s += __bfloat162float(dz[p * Co + co]);
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    __shared__ float part[32];
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.f;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += part[i];
        db[co] = t;
    }
}

__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       int n, float lr, float b1, float b2, float c1, float c2, float eps) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi, vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// batch gather: x[j] = all[idx[j]] (samples of kIn² · kC0 BF16), labels alike
__global__ void k_gather(const bf16* __restrict__ all, const int* __restrict__ lall, const uint32_t* __restrict__ idx,
                         int B, bf16* __restrict__ x, int* __restrict__ lab) {
    constexpr size_t per = (size_t)kIn * kIn * kC0;
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < (size_t)B * per / 8) {
        const size_t j = i / (per / 8), r = i - j * (per / 8);
        reinterpret_cast<uint4*>(x)[i] = reinterpret_cast<const uint4*>(all + (size_t)idx[j] * per)[r];
    }
    if (i < (size_t)B) lab[i] = lall[idx[i]];
}

// ── host: buffers and the passes ────────────────────────────────────────────────────────────

std::string g_err;

struct Net {
    int B = 0;
    float *params = nullptr, *grad = nullptr, *m = nullptr, *v = nullptr;
    bf16 *wb[4] = {}, *wt[4] = {};
    bf16 *act[5] = {};   // act[0]: input batch; act[l + 1]: layer l's ReLU output
    bf16 *dz[4] = {};    // dz[l]: layer l's pre-activation gradient
    float *h = nullptr, *z = nullptr, *dlog = nullptr, *loss = nullptr;
    int* lab = nullptr;
    cudaStream_t st = nullptr;

    bool ok(cudaError_t e, const char* what) {
        if (e == cudaSuccess) return true;
        g_err = std::string(what) + ": " + cudaGetErrorString(e);
        return false;
    }
    bool alloc(int batch, bool train) {
        B = batch;
        if (!ok(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "stream")) return false;
        const size_t np = kNParams;
        if (!ok(cudaMalloc(&params, np * 4), "params") || !ok(cudaMalloc(&grad, np * 4), "grad")) return false;
        if (train && (!ok(cudaMalloc(&m, np * 4), "adam") || !ok(cudaMalloc(&v, np * 4), "adam") ||
                      !ok(cudaMemsetAsync(m, 0, np * 4, st), "adam") || !ok(cudaMemsetAsync(v, 0, np * 4, st), "adam")))
            return false;
        for (int l = 0; l < 4; ++l) {
            if (!ok(cudaMalloc(&wb[l], (size_t)wsize(l) * 2), "weights") ||
                !ok(cudaMalloc(&wt[l], (size_t)wsize(l) * 2), "weights"))
                return false;
            if (!ok(cudaMalloc(&dz[l], (size_t)B * kSide[l + 1] * kSide[l + 1] * kCh[l + 1] * 2), "gradients"))
                return false;
        }
        for (int l = 0; l < 5; ++l)
            if (!ok(cudaMalloc(&act[l], (size_t)B * kSide[l] * kSide[l] * kCh[l] * 2), "activations")) return false;
        return ok(cudaMalloc(&h, (size_t)B * kFeat * 4), "head") && ok(cudaMalloc(&z, (size_t)B * kBins * 4), "head") &&
               ok(cudaMalloc(&dlog, (size_t)B * kBins * 4), "head") && ok(cudaMalloc(&loss, 4), "head") &&
               ok(cudaMalloc(&lab, (size_t)B * 4), "labels");
    }
    ~Net() {
        if (st) cudaStreamSynchronize(st);
        for (void* p : {(void*)params, (void*)grad, (void*)m, (void*)v, (void*)h, (void*)z, (void*)dlog, (void*)loss,
                        (void*)lab})
            if (p) cudaFree(p);
        for (int l = 0; l < 4; ++l)
            for (void* p : {(void*)wb[l], (void*)wt[l], (void*)dz[l]})
                if (p) cudaFree(p);
        for (bf16* p : act)
            if (p) cudaFree(p);
        if (st) cudaStreamDestroy(st);
    }
    ConvShape shape(int l) const { return ConvShape{B, kSide[l], kSide[l], kCh[l], kCh[l + 1]}; }

    bool cast_weights() {
        for (int l = 0; l < 4; ++l) {
            k_wcast<<<blocks(wsize(l)), 256, 0, st>>>(params + woff(l), kCh[l + 1], kCh[l], wb[l], l ? wt[l] : nullptr);
        }
        return ok(cudaGetLastError(), "weights");
    }
    // forward from act[0] (B samples) to logits z
    bool forward() {
        if (!cast_weights()) return false;
        for (int l = 0; l < 4; ++l) {
            const ConvShape s = shape(l);
            const int M = B * (s.H / 2) * (s.W / 2), N = s.Co, K = 9 * s.Ci;
            k_gemm<true, true><<<dim3((M + BM - 1) / BM, (N + BN - 1) / BN, 1), kThreads, 0, st>>>(
                M, N, K, K, Patch{act[l], s}, RowMajor{wb[l], K}, FwdEpi{params + woff(l) + wsize(l), act[l + 1], N});
        }
        k_gap<<<blocks((size_t)B * kFeat), 256, 0, st>>>(act[4], B, h);
        k_fc<<<blocks((size_t)B * kBins), 256, 0, st>>>(h, params + kFcW, params + kFcB, B, z);
        return ok(cudaGetLastError(), "forward");
    }
    // loss and gradient (into grad) for labels lab after forward()
    bool backward() {
        if (!ok(cudaMemsetAsync(loss, 0, 4, st), "backward") || !ok(cudaMemsetAsync(grad, 0, (size_t)kNParams * 4, st), "backward"))
            return false;
        k_xent<<<blocks(B), 256, 0, st>>>(z, lab, B, dlog, loss);
        k_fc_bwd_w<<<blocks(kBins * kFeat + kBins), 256, 0, st>>>(dlog, h, B, grad + kFcW, grad + kFcB);
        k_head_bwd<<<blocks((size_t)B * 64 * kFeat), 256, 0, st>>>(dlog, params + kFcW, act[4], B, dz[3]);
        for (int l = 3; l >= 0; --l) {
            const ConvShape s = shape(l);
            const int npx = B * (s.H / 2) * (s.W / 2), Kw = 9 * s.Ci;
            // weight gradient: M = Co, N = 9·Ci, K = pixels, split so that every SM has blocks
            const int tiles = ((s.Co + BM - 1) / BM) * ((Kw + BN - 1) / BN);
            int splits = std::max(1, std::min(npx / 256, (4 * 148 + tiles - 1) / tiles));
            const int kspan = ((npx + splits - 1) / splits + BK - 1) / BK * BK;
            splits = (npx + kspan - 1) / kspan;
            k_gemm<false, false><<<dim3((s.Co + BM - 1) / BM, (Kw + BN - 1) / BN, splits), kThreads, 0, st>>>(
                s.Co, Kw, npx, kspan, DzT{dz[l], s.Co}, PatchT{Patch{act[l], s}}, AtomicEpi{grad + woff(l), Kw});
            k_bias_grad<<<s.Co, 256, 0, st>>>(dz[l], (size_t)npx, s.Co, grad + woff(l) + wsize(l));
            if (l == 0) break;
            // input gradient through the previous layer's ReLU: M = input pixels, N = Ci, K = 9·Co
            const int M = B * s.H * s.W, K = 9 * s.Co;
            k_gemm<true, true><<<dim3((M + BM - 1) / BM, (s.Ci + BN - 1) / BN, 1), kThreads, 0, st>>>(
                M, s.Ci, K, K, DataGather{dz[l], s}, RowMajor{wt[l], K}, DataEpi{act[l], dz[l - 1], s.Ci});
        }
        return ok(cudaGetLastError(), "backward");
    }
    bool adam(int t, float lr) {
        const float b1 = 0.9f, b2 = 0.999f;
        k_adam<<<blocks(kNParams), 256, 0, st>>>(params, grad, m, v, kNParams, lr, b1, b2, 1.f - std::pow(b1, (float)t),
                                                 1.f - std::pow(b2, (float)t), 1e-8f);
        return ok(cudaGetLastError(), "adam");
    }
};

constexpr size_t kSample = (size_t)kIn * kIn * kC0;

int fail(const std::string& m) {
    g_err = m;
    return -1;
}

}  // namespace

extern "C" {

size_t zcb_cnn_nparams(void) { return kNParams; }

size_t zcb_cnn_error(char* buf, size_t cap) {
    if (buf && cap) {
        const size_t n = std::min(cap - 1, g_err.size());
        std::memcpy(buf, g_err.data(), n);
        buf[n] = 0;
    }
    return g_err.size();
}

int32_t zcb_cnn_forward(const float* params, size_t np, const uint16_t* x, uint32_t n, float* logits) {
    if (np != (size_t)kNParams) return fail("cnn_forward: expected " + std::to_string(kNParams) + " parameters");
    if (!params || !x || !logits || n == 0) return fail("cnn_forward: null input or empty batch");
    const int B = (int)std::min<uint32_t>(n, 256);
    Net net;
    if (!net.alloc(B, false)) return -1;
    if (!net.ok(cudaMemcpyAsync(net.params, params, np * 4, cudaMemcpyHostToDevice, net.st), "cnn_forward")) return -1;
    for (uint32_t b0 = 0; b0 < n; b0 += B) {
        const int nb = (int)std::min<uint32_t>(B, n - b0);
        net.B = nb;
        if (!net.ok(cudaMemcpyAsync(net.act[0], x + (size_t)b0 * kSample, (size_t)nb * kSample * 2, cudaMemcpyHostToDevice,
                                    net.st),
                    "cnn_forward") ||
            !net.forward() ||
            !net.ok(cudaMemcpyAsync(logits + (size_t)b0 * kBins, net.z, (size_t)nb * kBins * 4, cudaMemcpyDeviceToHost,
                                    net.st),
                    "cnn_forward") ||
            !net.ok(cudaStreamSynchronize(net.st), "cnn_forward"))
            return -1;
    }
    return 0;
}

int32_t zcb_cnn_grad(const float* params, size_t np, const uint16_t* x, const int32_t* labels, uint32_t n, float* loss,
                     float* grad) {
    if (np != (size_t)kNParams) return fail("cnn_grad: expected " + std::to_string(kNParams) + " parameters");
    if (!params || !x || !labels || !loss || !grad || n == 0 || n > 4096)
        return fail("cnn_grad: null input, or a batch outside 1..4096");
    for (uint32_t i = 0; i < n; ++i)
        if (labels[i] < 0 || labels[i] >= kBins) return fail("cnn_grad: label outside 0..215");
    Net net;
    if (!net.alloc((int)n, false)) return -1;
    if (!net.ok(cudaMemcpyAsync(net.params, params, np * 4, cudaMemcpyHostToDevice, net.st), "cnn_grad") ||
        !net.ok(cudaMemcpyAsync(net.act[0], x, (size_t)n * kSample * 2, cudaMemcpyHostToDevice, net.st), "cnn_grad") ||
        !net.ok(cudaMemcpyAsync(net.lab, labels, (size_t)n * 4, cudaMemcpyHostToDevice, net.st), "cnn_grad") ||
        !net.forward() || !net.backward() ||
        !net.ok(cudaMemcpyAsync(grad, net.grad, np * 4, cudaMemcpyDeviceToHost, net.st), "cnn_grad") ||
        !net.ok(cudaMemcpyAsync(loss, net.loss, 4, cudaMemcpyDeviceToHost, net.st), "cnn_grad") ||
        !net.ok(cudaStreamSynchronize(net.st), "cnn_grad"))
        return -1;
    return 0;
}

int32_t zcb_cnn_train(float* params, size_t np, const uint16_t* x, const int32_t* labels, uint32_t n, uint32_t batch,
                      uint32_t steps, float lr, uint64_t seed, float* losses, float* ms_per_step) {
    if (np != (size_t)kNParams) return fail("cnn_train: expected " + std::to_string(kNParams) + " parameters");
    if (!params || !x || !labels || n == 0 || batch == 0 || batch > 1024 || steps == 0)
        return fail("cnn_train: null input, no samples, no steps, or a batch outside 1..1024");
    for (uint32_t i = 0; i < n; ++i)
        if (labels[i] < 0 || labels[i] >= kBins) return fail("cnn_train: label outside 0..215");
    Net net;
    if (!net.alloc((int)batch, true)) return -1;
    bf16* all = nullptr;
    int* lall = nullptr;
    uint32_t* idx = nullptr;
    float* dlosses = nullptr;
    auto cleanup = [&] {
        cudaStreamSynchronize(net.st);
        for (void* p : {(void*)all, (void*)lall, (void*)idx, (void*)dlosses})
            if (p) cudaFree(p);
    };
    std::vector<uint32_t> hidx((size_t)steps * batch);
    uint64_t s = seed * 6364136223846793005ull + 1442695040888963407ull;
    for (auto& v : hidx) {  // a 64-bit LCG's high bits: the batches, with replacement
        s = s * 6364136223846793005ull + 1442695040888963407ull;
        v = (uint32_t)((s >> 33) % n);
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    bool good = net.ok(cudaMalloc(&all, (size_t)n * kSample * 2), "cnn_train: samples") &&
                net.ok(cudaMalloc(&lall, (size_t)n * 4), "cnn_train") &&
                net.ok(cudaMalloc(&idx, hidx.size() * 4), "cnn_train") &&
                net.ok(cudaMalloc(&dlosses, (size_t)steps * 4), "cnn_train") &&
                net.ok(cudaMemcpyAsync(all, x, (size_t)n * kSample * 2, cudaMemcpyHostToDevice, net.st), "cnn_train") &&
                net.ok(cudaMemcpyAsync(lall, labels, (size_t)n * 4, cudaMemcpyHostToDevice, net.st), "cnn_train") &&
                net.ok(cudaMemcpyAsync(idx, hidx.data(), hidx.size() * 4, cudaMemcpyHostToDevice, net.st), "cnn_train") &&
                net.ok(cudaMemcpyAsync(net.params, params, np * 4, cudaMemcpyHostToDevice, net.st), "cnn_train") &&
                net.ok(cudaEventCreate(&e0), "cnn_train") && net.ok(cudaEventCreate(&e1), "cnn_train") &&
                net.ok(cudaEventRecord(e0, net.st), "cnn_train");
    for (uint32_t t = 0; good && t < steps; ++t) {
        const size_t per = kSample * batch / 8;
        k_gather<<<blocks(std::max(per, (size_t)batch)), 256, 0, net.st>>>(all, lall, idx + (size_t)t * batch, (int)batch,
                                                                        net.act[0], net.lab);
        good = net.forward() && net.backward() && net.adam((int)t + 1, lr) &&
               net.ok(cudaMemcpyAsync(dlosses + t, net.loss, 4, cudaMemcpyDeviceToDevice, net.st), "cnn_train");
    }
    float ms = 0.f;
    good = good && net.ok(cudaEventRecord(e1, net.st), "cnn_train") && net.ok(cudaEventSynchronize(e1), "cnn_train") &&
           net.ok(cudaEventElapsedTime(&ms, e0, e1), "cnn_train") &&
           net.ok(cudaMemcpy(params, net.params, np * 4, cudaMemcpyDeviceToHost), "cnn_train") &&
           (!losses || net.ok(cudaMemcpy(losses, dlosses, (size_t)steps * 4, cudaMemcpyDeviceToHost), "cnn_train"));
    if (ms_per_step) *ms_per_step = ms / (float)steps;
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cleanup();
    return good ? 0 : -1;
}

}  // extern "C"
