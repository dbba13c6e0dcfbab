// The learned pose proposal's network on the GPU: forward, backward and Adam for a small circular
// 1-D convolutional network over a coarse sweep landscape (the best map peaks of 36 rotations ×
// 3 scales), whose output is a distribution over the plain sweep's full rotation × scale grid.
//
// Layers (parameters in this order, float32): conv 6 → 32 (k 5), ReLU, conv 32 → 32 (k 5), ReLU,
// conv 32 → 90 (k 3); every convolution circular over the 36 rotations (the landscape wraps at
// 360°), with a bias. The last layer's [n][90][36] is read position-major as 3240 logits per
// sample, index 90·i + o: position i (the coarse rotation −180° + 10·i°), channel o = 9·dθ + s
// (fine rotation −180° + 10·i − 5 + dθ degrees, fine scale s of 9).
// The loss is the softmax cross-entropy over the 3240 logits.
//
// The network is 15 k parameters and a batch is 128 × 36 positions: every kernel is a plain
// float32 loop on the CUDA cores (one thread per output element), far below the sizes at which
// tensor-core tiles pay.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <utility>
#include <vector>

#include "zcmir_b200.h"

namespace {

constexpr int kL = 36, kC0 = 6, kC1 = 32, kC2 = 32, kC3 = 90, kK1 = 5, kK2 = 5, kK3 = 3;
constexpr int kNW1 = kC1 * kC0 * kK1, kNW2 = kC2 * kC1 * kK2, kNW3 = kC3 * kC2 * kK3;
constexpr int kNParams = kNW1 + kC1 + kNW2 + kC2 + kNW3 + kC3;
constexpr int kOut = kC3 * kL;

// y[n][co][l] = b[co] + Σ_ci Σ_k w[co][ci][k] x[n][ci][(l + k − K/2) mod L]
__global__ void k_conv_fwd(const float* __restrict__ x, const float* __restrict__ w, const float* __restrict__ b,
                           int n, int ci, int co, int K, int relu, float* __restrict__ y) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * co * kL) return;
    const int l = i % kL, c = (i / kL) % co, s = i / (kL * co);
    float acc = b[c];
    const float* xs = x + (size_t)s * ci * kL;
    const float* wc = w + (size_t)c * ci * K;
    for (int j = 0; j < ci; ++j)
        for (int k = 0; k < K; ++k) {
            const int m = (l + k - K / 2 + kL) % kL;
            acc = fmaf(wc[j * K + k], xs[j * kL + m], acc);
        }
    y[i] = relu ? fmaxf(acc, 0.f) : acc;
}

// dx[n][ci][m] = Σ_co Σ_k w[co][ci][k] dy[n][co][(m − k + K/2) mod L]
__global__ void k_conv_bwd_data(const float* __restrict__ dy, const float* __restrict__ w, int n, int ci, int co,
                                int K, float* __restrict__ dx) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * ci * kL) return;
    const int m = i % kL, j = (i / kL) % ci, s = i / (kL * ci);
    float acc = 0.f;
    const float* ds = dy + (size_t)s * co * kL;
    for (int c = 0; c < co; ++c)
        for (int k = 0; k < K; ++k) {
            const int l = (m - k + K / 2 + 2 * kL) % kL;
            acc = fmaf(w[((size_t)c * ci + j) * K + k], ds[c * kL + l], acc);
        }
    dx[i] = acc;
}

// dw[co][ci][k] = Σ_n Σ_l dy[n][co][l] x[n][ci][(l + k − K/2) mod L]; db[co] = Σ_n Σ_l dy[n][co][l]
__global__ void k_conv_bwd_w(const float* __restrict__ dy, const float* __restrict__ x, int n, int ci, int co, int K,
                             float* __restrict__ dw, float* __restrict__ db) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int nw = co * ci * K;
    if (i < nw) {
        const int k = i % K, j = (i / K) % ci, c = i / (K * ci);
        float acc = 0.f;
        for (int s = 0; s < n; ++s) {
            const float* ds = dy + ((size_t)s * co + c) * kL;
            const float* xs = x + ((size_t)s * ci + j) * kL;
            for (int l = 0; l < kL; ++l) acc = fmaf(ds[l], xs[(l + k - K / 2 + kL) % kL], acc);
        }
        dw[i] = acc;
    } else if (i < nw + co) {
        const int c = i - nw;
        float acc = 0.f;
        for (int s = 0; s < n; ++s) {
            const float* ds = dy + ((size_t)s * co + c) * kL;
            for (int l = 0; l < kL; ++l) acc += ds[l];
        }
        db[c] = acc;
    }
}

// [n][a][b] → [n][b][a]: the last layer's channel-major output as position-major logits (index
// 90·i + o), and the logits' gradient back
__global__ void k_transpose(const float* __restrict__ in, int n, int a, int b, float* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * a * b) return;
    const int s = i / (a * b), r = i - s * a * b, u = r / b, w = r - u * b;
    out[(size_t)s * a * b + (size_t)w * a + u] = in[i];
}

// the ReLU's gradient in place: dy = 0 where the layer's output was clipped
__global__ void k_relu_bwd(float* __restrict__ dy, const float* __restrict__ y, int m) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m && !(y[i] > 0.f)) dy[i] = 0.f;
}

// per sample: loss = log Σ exp(z) − z[label]; dz = (softmax(z) − onehot) / n (one block per sample)
__global__ void k_softmax_xent(const float* __restrict__ z, const int* __restrict__ labels, int n, float* __restrict__ loss,
                               float* __restrict__ dz) {
    __shared__ float red[256];
    const int s = blockIdx.x;
    const float* zs = z + (size_t)s * kOut;
    float mx = -3.4e38f;
    for (int i = threadIdx.x; i < kOut; i += blockDim.x) mx = fmaxf(mx, zs[i]);
    red[threadIdx.x] = mx;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] = fmaxf(red[threadIdx.x], red[threadIdx.x + o]);
        __syncthreads();
    }
    mx = red[0];
    __syncthreads();
    float se = 0.f;
    for (int i = threadIdx.x; i < kOut; i += blockDim.x) se += expf(zs[i] - mx);
    red[threadIdx.x] = se;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    se = red[0];
    const int lab = labels[s];
    if (threadIdx.x == 0) loss[s] = logf(se) + mx - zs[lab];
    if (dz)
        for (int i = threadIdx.x; i < kOut; i += blockDim.x)
            dz[(size_t)s * kOut + i] = (expf(zs[i] - mx) / se - (i == lab ? 1.f : 0.f)) / (float)n;
}

// Adam (bias-corrected), one thread per parameter
__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       int np, float lr, float b1, float b2, float eps, float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np) return;
    const float gi = g[i];
    m[i] = b1 * m[i] + (1.f - b1) * gi;
    v[i] = b2 * v[i] + (1.f - b2) * gi * gi;
    p[i] -= lr * (m[i] / c1) / (sqrtf(v[i] / c2) + eps);
}

// a minibatch gathered from the whole set: sample k of the batch is sample idx[k]
__global__ void k_gather(const float* __restrict__ xall, const int* __restrict__ lall, const uint32_t* __restrict__ idx,
                         int batch, float* __restrict__ x, int* __restrict__ lab) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= batch * kC0 * kL) return;
    const int k = i / (kC0 * kL), r = i - k * kC0 * kL;
    x[i] = xall[(size_t)idx[k] * kC0 * kL + r];
    if (r == 0) lab[k] = lall[idx[k]];
}

int blocks(int m) { return (m + 255) / 256; }

// Device buffers of one batch size: parameters, gradients, Adam moments, activations and their
// gradients (zeroed on the stream that uses them).
struct Net {
    float *base = nullptr, *p = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
    float *x = nullptr, *a1 = nullptr, *a2 = nullptr, *a3 = nullptr, *z = nullptr, *d1 = nullptr, *d2 = nullptr,
          *d3 = nullptr, *dz = nullptr;
    float* loss = nullptr;
    int* lab = nullptr;
    bool alloc(int n, cudaStream_t st) {
        const size_t f = (size_t)4 * kNParams + (size_t)n * (kC0 + 2 * kC1 + 2 * kC2) * kL + 4 * (size_t)n * kOut + n;
        if (cudaMalloc(&base, f * sizeof(float)) != cudaSuccess) return false;
        if (cudaMalloc(&lab, (size_t)n * sizeof(int)) != cudaSuccess) {
            cudaFree(base);
            base = nullptr;
            return false;
        }
        cudaMemsetAsync(base, 0, f * sizeof(float), st);
        float* q = base;
        auto take = [&](size_t k) {
            float* r = q;
            q += k;
            return r;
        };
        p = take(kNParams), g = take(kNParams), m = take(kNParams), v = take(kNParams);
        x = take((size_t)n * kC0 * kL), a1 = take((size_t)n * kC1 * kL), d1 = take((size_t)n * kC1 * kL);
        a2 = take((size_t)n * kC2 * kL), d2 = take((size_t)n * kC2 * kL);
        a3 = take((size_t)n * kOut), z = take((size_t)n * kOut), d3 = take((size_t)n * kOut), dz = take((size_t)n * kOut);
        loss = take(n);
        return true;
    }
    void release() {
        cudaFree(base);
        cudaFree(lab);
        base = nullptr;
        lab = nullptr;
    }
    float* w1() const { return p; }
    float* b1() const { return p + kNW1; }
    float* w2() const { return p + kNW1 + kC1; }
    float* b2() const { return p + kNW1 + kC1 + kNW2; }
    float* w3() const { return p + kNW1 + kC1 + kNW2 + kC2; }
    float* b3() const { return p + kNW1 + kC1 + kNW2 + kC2 + kNW3; }
    // gradient slots, the parameters' layout
    float* gw(int layer) const { return g + (layer == 0 ? 0 : layer == 1 ? kNW1 + kC1 : kNW1 + kC1 + kNW2 + kC2); }
    float* gb(int layer) const { return gw(layer) + (layer == 0 ? kNW1 : layer == 1 ? kNW2 : kNW3); }

    void forward(int n, cudaStream_t st) const {
        k_conv_fwd<<<blocks(n * kC1 * kL), 256, 0, st>>>(x, w1(), b1(), n, kC0, kC1, kK1, 1, a1);
        k_conv_fwd<<<blocks(n * kC2 * kL), 256, 0, st>>>(a1, w2(), b2(), n, kC1, kC2, kK2, 1, a2);
        k_conv_fwd<<<blocks(n * kOut), 256, 0, st>>>(a2, w3(), b3(), n, kC2, kC3, kK3, 0, a3);
        k_transpose<<<blocks(n * kOut), 256, 0, st>>>(a3, n, kC3, kL, z);
    }
    // the loss per sample into `loss`, the mean loss's gradient into g
    void backward(int n, cudaStream_t st) const {
        k_softmax_xent<<<n, 256, 0, st>>>(z, lab, n, loss, dz);
        k_transpose<<<blocks(n * kOut), 256, 0, st>>>(dz, n, kL, kC3, d3);
        k_conv_bwd_w<<<blocks(kNW3 + kC3), 256, 0, st>>>(d3, a2, n, kC2, kC3, kK3, gw(2), gb(2));
        k_conv_bwd_data<<<blocks(n * kC2 * kL), 256, 0, st>>>(d3, w3(), n, kC2, kC3, kK3, d2);
        k_relu_bwd<<<blocks(n * kC2 * kL), 256, 0, st>>>(d2, a2, n * kC2 * kL);
        k_conv_bwd_w<<<blocks(kNW2 + kC2), 256, 0, st>>>(d2, a1, n, kC1, kC2, kK2, gw(1), gb(1));
        k_conv_bwd_data<<<blocks(n * kC1 * kL), 256, 0, st>>>(d2, w2(), n, kC1, kC2, kK2, d1);
        k_relu_bwd<<<blocks(n * kC1 * kL), 256, 0, st>>>(d1, a1, n * kC1 * kL);
        k_conv_bwd_w<<<blocks(kNW1 + kC1), 256, 0, st>>>(d1, x, n, kC0, kC1, kK1, gw(0), gb(0));
    }
};

thread_local char g_err[512];
int fail(const char* what, cudaError_t e) {
    snprintf(g_err, sizeof g_err, "%s: %s", what, e == cudaSuccess ? "invalid arguments" : cudaGetErrorString(e));
    return -1;
}

bool labels_ok(const int32_t* labels, uint32_t n) {
    for (uint32_t i = 0; i < n; ++i)
        if (labels[i] < 0 || labels[i] >= kOut) return false;
    return true;
}

}  // namespace

extern "C" {

size_t zcb_prop_nparams(void) { return kNParams; }

size_t zcb_prop_error(char* buf, size_t cap) {
    const size_t n = strlen(g_err);
    if (buf && cap) {
        const size_t k = n < cap - 1 ? n : cap - 1;
        memcpy(buf, g_err, k);
        buf[k] = 0;
    }
    return n;
}

int32_t zcb_prop_forward(const float* params, size_t np, const float* x, uint32_t n, float* logits) {
    if (np != (size_t)kNParams || !params || !x || !logits || n == 0) return fail("prop_forward", cudaSuccess);
    cudaStream_t st;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return fail("prop_forward", cudaGetLastError());
    Net net;
    if (!net.alloc((int)n, st)) {
        cudaStreamDestroy(st);
        return fail("prop_forward", cudaErrorMemoryAllocation);
    }
    cudaMemcpyAsync(net.p, params, np * 4, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(net.x, x, (size_t)n * kC0 * kL * 4, cudaMemcpyHostToDevice, st);
    net.forward((int)n, st);
    cudaMemcpyAsync(logits, net.z, (size_t)n * kOut * 4, cudaMemcpyDeviceToHost, st);
    const cudaError_t e = cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
    net.release();
    return e == cudaSuccess ? 0 : fail("prop_forward", e);
}

int32_t zcb_prop_grad(const float* params, size_t np, const float* x, const int32_t* labels, uint32_t n, float* loss,
                      float* grad) {
    if (np != (size_t)kNParams || !params || !x || !labels || !loss || !grad || n == 0) return fail("prop_grad", cudaSuccess);
    if (!labels_ok(labels, n)) return fail("prop_grad: label outside 0..3239", cudaSuccess);
    cudaStream_t st;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return fail("prop_grad", cudaGetLastError());
    Net net;
    if (!net.alloc((int)n, st)) {
        cudaStreamDestroy(st);
        return fail("prop_grad", cudaErrorMemoryAllocation);
    }
    cudaMemcpyAsync(net.p, params, np * 4, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(net.x, x, (size_t)n * kC0 * kL * 4, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(net.lab, labels, (size_t)n * 4, cudaMemcpyHostToDevice, st);
    net.forward((int)n, st);
    net.backward((int)n, st);
    cudaMemcpyAsync(loss, net.loss, (size_t)n * 4, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(grad, net.g, np * 4, cudaMemcpyDeviceToHost, st);
    const cudaError_t e = cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
    net.release();
    return e == cudaSuccess ? 0 : fail("prop_grad", e);
}

int32_t zcb_prop_train(float* params, size_t np, const float* x, const int32_t* labels, uint32_t n, uint32_t batch,
                       uint32_t epochs, float lr, uint32_t seed, float* epoch_loss) {
    if (np != (size_t)kNParams || !params || !x || !labels || n == 0 || batch == 0 || batch > n)
        return fail("prop_train", cudaSuccess);
    if (!labels_ok(labels, n)) return fail("prop_train: label outside 0..3239", cudaSuccess);
    cudaStream_t st;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return fail("prop_train", cudaGetLastError());
    Net net;
    float* xall = nullptr;
    int* lall = nullptr;
    uint32_t* idx = nullptr;
    if (!net.alloc((int)batch, st) || cudaMalloc(&xall, (size_t)n * kC0 * kL * 4) != cudaSuccess ||
        cudaMalloc(&lall, (size_t)n * 4) != cudaSuccess || cudaMalloc(&idx, (size_t)n * 4) != cudaSuccess) {
        cudaFree(xall);
        cudaFree(lall);
        net.release();
        cudaStreamDestroy(st);
        return fail("prop_train", cudaErrorMemoryAllocation);
    }
    cudaMemcpyAsync(net.p, params, np * 4, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(xall, x, (size_t)n * kC0 * kL * 4, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(lall, labels, (size_t)n * 4, cudaMemcpyHostToDevice, st);
    // a seeded shuffle per epoch (host), minibatches gathered on the device
    std::vector<uint32_t> order(n);
    for (uint32_t i = 0; i < n; ++i) order[i] = i;
    uint64_t rs = 0x9E3779B97F4A7C15ull ^ seed;
    auto rnd = [&]() {
        rs ^= rs << 13, rs ^= rs >> 7, rs ^= rs << 17;
        return rs;
    };
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    int t = 0;
    std::vector<float> hl(batch);
    cudaError_t e = cudaSuccess;
    for (uint32_t ep = 0; ep < epochs && e == cudaSuccess; ++ep) {
        for (uint32_t i = n - 1; i > 0; --i) std::swap(order[i], order[rnd() % (i + 1)]);
        cudaMemcpyAsync(idx, order.data(), (size_t)n * 4, cudaMemcpyHostToDevice, st);
        double sum = 0;
        uint32_t cnt = 0;
        for (uint32_t b0 = 0; b0 + batch <= n; b0 += batch) {
            k_gather<<<blocks((int)batch * kC0 * kL), 256, 0, st>>>(xall, lall, idx + b0, (int)batch, net.x, net.lab);
            net.forward((int)batch, st);
            net.backward((int)batch, st);
            ++t;
            const float c1 = 1.f - powf(b1, (float)t), c2 = 1.f - powf(b2, (float)t);
            k_adam<<<blocks(kNParams), 256, 0, st>>>(net.p, net.g, net.m, net.v, kNParams, lr, b1, b2, eps, c1, c2);
            cudaMemcpyAsync(hl.data(), net.loss, batch * 4, cudaMemcpyDeviceToHost, st);
            e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) break;
            for (float v : hl) sum += v;
            cnt += batch;
        }
        if (epoch_loss) epoch_loss[ep] = cnt ? (float)(sum / cnt) : 0.f;
    }
    if (e == cudaSuccess) {
        cudaMemcpyAsync(params, net.p, np * 4, cudaMemcpyDeviceToHost, st);
        e = cudaStreamSynchronize(st);
    }
    cudaStreamDestroy(st);
    cudaFree(xall);
    cudaFree(lall);
    cudaFree(idx);
    net.release();
    return e == cudaSuccess ? 0 : fail("prop_train", e);
}

}  // extern "C"
