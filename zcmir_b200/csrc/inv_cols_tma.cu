// The map's inverse-column pass for 1024- and 2048-point columns, fed by TMA.
//
// Per item (column tile of TX columns, correlation slot k) the pass forms the products
// A_ca[k] · conj(B_cb[k]) over the whole tile and inverse-FFTs its columns into Q[k]. The
// correlations are walked in runs that share one operand plane (make_units: the 45 of the full
// plan in 10 runs of 4–5), and one 512-thread block per SM walks the (column tile, run) units,
// run fastest (so the blocks running together share the tile's planes in L2). Both operand tiles
// (N rows × TX complex columns each) arrive in shared memory by TMA: one thread issues N/256
// box loads per side on an mbarrier. Within a run only the streamed side's tile is copied again,
// so a column tile costs 55 tile copies out of L2 instead of 90. The next item's copies are
// issued as soon as the current item's first butterflies have read the staging buffers, so they
// land while the rest of the transform runs. No thread spends registers
// or load instructions on the operands, and the twiddles of every stage after the first, which
// depend only on a thread's place in its line, are read once per block into registers rather
// than once per item.
//
// Line schedule: N = 2048 → radices 16 · 16 · 8 with 128 threads per line (TX = 4 columns);
// N = 1024 → 16 · 8 · 8 with 64 threads per line (TX = 8). The first stage's butterfly of
// thread t takes rows t + r·N/16; the middle stages pass through a padded line buffer; the last
// stage stores straight to Q.
#include <mutex>

#include "fft.cuh"
#include "kernels.hpp"
#include "tma.cuh"

namespace zc {

// ── host: tensor maps ───────────────────────────────────────────────────────────────────────

namespace {

using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encode_fn() {
    static std::once_flag once;
    static EncodeTiled fn = nullptr;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiled>(p);
    });
    return fn;
}

}  // namespace

bool encode_cplx_map(CUtensorMap* out, const void* base, int cols, int rows, int planes, size_t pitch, size_t pstride,
                     int box_cols, int box_rows) {
    const EncodeTiled enc = encode_fn();
    if (!enc || box_cols % 2 || box_cols <= 0 || box_rows <= 0 || box_rows > 256 || 2 * box_cols > 256) return false;
    const cuuint64_t dims[3] = {2ull * (cuuint64_t)cols, (cuuint64_t)rows, (cuuint64_t)planes};
    const cuuint64_t strides[2] = {(cuuint64_t)pitch * 8, (cuuint64_t)pstride * 8};  // bytes, dimensions 1 and 2
    const cuuint32_t box[3] = {(cuuint32_t)(2 * box_cols), (cuuint32_t)box_rows, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    return enc(out, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<void*>(base), dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

namespace {

// ── line stages with the twiddles in registers ──────────────────────────────────────────────

// points transformed before stage s of a line of n
__host__ __device__ constexpr int ns_before(int n, int s) {
    int ns = 1;
    for (int i = 0; i < s; ++i) ns *= mix_radix(n, i);
    return ns;
}
// butterflies per thread of stage s (TL threads per line)
__host__ __device__ constexpr int bm_of(int n, int tl, int s) { return (n / mix_radix(n, s) + tl - 1) / tl; }
// register twiddles of stages ≥ 1 before stage s (stage s's block starts there)
__host__ __device__ constexpr int rt_off(int n, int tl, int s) {
    int off = 0;
    for (int i = 1; i < s; ++i) off += bm_of(n, tl, i) * (mix_radix(n, i) - 1);
    return off;
}
__host__ __device__ constexpr int rt_total(int n, int tl) { return rt_off(n, tl, mix_stages(n)); }

// thread t's twiddles of every stage after the first (conjugated for the inverse transform)
template <int N, int TL, bool INV, int S = 1>
__device__ __forceinline__ void rt_load(float2 (&w)[rt_total(N, TL)], const float2* __restrict__ tw, int t) {
    if constexpr (S < mix_stages(N)) {
        constexpr int R = mix_radix(N, S), NS = ns_before(N, S), M = N / R, BM = bm_of(N, TL, S);
        constexpr int OFF = rt_off(N, TL, S), TOFF = N + stage_tw_off(N, S);
#pragma unroll
        for (int b = 0; b < BM; ++b) {
            const int j = t + b * TL;
            const int k = (j < M ? j : 0) % NS;
#pragma unroll
            for (int r = 1; r < R; ++r) {
                float2 v = __ldg(&tw[TOFF + (r - 1) * NS + k]);
                if (INV) v.y = -v.y;
                w[OFF + b * (R - 1) + (r - 1)] = v;
            }
        }
        rt_load<N, TL, INV, S + 1>(w, tw, t);
    }
}

// the stages after the first and before the last, through the line buffer
template <int N, int TL, bool INV, int S>
__device__ __forceinline__ void rt_mid(float2* __restrict__ buf, const float2 (&w)[rt_total(N, TL)], int t) {
    if constexpr (S < mix_stages(N) - 1) {
        constexpr int R = mix_radix(N, S), NS = ns_before(N, S), M = N / R, BM = bm_of(N, TL, S);
        constexpr int OFF = rt_off(N, TL, S);
        float2 v[BM][R];
#pragma unroll
        for (int b = 0; b < BM; ++b) {
            const int j = t + b * TL;
            if (M % TL == 0 || j < M) {
                if constexpr (M % 16 == 0) {
                    const int p = pad_idx(j);
#pragma unroll
                    for (int r = 0; r < R; ++r) v[b][r] = buf[pad_at<M>(p, r)];
                } else {
#pragma unroll
                    for (int r = 0; r < R; ++r) v[b][r] = buf[pad_idx(j + r * M)];
                }
            }
        }
        __syncthreads();
#pragma unroll
        for (int b = 0; b < BM; ++b) {
            const int j = t + b * TL;
            if (M % TL == 0 || j < M) {
                const int k = j % NS;
#pragma unroll
                for (int r = 1; r < R; ++r) v[b][r] = cmul(v[b][r], w[OFF + b * (R - 1) + (r - 1)]);
                dft<R, INV>(v[b]);
                const int base = (j - k) * R + k;
                if constexpr (NS % 16 == 0 || 16 % (R * NS) == 0) {
                    const int p = pad_idx(base);
#pragma unroll
                    for (int r = 0; r < R; ++r) buf[pad_at<NS, (NS % 16 != 0)>(p, r)] = v[b][r];
                } else {
#pragma unroll
                    for (int r = 0; r < R; ++r) buf[pad_idx(base + r * NS)] = v[b][r];
                }
            }
        }
        __syncthreads();
        rt_mid<N, TL, INV, S + 1>(buf, w, t);
    }
}

// the last stage: outputs to out(y, v)
template <int N, int TL, bool INV, class Out>
__device__ __forceinline__ void rt_last(const float2* __restrict__ buf, const float2 (&w)[rt_total(N, TL)], int t,
                                        Out&& out) {
    constexpr int S = mix_stages(N) - 1;
    constexpr int R = mix_radix(N, S), NS = ns_before(N, S), M = N / R, BM = bm_of(N, TL, S);
    constexpr int OFF = rt_off(N, TL, S);
    static_assert(NS == M, "the last stage's sub-transforms span the line");
#pragma unroll
    for (int b = 0; b < BM; ++b) {
        const int j = t + b * TL;
        if (M % TL == 0 || j < M) {
            float2 v[R];
            if constexpr (M % 16 == 0) {
                const int p = pad_idx(j);
#pragma unroll
                for (int r = 0; r < R; ++r) v[r] = buf[pad_at<M>(p, r)];
            } else {
#pragma unroll
                for (int r = 0; r < R; ++r) v[r] = buf[pad_idx(j + r * M)];
            }
#pragma unroll
            for (int r = 1; r < R; ++r) v[r] = cmul(v[r], w[OFF + b * (R - 1) + (r - 1)]);
            dft<R, INV>(v);
#pragma unroll
            for (int r = 0; r < R; ++r) out(j + r * NS, v[r]);
        }
    }
}

constexpr int kBoxRows = 256;

template <int N>
struct InvColsShape {
    static constexpr int TL = N / 16;          // threads per line
    static constexpr int TX = 512 / TL;        // columns per item
    static constexpr size_t tile_bytes = (size_t)N * TX * sizeof(float2);
    static constexpr size_t smem = 2 * tile_bytes + (size_t)TX * line_pitch(N) * sizeof(float2) + 16;
};

// Runs of correlations that share one operand plane: unit u keeps side side[u]'s plane res[u]
// resident in shared memory while its n[u] correlations k[u][·] stream the other side's plane.
constexpr int kUnitMax = 5;
constexpr int kMaxUnits = 48;
struct InvUnits {
    int count;
    signed char side[kMaxUnits];  // 0: side A's plane stays, 1: side B's
    signed char n[kMaxUnits];
    signed char k[kMaxUnits][kUnitMax];
};

// Cover the plan's correlations with runs sharing an operand: repeatedly take the plane (of
// either side) shared by the most correlations left, and cut its correlations into runs of at
// most kUnitMax of nearly equal length. The 45-correlation plan gives 10 runs (plane 1 of A:
// 15 in 3 runs, plane 1 of B: 14 in 3, then A's f_i planes: 4 runs of 4), so a column tile
// loads 55 operand tiles instead of 90.
bool make_units(const CorrPlanDev& plan, InvUnits& u) {
    u = InvUnits{};
    bool left[45] = {};
    int n_left = plan.n_corr;
    for (int c = 0; c < plan.n_corr; ++c) left[c] = true;
    while (n_left > 0) {
        int best_side = 0, best_plane = -1, best_n = 0;
        for (int sd = 0; sd < 2; ++sd)
            for (int pl = 0; pl < plan.n_real; ++pl) {
                int cnt = 0;
                for (int c = 0; c < plan.n_corr; ++c)
                    if (left[c] && (sd == 0 ? plan.ca[c] : plan.cb[c]) == pl) ++cnt;
                if (cnt > best_n) best_side = sd, best_plane = pl, best_n = cnt;
            }
        if (best_n == 0) return false;
        const int runs = (best_n + kUnitMax - 1) / kUnitMax;
        int c = 0;
        for (int r = 0; r < runs; ++r) {
            if (u.count >= kMaxUnits) return false;
            const int len = best_n / runs + (r < best_n % runs ? 1 : 0);
            const int ui = u.count++;
            u.side[ui] = (signed char)best_side;
            u.n[ui] = (signed char)len;
            for (int i = 0; i < len; ++i) {
                while (!(left[c] && (best_side == 0 ? plan.ca[c] : plan.cb[c]) == best_plane)) ++c;
                u.k[ui][i] = (signed char)c;
                left[c] = false;
                ++c;
            }
            n_left -= len;
        }
    }
    return true;
}

template <int N>
__global__ void __launch_bounds__(512, 1) k_inv_cols_tma(const __grid_constant__ CUtensorMap map_a,
                                                         const __grid_constant__ CUtensorMap map_b, CorrPlanDev plan,
                                                         const __grid_constant__ InvUnits units,
                                                         const float2* __restrict__ tw, int ncols,
                                                         float2* __restrict__ Q, size_t pstride, int WP, int nwork,
                                                         unsigned* __restrict__ fault) {
    using SH = InvColsShape<N>;
    constexpr int TL = SH::TL, TX = SH::TX, R0 = mix_radix(N, 0), M0 = N / R0;
    static_assert(R0 == 16 && M0 == TL, "one 16-point first butterfly per line thread");
    static_assert(N % kBoxRows == 0, "whole boxes of rows");
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    float2* sa = reinterpret_cast<float2*>(smem_raw);  // [N][TX]: side A's tile
    float2* sb = sa + (size_t)N * TX;                    // [N][TX]: side B's tile
    float2* lines = sb + (size_t)N * TX;                 // TX line buffers
    uint64_t* bar = reinterpret_cast<uint64_t*>(lines + (size_t)TX * line_pitch(N));
    const int tid = threadIdx.x, c = tid % TX, t = tid / TX;
    float2* buf = lines + c * line_pitch(N);
    const int nu = units.count;
    if (smem_addr(sa) & 127) {  // a tiled copy's destination must be 128-byte aligned
        if (tid == 0) atomicOr(fault, 2u);
        return;
    }
    // copies of column tile col0: side A's plane pa into sa and side B's pb into sb; a negative
    // plane leaves that side's tile as it is
    auto issue = [&](int col0, int pa, int pb) {
        mbar_expect_tx(bar, (uint32_t)(((pa >= 0) + (pb >= 0)) * SH::tile_bytes));
#pragma unroll 1
        for (int i = 0; i < N / kBoxRows; ++i) {
            if (pa >= 0) tma_load_3d(sa + (size_t)i * kBoxRows * TX, &map_a, 2 * col0, i * kBoxRows, pa, bar);
            if (pb >= 0) tma_load_3d(sb + (size_t)i * kBoxRows * TX, &map_b, 2 * col0, i * kBoxRows, pb, bar);
        }
    };
    float2 w[rt_total(N, TL)];
    rt_load<N, TL, true>(w, tw, t);
    if (tid == 0) {
        mbar_init(bar, 1);
        mbar_init_fence();
    }
    __syncthreads();
    int wk = blockIdx.x;
    if (tid == 0 && wk < nwork) {
        const int k0 = units.k[wk % nu][0];
        issue((wk / nu) * TX, plan.ca[k0], plan.cb[k0]);
    }
    uint32_t phase = 0;
    for (; wk < nwork; wk += gridDim.x) {
        const int un = wk % nu, col0 = (wk / nu) * TX, len = units.n[un];
        const bool keep_a = units.side[un] == 0;
        const int col = col0 + c;
        const bool okc = col < ncols;
#pragma unroll 1
        for (int i = 0; i < len; ++i) {
            const bool ok = mbar_wait(bar, phase);
            if (__syncthreads_or(!ok)) {
                // a copy did not land: report it, give the copies in flight one more bounded wait, stop
                if (tid == 0) {
                    atomicOr(fault, 1u);
                    mbar_wait(bar, phase);
                }
                return;
            }
            phase ^= 1u;
            const int k = units.k[un][i];
            float2* O = Q + (size_t)k * pstride + (okc ? col : 0);
            float2 v[R0];
#pragma unroll
            for (int r = 0; r < R0; ++r) {
                const int y = t + r * M0;
                v[r] = cmulc(sa[y * TX + c], sb[y * TX + c]);
            }
            dft<R0, true>(v);
#pragma unroll
            for (int r = 0; r < R0; ++r) buf[first_slot<R0>(t, r)] = v[r];
            __syncthreads();  // both tiles are read: the next copies may land in them
            if (tid == 0) {
                if (i + 1 < len) {
                    // the run's next correlation: only the streamed side's plane changes
                    const int kn = units.k[un][i + 1];
                    fence_proxy_async();
                    issue(col0, keep_a ? -1 : plan.ca[kn], keep_a ? plan.cb[kn] : -1);
                } else if (wk + (int)gridDim.x < nwork) {
                    const int wn = wk + gridDim.x, kn = units.k[wn % nu][0];
                    fence_proxy_async();
                    issue((wn / nu) * TX, plan.ca[kn], plan.cb[kn]);
                }
            }
            rt_mid<N, TL, true, 1>(buf, w, t);
            rt_last<N, TL, true>(buf, w, t, [&](int y, float2 val) {
                if (okc) O[(size_t)y * WP] = val;
            });
            __syncthreads();  // the line buffers are refilled by the next item
        }
    }
}

// where a launch with no fault word of its caller's reports (nobody reads it back)
__device__ unsigned g_inv_cols_fault;

constexpr int kMaxDev = 64;
std::mutex g_fault_mu;
unsigned* g_fault_ptr[kMaxDev];

cudaError_t fault_word(unsigned** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDev) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_fault_mu);
    if (!g_fault_ptr[dev]) {
        unsigned* p = nullptr;
        if ((e = cudaGetSymbolAddress((void**)&p, g_inv_cols_fault)) != cudaSuccess) return e;
        g_fault_ptr[dev] = p;
    }
    *out = g_fault_ptr[dev];
    return cudaSuccess;
}

template <int N>
cudaError_t launch_tma(const float2* ha, const float2* hb, const MapGeom& g, const CorrPlanDev& plan,
                       const float2* tw, float2* Q, cudaStream_t st, unsigned* fault) {
    using SH = InvColsShape<N>;
    const int ncols = g.nx / 2 + 1;
    const size_t pstride = (size_t)g.ny * g.WP;
    CUtensorMap ma, mb;
    if (!encode_cplx_map(&ma, ha, ncols, g.ny, plan.n_real, g.WP, pstride, SH::TX, kBoxRows) ||
        !encode_cplx_map(&mb, hb, ncols, g.ny, plan.n_real, g.WP, pstride, SH::TX, kBoxRows))
        return cudaErrorInvalidValue;
    cudaError_t e = cudaSuccess;
    if (!fault && (e = fault_word(&fault)) != cudaSuccess) return e;
    InvUnits units;
    if (!make_units(plan, units)) return cudaErrorInvalidValue;
    const int nitems = units.count * ((ncols + SH::TX - 1) / SH::TX);
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    auto k = k_inv_cols_tma<N>;
    if ((e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SH::smem)) != cudaSuccess)
        return e;
    k<<<std::min(nitems, sms), 512, SH::smem, st>>>(ma, mb, plan, units, tw, ncols, Q, pstride, g.WP, nitems, fault);
    return cudaGetLastError();
}

}  // namespace

bool inverse_columns_tma_supported(const MapGeom& g, int batch) {
    return batch == 1 && g.nx == g.ny && (g.ny == 1024 || g.ny == 2048) && g.WP % 2 == 0 && encode_fn() != nullptr;
}

cudaError_t inverse_columns_tma(const float2* ha, const float2* hb, const MapGeom& g, const CorrPlanDev& plan,
                                const float2* tw, float2* Q, cudaStream_t st, unsigned* fault) {
    if (g.ny == 2048) return launch_tma<2048>(ha, hb, g, plan, tw, Q, st, fault);
    if (g.ny == 1024) return launch_tma<1024>(ha, hb, g, plan, tw, Q, st, fault);
    return cudaErrorInvalidValue;
}

}  // namespace zc
