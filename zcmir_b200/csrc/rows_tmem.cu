// The map's last pass with the correlation sums in tensor memory: one block per output row.
//
// For row y the block forms every correlation pair's Hermitian full row from its half spectrum
// (Z = Q1 + i·Q2 for x ≤ N/2, conj(Q1) + i·conj(Q2) mirrored above), inverse-FFTs it (N points,
// N/8 threads per line, 512 / (N/8) lines per round), and keeps each correlation's N sums for
// the score: slots 0..31 in tensor memory (TMEM: 128 lanes × 32·N/128 columns, cell m in lane
// m mod 128, column (m / 128)·32 + slot), slots 32.. in shared memory. With no correlation row
// in shared memory beyond 13, a block holds a whole 2048-point row, so every half-spectrum row is
// read from memory once. The next round's half rows are loaded into registers while the current
// round transforms. Then every cell's 45 sums are scored (float64) and the block's argmax is
// merged into the map's.
//
// tcgen05 rules kept here: one warp allocates and frees the columns (a power of two ≥ 32) and
// gives up its allocation permit at once; warp w reaches lanes 32·(w mod 4) .. +31 only; every
// tcgen05.ld / st is executed by whole warps with uniform control flow; tcgen05.wait::st before
// the barrier that precedes the loads, with the thread-sync fences around it.
#include "combine.cuh"
#include "common.cuh"
#include "kernels.hpp"

namespace zc {
namespace {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tmem_st1(uint32_t taddr, float v) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x1.b32 [%0], {%1};" ::"r"(taddr), "r"(__float_as_uint(v)) : "memory");
}
// two consecutive columns (taddr, taddr + 1) of this thread's lane
__device__ __forceinline__ void tmem_st2(uint32_t taddr, float a, float b) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x2.b32 [%0], {%1, %2};" ::"r"(taddr), "r"(__float_as_uint(a)),
                 "r"(__float_as_uint(b))
                 : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
          "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
}

constexpr int kTmemSlots = 32;

// Lines of N ≥ 1024 run with 128 threads each and their ends in registers (run_io): the first
// butterflies read the Hermitian row straight from the half spectra, and the last hand each
// thread the outputs m ≡ t (mod 128) of its line thread t — exactly the TMEM lane that thread's
// warp reaches — so the sums go from registers to TMEM with no pass through shared memory.
template <int N>
constexpr bool rows_io() { return N >= 1024; }
template <int N>
constexpr int rows_tl() { return rows_io<N>() ? 128 : N / 8; }

template <int N, int NF, bool EXACT, bool CALIB>
__global__ void __launch_bounds__(512, 1) k_rows_tmem(const float2* __restrict__ Q, size_t pstride, int WP, int n_corr,
                                                      const float2* __restrict__ tw, CombineParams cp,
                                                      const double* __restrict__ n00p, float* __restrict__ map,
                                                      unsigned long long* best, float* zero_out, int y0) {
    constexpr int TL = rows_tl<N>();           // threads per line
    constexpr int LINES = 512 / TL;            // lines per round
    constexpr int J = N / 128;                 // cells per TMEM lane
    constexpr int TCOLS = J * kTmemSlots;      // columns allocated (power of two ≥ 32)
    constexpr int PER = (N / 2) / TL;          // half-row points per thread (4)
    static_assert(TCOLS >= 32 && TCOLS <= 512 && (TCOLS & (TCOLS - 1)) == 0, "TMEM columns");
    extern __shared__ float2 smem[];
    __shared__ uint32_t tbase_sh;
    constexpr int PL = (N + (N >> 4) + 1);
    float2* lines = smem;
    float* cs = reinterpret_cast<float*>(smem + LINES * PL);  // slots ≥ 32: [slot − 32][N]
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (w == 0) {
        tmem_alloc(&tbase_sh, TCOLS);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tb = tbase_sh;
    const uint32_t tq = tb + ((uint32_t)(32 * (w & 3)) << 16);  // this warp's lane quadrant
    const int grp = w >> 2;                                      // 0..3: which j's this warp takes

    const int y = y0 + blockIdx.x;  // rows y0 .. y0 + gridDim.x − 1
    const int line = threadIdx.x / TL, t = threadIdx.x - line * TL;
    float2* buf = lines + line * PL;
    const int npairs = (n_corr + 1) / 2;
    const Pow2Line<N, TL> fft{tw};

    if constexpr (rows_io<N>()) {
        static_assert(N / Mix<N>::radix(Mix<N>::kStages - 1) % 128 == 0, "last-stage outputs must fall in lane t");
        const int n_tm = n_corr < kTmemSlots ? n_corr : kTmemSlots;
        for (int p0 = 0; p0 < npairs; p0 += LINES) {
            const int pr = p0 + line;
            const bool act = pr < npairs;
            const int k1 = 2 * pr, k2 = 2 * pr + 1;
            const bool h2 = k2 < n_corr;
            const float2* q1 = Q + (size_t)(act ? k1 : 0) * pstride + (size_t)y * WP;
            const float2* q2 = Q + (size_t)(act && h2 ? k2 : 0) * pstride + (size_t)y * WP;
            // Z = Q1 + i·Q2 on the half row, conj(Q1) + i·conj(Q2) mirrored above it
            auto in = [&](int x) {
                const int ix = x <= N / 2 ? x : N - x;
                const float2 a = __ldg(&q1[ix]);
                const float2 b = h2 ? __ldg(&q2[ix]) : make_float2(0.f, 0.f);
                return x <= N / 2 ? make_float2(a.x - b.y, a.y + b.x) : make_float2(a.x + b.y, b.x - a.y);
            };
            if (2 * (p0 + LINES) <= n_tm) {
                // every line of the round has both its slots in TMEM: one two-column store per
                // output (cell m lies in TMEM lane m mod 128 = t, this warp's quadrant)
                fft.template run_io<true>(buf, t, true, in, [&](int m, float2 z) {
                    tmem_st2(tq + (uint32_t)(m >> 7) * kTmemSlots + (uint32_t)k1, z.x, z.y);
                });
            } else {
                fft.template run_io<true>(buf, t, act, in, [&](int m, float2 z) {
                    // the warp's lines all run, so each store is executed by the whole warp
                    const uint32_t col = (uint32_t)(m >> 7) * kTmemSlots;
                    if (k1 < kTmemSlots) tmem_st1(tq + col + (uint32_t)k1, z.x);
                    else cs[(size_t)(k1 - kTmemSlots) * N + m] = z.x;
                    if (h2) {
                        if (k2 < kTmemSlots) tmem_st1(tq + col + (uint32_t)k2, z.y);
                        else cs[(size_t)(k2 - kTmemSlots) * N + m] = z.y;
                    }
                });
            }
            __syncthreads();  // the line buffers are refilled next round
        }
    } else {

    float2 pa[PER], pb[PER], na = make_float2(0.f, 0.f), nb = make_float2(0.f, 0.f);
    auto fetch = [&](int pr) {
        const int k1 = 2 * pr, k2 = 2 * pr + 1;
        const float2* q1 = Q + (size_t)k1 * pstride + (size_t)y * WP;
        const float2* q2 = Q + (size_t)(k2 < n_corr ? k2 : k1) * pstride + (size_t)y * WP;
        const bool h2 = k2 < n_corr;
#pragma unroll
        for (int i = 0; i < PER; ++i) {
            pa[i] = __ldg(&q1[t + TL * i]);
            pb[i] = h2 ? __ldg(&q2[t + TL * i]) : make_float2(0.f, 0.f);
        }
        if (t == 0) {
            na = __ldg(&q1[N / 2]);
            nb = h2 ? __ldg(&q2[N / 2]) : make_float2(0.f, 0.f);
        }
    };
    if (line < npairs) fetch(line);

    for (int p0 = 0; p0 < npairs; p0 += LINES) {
        const int pr = p0 + line;
        const bool act = pr < npairs;
        if (act) {
#pragma unroll
            for (int i = 0; i < PER; ++i) {
                const int ix = t + TL * i;
                const float2 a = pa[i], b = pb[i];
                buf[pad_idx(ix)] = make_float2(a.x - b.y, a.y + b.x);
                if (ix > 0) buf[pad_idx(N - ix)] = make_float2(a.x + b.y, b.x - a.y);
            }
            if (t == 0) buf[pad_idx(N / 2)] = make_float2(na.x - nb.y, na.y + nb.x);
            if (pr + LINES < npairs) fetch(pr + LINES);  // next round's rows, in flight during the FFT
        }
        __syncthreads();
        fft.template run<true>(buf, t, act);
        // scatter the round's sums: TMEM slots by whole warps, the rest to shared memory
#pragma unroll 1
        for (int l = 0; l < LINES; ++l) {
            const int prl = p0 + l;
            if (prl >= npairs) break;
            const float2* bl = lines + l * PL;
#pragma unroll
            for (int comp = 0; comp < 2; ++comp) {
                const int slot = 2 * prl + comp;
                if (slot >= n_corr) break;
                if (slot < kTmemSlots) {
#pragma unroll
                    for (int j = grp; j < J; j += 4) {
                        const int m = 32 * (w & 3) + lane + 128 * j;
                        const float2 z = bl[pad_idx(m)];
                        tmem_st1(tq + (uint32_t)(j * kTmemSlots + slot), comp ? z.y : z.x);
                    }
                } else {
                    float* dst = cs + (size_t)(slot - kTmemSlots) * N;
                    for (int m = threadIdx.x; m < N; m += 512) {
                        const float2 z = bl[pad_idx(m)];
                        dst[m] = comp ? z.y : z.x;
                    }
                }
            }
        }
        __syncthreads();
    }
    }
    tmem_wait_st();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();

    const double n00 = *n00p;
    float bv = -3.4e38f;
    uint32_t bi = 0xffffffffu;
#pragma unroll 1
    for (int j = grp; j < J; j += 4) {
        const int m = 32 * (w & 3) + lane + 128 * j;
        uint32_t r[32];
        tmem_ld32(tq + (uint32_t)(j * kTmemSlots), r);
        tmem_wait_ld();
        const float sc = combine_t<NF, EXACT, CALIB>(
            [&](int k) { return k < kTmemSlots ? __uint_as_float(r[k]) : cs[(size_t)(k - kTmemSlots) * N + m]; }, cp, n00);
        const uint32_t idx = (uint32_t)y * (uint32_t)N + (uint32_t)m;
        map[idx] = sc;
        if (sc > bv || (sc == bv && idx < bi)) {
            bv = sc;
            bi = idx;
        }
        if (idx == 0) *zero_out = sc;
    }
    unsigned long long key = (bi == 0xffffffffu) ? 0ull : argmax_key(bv, bi);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long other = __shfl_xor_sync(0xffffffffu, key, o);
        key = other > key ? other : key;
    }
    if (lane == 0 && key) atomicMax(best, key);

    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (w == 0) tmem_dealloc(tb, TCOLS);
}

template <int N, int NF, bool EXACT, bool CALIB>
cudaError_t launch_tmem(const float2* Q, const MapGeom& g, int n_corr, const float2* tw, const CombineParams& cp,
                        const double* n00, float* map, unsigned long long* best, float* zero, cudaStream_t st, int y0,
                        int rows) {
    constexpr int TL = rows_tl<N>(), LINES = 512 / TL;
    const int extra = n_corr > kTmemSlots ? n_corr - kTmemSlots : 0;
    const size_t sm = (size_t)LINES * padded_len(N) * sizeof(float2) + (size_t)extra * N * sizeof(float);
    auto k = k_rows_tmem<N, NF, EXACT, CALIB>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k<<<rows, 512, sm, st>>>(Q, (size_t)g.ny * g.WP, g.WP, n_corr, tw, cp, n00, map, best, zero, y0);
    return cudaGetLastError();
}

template <int N>
cudaError_t dispatch_tmem(const float2* Q, const MapGeom& g, int n_corr, const float2* tw, const CombineParams& cp,
                          const double* n00, float* map, unsigned long long* best, float* zero, cudaStream_t st, int y0,
                          int rows) {
    if (cp.nf == 4) {
        if (!cp.exact) return launch_tmem<N, 4, false, false>(Q, g, n_corr, tw, cp, n00, map, best, zero, st, y0, rows);
        if (cp.calib) return launch_tmem<N, 4, true, true>(Q, g, n_corr, tw, cp, n00, map, best, zero, st, y0, rows);
        return launch_tmem<N, 4, true, false>(Q, g, n_corr, tw, cp, n00, map, best, zero, st, y0, rows);
    }
    if (!cp.exact) return launch_tmem<N, 3, false, false>(Q, g, n_corr, tw, cp, n00, map, best, zero, st, y0, rows);
    if (cp.calib) return launch_tmem<N, 3, true, true>(Q, g, n_corr, tw, cp, n00, map, best, zero, st, y0, rows);
    return launch_tmem<N, 3, true, false>(Q, g, n_corr, tw, cp, n00, map, best, zero, st, y0, rows);
}

}  // namespace

bool rows_tmem_supported(int nx, int n_corr) { return (nx == 512 || nx == 1024 || nx == 2048) && n_corr <= 45; }

cudaError_t inverse_rows_score_tmem(const float2* Q, const MapGeom& g, const CorrPlanDev& plan, const float2* tw_nx,
                                    const CombineParams& cp, const double* n00, float* map, unsigned long long* best,
                                    float* zero, cudaStream_t st, int y0, int rows) {
    if (rows < 0) rows = g.ny - y0;
    if (y0 < 0 || rows <= 0 || y0 + rows > g.ny) return cudaErrorInvalidValue;
    switch (g.nx) {
        case 512: return dispatch_tmem<512>(Q, g, plan.n_corr, tw_nx, cp, n00, map, best, zero, st, y0, rows);
        case 1024: return dispatch_tmem<1024>(Q, g, plan.n_corr, tw_nx, cp, n00, map, best, zero, st, y0, rows);
        case 2048: return dispatch_tmem<2048>(Q, g, plan.n_corr, tw_nx, cp, n00, map, best, zero, st, y0, rows);
        default: return cudaErrorNotSupported;
    }
}

}  // namespace zc
