// The first stage of the column FFTs on the tensor cores, with split-BF16 products: a precision
// study of the small-radix DFT stage, not a path the maps take by default.
//
// Stage 0 of a Stockham line of n points with radix 16 is a matrix product: with M = n/16,
// output j·16 + r = Σ_q x[q·M + j]·ω^{qr}, ω = e^{−2πi/16}. Over real numbers, a row holding
// (Re x_0..x_15, Im x_0..x_15) (K = 32) times the 32 × 32 matrix [[C, −S], [S, C]] (C, S: the
// cosines and sines of 2π·qr/16, rows q, columns r) gives (Re y_0..y_15, Im y_0..y_15) (N = 32). A block takes tiles
// of 128 rows — 4 butterflies j × 32 adjacent columns, so the loads and stores of a warp are
// one contiguous 256-byte run per point — and runs the product as tcgen05.mma of kind::f16
// (BF16 × BF16, FP32 accumulators in tensor memory, M = 128, N = 32, K = 16 per instruction).
//
// BF16 keeps 8 significant bits, so each FP32 input and each coefficient is split into `P`
// pieces a = a0 (+ a1 (+ a2)), a_i = bf16(a − a_0 − … − a_{i−1}), and the products with
// i + k < P are summed (1 for P = 1: plain BF16; 3 for P = 2, about 16 significant bits; 6 for
// P = 3, about 24, close to FP32), the small ones first. The coefficients' pieces are split from
// float64 values.
//
// Operands sit in shared memory in the no-swizzle K-major layout the MMA's descriptors describe:
// 8-row × 16-byte core matrices, cores adjacent along K 128 bytes apart (the descriptor's leading
// byte offset), cores adjacent along the rows 512 bytes apart (its stride byte offset). One
// thread issues the MMAs and commits them to an mbarrier; every wait on it is bounded (a wait
// that gives up sets the fault word, waits once more, frees the tensor memory and returns).
#include <cuda_bf16.h>

#include "fft.cuh"
#include "kernels.hpp"
#include "tma.cuh"

namespace zc {
namespace {

constexpr int kRadix = 16;
constexpr int kRows = 128;                  // MMA M: 4 butterflies × 32 columns
constexpr int kK = 32;                      // real K: Re, then Im of the 16 inputs
constexpr int kN = 32;                      // real N: Re, then Im of the 16 outputs
constexpr int kPieceA = kRows * kK * 2;     // bytes of one BF16 piece of a tile (8 KB)
constexpr int kPieceB = kN * kK * 2;        // bytes of one piece of the coefficients (2 KB)
constexpr uint32_t kTmemCols = 32;          // FP32 accumulator columns (N)

// byte offset of element (row, k) of a K-major operand in the no-swizzle canonical layout
__host__ __device__ constexpr int kmaj_off(int row, int k) {
    return ((row >> 3) * 4 + (k >> 3)) * 128 + (row & 7) * 16 + (k & 7) * 2;
}

// shared-memory matrix descriptor: start address, leading byte offset 128 (K), stride byte
// offset 512 (rows), version 1 (bits 46–47), base offset 0, no swizzle
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
    return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(512 >> 4) << 32) |
           ((uint64_t)1 << 46);
}

// instruction descriptor of kind::f16: D FP32 (bits 4–5 = 1), A and B BF16 (bits 7–9, 10–12 = 1),
// both K-major (bits 15, 16 = 0), N >> 3 at bits 17–22, M >> 4 at bits 24–28
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kN >> 3) << 17) |
                            ((uint32_t)(kRows >> 4) << 24);

__device__ __forceinline__ void tc_alloc(uint32_t* dst, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(dst)), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tc_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// D (+)= A·Bᵀ for one K = 16 slice; acc = 0 overwrites D
__device__ __forceinline__ void mma_bf16(uint32_t d, uint64_t a, uint64_t b, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d),
        "l"(a), "l"(b), "r"(kIdesc), "r"(acc)
        : "memory");
}
// the MMAs issued so far by this thread arrive on bar when they complete
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
                 : "memory");
}

// 32 FP32 columns of this warp's 32 lanes: lane i of warp w gets row 32w + i
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
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
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// the P BF16 pieces of a (each the rounding of what the earlier pieces left)
template <int P>
__device__ __forceinline__ void split_f32(float a, __nv_bfloat16 (&h)[P]) {
    float rest = a;
#pragma unroll
    for (int i = 0; i < P; ++i) {
        h[i] = __float2bfloat16_rn(rest);
        rest -= __bfloat162float(h[i]);
    }
}

// Block: columns 32·bx .. +31 of plane bz, butterfly tiles by·tpb .. +tpb−1 (4 butterflies each;
// warp w takes butterfly 4·tile + w, lane i column 32·bx + i). Rows ≥ rows_in read as zero.
// Output point j·16 + r of each column goes to `out` (the stage's Stockham order).
template <int P>
__global__ void __launch_bounds__(128) k_dft16_tc(const float2* __restrict__ in, float2* __restrict__ out,
                                                  size_t pstride, int WP, int ncols, int n, int rows_in, int tpb,
                                                  unsigned* __restrict__ fault) {
    __shared__ __align__(128) unsigned char sA[P * kPieceA];
    __shared__ __align__(128) unsigned char sB[P * kPieceB];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t s_taddr;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int M = n / kRadix;
    const int c = blockIdx.x * 32 + lane;
    const bool okc = c < ncols;
    const size_t base = (size_t)blockIdx.z * pstride + (okc ? c : 0);
    // the coefficients' pieces, B[n][k] = the real matrix's entry (k, n), split from float64
    for (int e = tid; e < kN * kK; e += blockDim.x) {
        const int nn = e / kK, k = e % kK;
        const int r = nn & 15, q = k & 15;
        double sv, cv;
        sincospi((double)((q * r) & 15) / 8.0, &sv, &cv);
        const bool re_out = nn < 16, re_in = k < 16;
        double rest = re_out ? (re_in ? cv : sv) : (re_in ? -sv : cv);
#pragma unroll
        for (int i = 0; i < P; ++i) {
            const __nv_bfloat16 h = __double2bfloat16(rest);
            *reinterpret_cast<__nv_bfloat16*>(sB + i * kPieceB + kmaj_off(nn, k)) = h;
            rest -= (double)__bfloat162float(h);
        }
    }
    if (warp == 0) tc_alloc(&s_taddr, kTmemCols);
    if (tid == 0) {
        mbar_init(&bar, 1);
        mbar_init_fence();
    }
    tc_before();
    __syncthreads();
    tc_after();
    const uint32_t taddr = s_taddr;
    uint32_t phase = 0;
    bool bad = false;
    for (int it = 0; it < tpb; ++it) {
        const int jt = blockIdx.y * tpb + it;
        if (jt * 4 >= M) break;  // uniform over the block
        const int j = jt * 4 + warp;
        // this row's 16 points (pairs q, q + 1 → one 4-byte store per piece and part)
#pragma unroll 2
        for (int q = 0; q < kRadix; q += 2) {
            float2 v0 = make_float2(0.f, 0.f), v1 = v0;
            const int y0 = q * M + j, y1 = y0 + M;
            if (okc && y0 < rows_in) v0 = in[base + (size_t)y0 * WP];
            if (okc && y1 < rows_in) v1 = in[base + (size_t)y1 * WP];
            __nv_bfloat16 r0[P], r1[P], i0[P], i1[P];
            split_f32<P>(v0.x, r0);
            split_f32<P>(v1.x, r1);
            split_f32<P>(v0.y, i0);
            split_f32<P>(v1.y, i1);
#pragma unroll
            for (int i = 0; i < P; ++i) {
                __nv_bfloat162 re, im;
                re.x = r0[i], re.y = r1[i];
                im.x = i0[i], im.y = i1[i];
                *reinterpret_cast<__nv_bfloat162*>(sA + i * kPieceA + kmaj_off(tid, q)) = re;
                *reinterpret_cast<__nv_bfloat162*>(sA + i * kPieceA + kmaj_off(tid, 16 + q)) = im;
            }
        }
        fence_proxy_async();  // the operand writes, before the tensor cores read them
        tc_before();
        __syncthreads();
        if (tid == 0) {
            tc_after();
            const uint32_t a0 = smem_addr(sA), b0 = smem_addr(sB);
            uint32_t acc = 0;
            // the products with piece indices summing to P − 1 first, the leading one last
            for (int sum = P - 1; sum >= 0; --sum)
                for (int ia = 0; ia <= sum; ++ia)
                    for (int kk = 0; kk < 2; ++kk) {
                        mma_bf16(taddr, smem_desc(a0 + ia * kPieceA + kk * 256),
                                 smem_desc(b0 + (sum - ia) * kPieceB + kk * 256), acc);
                        acc = 1;
                    }
            mma_commit(&bar);
        }
        const bool ok = mbar_wait(&bar, phase);
        phase ^= 1;
        if (__syncthreads_or(!ok)) {
            bad = true;
            break;
        }
        tc_after();
        float d[32];
        tmem_ld32(taddr + ((uint32_t)(warp * 32) << 16), d);
        if (okc) {
#pragma unroll
            for (int r = 0; r < kRadix; ++r) out[base + (size_t)(j * kRadix + r) * WP] = make_float2(d[r], d[16 + r]);
        }
        tc_before();
        __syncthreads();  // every warp's read of the accumulators, before the next tile's MMAs
    }
    if (bad) {
        if (tid == 0) atomicOr(fault, 1u);
        mbar_wait(&bar, phase ^ 1);  // the phase given up on, once more (bounded)
    }
    tc_before();
    __syncthreads();
    if (warp == 0) {
        tc_after();
        tc_dealloc(taddr, kTmemCols);
    }
}

}  // namespace

cudaError_t forward_cols_tc(float2* half, float2* scratch, const MapGeom& g, const CorrPlanDev& plan,
                            const LinePlan& col, int pieces, unsigned* fault, cudaStream_t st) {
    if (col.n != g.ny || col.nst < 2 || col.radix[0] != kRadix || (g.ny / kRadix) % 4 != 0 || !fault ||
        pieces < 1 || pieces > 3)
        return cudaErrorInvalidValue;
    const int ncols = g.nx / 2 + 1, tiles = g.ny / kRadix / 4, tpb = 8;
    const size_t pstride = (size_t)g.ny * g.WP;
    const dim3 grid((ncols + 31) / 32, (tiles + tpb - 1) / tpb, plan.n_real);
    auto k = pieces == 1 ? k_dft16_tc<1> : pieces == 2 ? k_dft16_tc<2> : k_dft16_tc<3>;
    k<<<grid, 128, 0, st>>>(half, scratch, pstride, g.WP, ncols, g.ny, g.ch, tpb, fault);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    // the other stages in FP32 from stage 1; every row of the stage's output is data
    LinePlan rest = col;
    rest.s0 = 1;
    MapGeom gr = g;
    gr.ch = g.ny;
    if ((e = forward_cols_generic(scratch, gr, plan, rest, st)) != cudaSuccess) return e;
    return cudaMemcpy2DAsync(half, g.WP * sizeof(float2), scratch, g.WP * sizeof(float2), ncols * sizeof(float2),
                             (size_t)plan.n_real * g.ny, cudaMemcpyDeviceToDevice, st);
}

}  // namespace zc
