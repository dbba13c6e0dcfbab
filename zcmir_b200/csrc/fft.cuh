// Line FFTs in shared memory for the SMI maps.
//
// A line of n complex points (n = 2^a·3^b, the reference's "ladder" sizes, src/fft.zig:14-34)
// is transformed in place in shared memory by a Stockham autosort schedule of radix-16/8/4/2/3
// stages (radices 16, 8, 4, 2 for the power of two, 3 for each factor 3). Each stage reads every
// butterfly's inputs into registers, synchronises, then twiddles, runs the small DFT and writes
// the outputs at their autosorted places, so one buffer of n points serves all stages.
// Forward: e^{−2πi k t/n}, no scaling; inverse: e^{+2πi k t/n}, no scaling (the 1/(nx·ny) of
// src/fft.zig:280-286 is applied where the correlations are scored).
//
// Shared-memory index padding (one slot per 16 points) keeps the strided writes of the first
// stages free of bank conflicts.
#pragma once

#include "common.cuh"

namespace zc {

constexpr int kMaxStages = 16;
constexpr int kMaxLine = 8192;

struct LinePlan {
    int n;                    // line length
    int nst;                  // number of stages
    int radix[kMaxStages];    // radix of each stage, in order
    int tl;                   // threads per line (each stage's butterflies fit in tl·16/R)
    const float2* tw;         // n twiddles e^{−2πi t/n}, t < n (device memory)
    int s0 = 0;               // first stage run: stages before it were applied by another pass
};

__host__ __device__ __forceinline__ constexpr int pad_idx(int i) { return i + (i >> 4); }
__host__ __device__ __forceinline__ constexpr int padded_len(int n) { return n + (n >> 4) + 1; }
// pitch between lines stored side by side (column tiles): ≡ 4 (mod 16) points, so a half-warp
// touching 4 lines × 4 consecutive points hits 16 distinct bank pairs
__host__ __device__ __forceinline__ constexpr int line_pitch(int n) {
    const int p = padded_len(n);
    return p + ((4 - (p & 15)) & 15);
}

// Pitch between the tx lines of a column tile whose threads run column-fastest (line c = thread
// mod tx): a half-warp then touches min(tx, 16) lines at 16 / min(tx, 16) consecutive points each,
// and the pitch puts them in distinct bank pairs — ≡ 16/tx (mod 16) for tx = 2, 4, 8, odd for
// 16 or more lines (or a count that is not a power of two), where each line is touched once.
__host__ __device__ __forceinline__ constexpr int tile_pitch(int n, int tx) {
    return (tx >= 16 || (tx & (tx - 1)) != 0) ? (padded_len(n) | 1)
                                               : padded_len(n) + (((16 / tx) - (padded_len(n) & 15)) & 15);
}

// Padded slots of the points i0 + r·D (r = 0, 1, ...) from p0 = pad_idx(i0), for a compile-time
// step D, folded to constant offsets: when D is a multiple of 16 every step adds D + D/16; when
// all the points lie in one aligned group of 16 (the caller guarantees it) every step adds D.
template <int D, bool ONE_GROUP = false>
__device__ __forceinline__ int pad_at(int p0, int r) {
    static_assert(D % 16 == 0 || ONE_GROUP, "steps that cross 16-point groups need pad_idx");
    return p0 + r * (D % 16 == 0 ? D + D / 16 : D);
}

// The padded slot of output r of first-stage butterfly j (point j·R0 + r): one aligned group of
// 16 holds the butterfly when R0 divides 16.
template <int R0>
__device__ __forceinline__ int first_slot(int j, int r) {
    if constexpr (16 % R0 == 0) return pad_at<1, true>(pad_idx(j * R0), r);
    else return pad_idx(j * R0 + r);
}

// ── small DFTs, natural order in and out; INV flips the sign of the exponent ──

template <bool INV>
__device__ __forceinline__ float2 mul_mi(float2 a) {  // a·(−i) forward, a·(+i) inverse
    return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

template <bool INV>
__device__ __forceinline__ void dft2(float2* v) {
    const float2 a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
}

template <bool INV>
__device__ __forceinline__ void dft3(float2* v) {
    const float s3 = 0.86602540378443864676f;
    const float2 t = cadd(v[1], v[2]);
    const float2 d = csub(v[1], v[2]);
    const float2 m = make_float2(v[0].x - 0.5f * t.x, v[0].y - 0.5f * t.y);
    const float2 j = mul_mi<INV>(cscale(d, s3));
    v[0] = cadd(v[0], t);
    v[1] = cadd(m, j);
    v[2] = csub(m, j);
}

template <bool INV>
__device__ __forceinline__ void dft4(float2* v) {
    const float2 a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
    const float2 a2 = cadd(v[1], v[3]), a3 = mul_mi<INV>(csub(v[1], v[3]));
    v[0] = cadd(a0, a2);
    v[2] = csub(a0, a2);
    v[1] = cadd(a1, a3);
    v[3] = csub(a1, a3);
}

// dft8 after its first butterfly layer: a_r = v_r + v_{r+4}, b_r = v_r − v_{r+4}
template <bool INV>
__device__ __forceinline__ void dft8_ab(float2 (&a)[4], float2 (&b)[4], float2* v) {
    const float h = 0.70710678118654752440f;
    // b_r ·= w8^r
    b[1] = INV ? make_float2(h * (b[1].x - b[1].y), h * (b[1].x + b[1].y))
               : make_float2(h * (b[1].x + b[1].y), h * (b[1].y - b[1].x));
    b[2] = mul_mi<INV>(b[2]);
    b[3] = INV ? make_float2(-h * (b[3].x + b[3].y), h * (b[3].x - b[3].y))
               : make_float2(h * (b[3].y - b[3].x), -h * (b[3].x + b[3].y));
    dft4<INV>(a);
    dft4<INV>(b);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        v[2 * k] = a[k];
        v[2 * k + 1] = b[k];
    }
}

template <bool INV>
__device__ __forceinline__ void dft8(float2* v) {
    float2 a[4], b[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        a[r] = cadd(v[r], v[r + 4]);
        b[r] = csub(v[r], v[r + 4]);
    }
    dft8_ab<INV>(a, b, v);
}

// dft16 after its first butterfly layer: a_r = v_r + v_{r+8}, d_r = v_r − v_{r+8}
template <bool INV>
__device__ __forceinline__ void dft16_ad(float2 (&a)[8], float2 (&d)[8], float2* v) {
    // w16^r = (cos 2πr/16, ∓sin 2πr/16), r = 0..7
    const float c1 = 0.92387953251128675613f, s1 = 0.38268343236508977173f;
    const float h = 0.70710678118654752440f;
    const float cs[8] = {1.f, c1, h, s1, 0.f, -s1, -h, -c1};
    const float sn[8] = {0.f, s1, h, c1, 1.f, c1, h, s1};
    float2 b[8];
#pragma unroll
    for (int r = 0; r < 8; ++r) {
        const float si = INV ? sn[r] : -sn[r];
        b[r] = make_float2(d[r].x * cs[r] - d[r].y * si, d[r].x * si + d[r].y * cs[r]);
    }
    dft8<INV>(a);
    dft8<INV>(b);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        v[2 * k] = a[k];
        v[2 * k + 1] = b[k];
    }
}

template <bool INV>
__device__ __forceinline__ void dft16(float2* v) {
    float2 a[8], d[8];
#pragma unroll
    for (int r = 0; r < 8; ++r) {
        a[r] = cadd(v[r], v[r + 8]);
        d[r] = csub(v[r], v[r + 8]);
    }
    dft16_ad<INV>(a, d, v);
}

template <int R, bool INV>
__device__ __forceinline__ void dft(float2* v) {
    if constexpr (R == 2) dft2<INV>(v);
    else if constexpr (R == 3) dft3<INV>(v);
    else if constexpr (R == 4) dft4<INV>(v);
    else if constexpr (R == 8) dft8<INV>(v);
    else dft16<INV>(v);
}

// The small DFT of R points whose upper half (v_r, r ≥ R/2) is zero and is not read: the first
// butterfly layer reduces to copies (zero-padded lines: their first stage reads half the points).
template <int R, bool INV>
__device__ __forceinline__ void dft_lo(float2* v) {
    static_assert(R % 2 == 0, "an odd radix has no zero half");
    if constexpr (R == 16) {
        float2 a[8], d[8];
#pragma unroll
        for (int r = 0; r < 8; ++r) a[r] = d[r] = v[r];
        dft16_ad<INV>(a, d, v);
    } else if constexpr (R == 8) {
        float2 a[4], b[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) a[r] = b[r] = v[r];
        dft8_ab<INV>(a, b, v);
    } else if constexpr (R == 4) {
        const float2 a = v[0], b = v[1], mb = mul_mi<INV>(v[1]);
        v[0] = cadd(a, b);
        v[1] = cadd(a, mb);
        v[2] = csub(a, b);
        v[3] = csub(a, mb);
    } else {
        v[1] = v[0];
    }
}

// One Stockham stage of radix R over a line in shared memory. Thread `t` of the line's `tlc`
// threads takes butterflies j = t + b·tlc, b < BM (BM·R ≤ 18 registers of points). Ns: the
// length of the sub-transforms done so far. All threads of the block must call it (it holds two
// __syncthreads); threads without a line pass t ≥ 2^30.
template <int R, int BM, bool INV>
__device__ __noinline__ void fft_stage(float2* __restrict__ buf, const float2* __restrict__ tw,
                                          int n, int Ns, int t, int tlc) {
    const int m = n / R;
    const int tws = n / (Ns * R);
    float2 v[BM][R];
#pragma unroll
    for (int b = 0; b < BM; ++b) {
        const int j = t + b * tlc;
        if (j < m) {
#pragma unroll
            for (int r = 0; r < R; ++r) v[b][r] = buf[pad_idx(j + r * m)];
        }
    }
    __syncthreads();
#pragma unroll
    for (int b = 0; b < BM; ++b) {
        const int j = t + b * tlc;
        if (j < m) {
            const int k = j % Ns;
            if (Ns > 1) {
#pragma unroll
                for (int r = 1; r < R; ++r) {
                    float2 w = __ldg(&tw[r * k * tws]);
                    if (INV) w.y = -w.y;
                    v[b][r] = cmul(v[b][r], w);
                }
            }
            dft<R, INV>(v[b]);
            const int base = (j - k) * R + k;
#pragma unroll
            for (int r = 0; r < R; ++r) buf[pad_idx(base + r * Ns)] = v[b][r];
        }
    }
    __syncthreads();
}

// The whole line: every thread of the block calls it; `t` is the thread's index within its
// line's plan.tl threads (≥ 2^30 for threads without a line).
template <bool INV>
__device__ __forceinline__ void line_fft(float2* __restrict__ buf, const LinePlan& p, int t) {
    int Ns = 1;
    for (int s = 0; s < p.s0; ++s) Ns *= p.radix[s];
    for (int s = p.s0; s < p.nst; ++s) {
        const int R = p.radix[s];
        switch (R) {
            case 16: fft_stage<16, 1, INV>(buf, p.tw, p.n, Ns, t, p.tl); break;
            case 8: fft_stage<8, 2, INV>(buf, p.tw, p.n, Ns, t, p.tl); break;
            case 4: fft_stage<4, 4, INV>(buf, p.tw, p.n, Ns, t, p.tl); break;
            case 2: fft_stage<2, 8, INV>(buf, p.tw, p.n, Ns, t, p.tl); break;
            default: fft_stage<3, 6, INV>(buf, p.tw, p.n, Ns, t, p.tl); break;
        }
        Ns *= R;
    }
}

// ── lines of N = 2^a·3^b points with the whole schedule known at compile time ──
// ⌈a/4⌉ power-of-two stages with balanced radices (16/8/4/2), then b radix-3 stages; TL threads
// per line, each taking ⌈(N/R)/TL⌉ butterflies of a radix-R stage. Strides, twiddle steps and
// index arithmetic fold to constants.
constexpr int ilog2(int n) { return n <= 1 ? 0 : 1 + ilog2(n >> 1); }
constexpr int twos_of(int n) { return (n > 0 && n % 2 == 0) ? 1 + twos_of(n / 2) : 0; }
constexpr int threes_of(int n) { return (n > 0 && n % 3 == 0) ? 1 + threes_of(n / 3) : 0; }
constexpr int ipow(int b, int e) { return e == 0 ? 1 : b * ipow(b, e - 1); }

// The schedule of a line of n = 2^a·3^b points (compile-time for the kernels, run-time for the
// host building the twiddle tables): the number of stages and stage s's radix.
__host__ __device__ constexpr int mix_stages(int n) { return (twos_of(n) + 3) / 4 + threes_of(n); }
__host__ __device__ constexpr int mix_radix(int n, int s) {
    return s < (twos_of(n) + 3) / 4
               ? 1 << (twos_of(n) / ((twos_of(n) + 3) / 4) + (s < twos_of(n) % ((twos_of(n) + 3) / 4) ? 1 : 0))
               : 3;
}
// Per-stage twiddle tables, after the n entries e^{−2πi t/n} of a line's table: stage s (radix R,
// NS points transformed before it, NS > 1) holds w(r, k) = e^{−2πi r k/(NS·R)} at
// (r − 1)·NS + k, r = 1..R−1, k < NS, so the threads of a stage (consecutive k) read consecutive
// entries. stage_tw_off: where stage s's table starts (past the n entries); its value at
// s = mix_stages(n) is the tables' total length.
__host__ __device__ constexpr int stage_tw_off(int n, int s) {
    int off = 0, ns = 1;
    for (int i = 0; i < s; ++i) {
        const int r = mix_radix(n, i);
        if (ns > 1) off += (r - 1) * ns;
        ns *= r;
    }
    return off;
}

template <int N>
struct Mix {
    static constexpr int kA = twos_of(N), kB = threes_of(N);
    static_assert(ipow(2, twos_of(N)) * ipow(3, threes_of(N)) == N, "line length must be 2^a·3^b");
    static constexpr int kP2 = (kA + 3) / 4;
    static constexpr int kStages = kP2 + kB;
    static_assert(kStages == mix_stages(N), "stage count");
    static constexpr int radix(int s) { return mix_radix(N, s); }
};

// One stage of a compile-time line; OFF: this stage's twiddle table (stage_tw_off).
template <int R, int NS, int N, int TL, bool INV, int OFF>
__device__ __forceinline__ void mix_stage(float2* __restrict__ buf, const float2* __restrict__ tw, int t, bool act) {
    constexpr int M = N / R, BM = (M + TL - 1) / TL;
    float2 v[BM][R];
    if (act) {
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
    }
    __syncthreads();
    if (act) {
#pragma unroll
        for (int b = 0; b < BM; ++b) {
            const int j = t + b * TL;
            if (M % TL == 0 || j < M) {
                const int k = j % NS;
                if (NS > 1) {
#pragma unroll
                    for (int r = 1; r < R; ++r) {
                        float2 w = __ldg(&tw[N + OFF + (r - 1) * NS + k]);
                        if (INV) w.y = -w.y;
                        v[b][r] = cmul(v[b][r], w);
                    }
                }
                dft<R, INV>(v[b]);
                const int base = (j - k) * R + k;
                // a butterfly's outputs are R points NS apart from base; when R·NS divides 16
                // they lie in one aligned group of 16 (base mod R·NS = k < NS)
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
    }
    __syncthreads();
}

template <int N, int TL, bool INV, int S = 0, int NS = 1>
__device__ __forceinline__ void mix_fft(float2* __restrict__ buf, const float2* __restrict__ tw, int t, bool act) {
    if constexpr (S < Mix<N>::kStages) {
        constexpr int R = Mix<N>::radix(S);
        mix_stage<R, NS, N, TL, INV, stage_tw_off(N, S)>(buf, tw, t, act);
        mix_fft<N, TL, INV, S + 1, NS * R>(buf, tw, t, act);
    }
}

// The stages after the first and before the last (S = 1 .. kStages − 2), through shared memory.
template <int N, int TL, bool INV, int S, int NS>
__device__ __forceinline__ void mix_mid(float2* __restrict__ buf, const float2* __restrict__ tw, int t, bool act) {
    if constexpr (S < Mix<N>::kStages - 1) {
        constexpr int R = Mix<N>::radix(S);
        mix_stage<R, NS, N, TL, INV, stage_tw_off(N, S)>(buf, tw, t, act);
        mix_mid<N, TL, INV, S + 1, NS * R>(buf, tw, t, act);
    }
}

// the last stage of a compile-time line, its outputs to out(y, v)
template <int N, int TL, bool INV, class Out>
__device__ __forceinline__ void mix_last(float2* __restrict__ buf, const float2* __restrict__ tw, int t, bool act,
                                         Out&& out) {
    using MX = Mix<N>;
    constexpr int RL = MX::radix(MX::kStages - 1), NSL = N / RL, ML = N / RL, BML = (ML + TL - 1) / TL;
    if (act) {
#pragma unroll 1
        for (int b = 0; b < BML; ++b) {
            const int j = t + b * TL;
            if (ML % TL == 0 || j < ML) {
                float2 v[RL];
                if constexpr (ML % 16 == 0) {
                    const int p = pad_idx(j);
#pragma unroll
                    for (int r = 0; r < RL; ++r) v[r] = buf[pad_at<ML>(p, r)];
                } else {
#pragma unroll
                    for (int r = 0; r < RL; ++r) v[r] = buf[pad_idx(j + r * ML)];
                }
                // k = j mod NSL = j
                constexpr int OFFL = stage_tw_off(N, MX::kStages - 1);
#pragma unroll
                for (int r = 1; r < RL; ++r) {
                    float2 w = __ldg(&tw[N + OFFL + (r - 1) * NSL + j]);
                    if (INV) w.y = -w.y;
                    v[r] = cmul(v[r], w);
                }
                dft<RL, INV>(v);
#pragma unroll
                for (int r = 0; r < RL; ++r) out(j + r * NSL, v[r]);
            }
        }
    }
}

// The first stage's butterfly j from in(y), y = j + r·M0: all R0 points, or with LO (the line's
// points y ≥ N/2 are zero, R0 even) only the lower R0/2, and the transformed points left in v.
template <int R0, int M0, bool INV, bool LO, class In>
__device__ __forceinline__ void first_in(float2 (&v)[R0], int j, In& in) {
    if constexpr (LO && R0 % 2 == 0) {
#pragma unroll
        for (int r = 0; r < R0 / 2; ++r) v[r] = in(j + r * M0);
        dft_lo<R0, INV>(v);
    } else {
#pragma unroll
        for (int r = 0; r < R0; ++r) v[r] = in(j + r * M0);
        dft<R0, INV>(v);
    }
}

// The whole line with its ends in registers: the first stage's butterflies take their inputs
// straight from in(y) (point y of the line, typically a global load) and the last stage hands
// its outputs to out(y, v), so the line is staged into and out of shared memory by neither the
// caller nor this function (two shared-memory passes fewer than run()). Every thread of the
// block calls it; buf is this thread's line buffer (padded_len(N) points). On return the
// buffer may still be read by other threads of the line: synchronise before reusing it.
template <int N, int TL, bool INV, bool LO = false, class In, class Out>
__device__ __forceinline__ void mix_fft_io(float2* __restrict__ buf, const float2* __restrict__ tw, int t, bool act,
                                           In&& in, Out&& out) {
    using MX = Mix<N>;
    static_assert(MX::kStages >= 2, "a line of one stage has no middle to run through shared memory");
    constexpr int R0 = MX::radix(0), M0 = N / R0, BM0 = (M0 + TL - 1) / TL;
    if (act) {
#pragma unroll
        for (int b = 0; b < BM0; ++b) {
            const int j = t + b * TL;
            if (M0 % TL == 0 || j < M0) {
                float2 v[R0];
                first_in<R0, M0, INV, LO>(v, j, in);
#pragma unroll
                for (int r = 0; r < R0; ++r) buf[first_slot<R0>(j, r)] = v[r];
            }
        }
    }
    __syncthreads();
    mix_mid<N, TL, INV, 1, R0>(buf, tw, t, act);
    mix_last<N, TL, INV>(buf, tw, t, act, out);
}

// The whole line with its first stage's inputs already in registers: v = this thread's one
// butterfly (j = t, so the first stage's butterflies must number exactly TL), then as mix_fft_io,
// with between() called once the first stage has consumed v. Lets a caller start loading the next
// line's inputs while this one transforms.
template <int N, int TL, bool INV, class Out, class Between>
__device__ __forceinline__ void mix_fft_regs(float2* __restrict__ buf, const float2* __restrict__ tw, int t, bool act,
                                             float2 (&v)[Mix<N>::radix(0)], Out&& out, Between&& between) {
    constexpr int R0 = Mix<N>::radix(0);
    static_assert(N / R0 == TL, "one first-stage butterfly per thread");
    if (act) {
        dft<R0, INV>(v);
#pragma unroll
        for (int r = 0; r < R0; ++r) buf[first_slot<R0>(t, r)] = v[r];
    }
    __syncthreads();
    between();  // after the first stage: v is consumed, so the caller may refill its source
    mix_mid<N, TL, INV, 1, R0>(buf, tw, t, act);
    mix_last<N, TL, INV>(buf, tw, t, act, out);
}


// The whole line with its first stage fed from in(y) (as mix_fft_io) and the result left in buf
// in natural order, the block synchronised, as run() leaves it.
template <int N, int TL, bool INV, bool LO = false, class In>
__device__ __forceinline__ void mix_fft_in(float2* __restrict__ buf, const float2* __restrict__ tw, int t, bool act,
                                           In&& in) {
    constexpr int R0 = Mix<N>::radix(0), M0 = N / R0, BM0 = (M0 + TL - 1) / TL;
    if (act) {
#pragma unroll
        for (int b = 0; b < BM0; ++b) {
            const int j = t + b * TL;
            if (M0 % TL == 0 || j < M0) {
                float2 v[R0];
                first_in<R0, M0, INV, LO>(v, j, in);
#pragma unroll
                for (int r = 0; r < R0; ++r) buf[first_slot<R0>(j, r)] = v[r];
            }
        }
    }
    __syncthreads();
    mix_fft<N, TL, INV, 1, R0>(buf, tw, t, act);
}

// Line-FFT policies the map kernels are written against: n(), threads per line, run<INV>(),
// run_io<INV, LO>(buf, t, act, in, out) (mix_fft_io's contract) and run_in<INV, LO>(buf, t, act,
// in); LO: the caller guarantees in(y) = 0 for y ≥ n/2, so a compile-time line reads only y < n/2.
struct GenericLine {
    LinePlan p;
    __host__ __device__ __forceinline__ int n() const { return p.n; }
    __host__ __device__ __forceinline__ int tl() const { return p.tl; }
    template <bool INV>
    __device__ __forceinline__ void run(float2* buf, int t, bool act) const {
        line_fft<INV>(buf, p, act ? t : (1 << 30));
    }
    // runtime lines stage through shared memory around the transform (LO: no shortcut)
    template <bool INV, bool LO = false, class In, class Out>
    __device__ __forceinline__ void run_io(float2* buf, int t, bool act, In&& in, Out&& out) const {
        const bool a = act && t < p.tl;
        if (a)
            for (int y = t; y < p.n; y += p.tl) buf[pad_idx(y)] = in(y);
        __syncthreads();
        line_fft<INV>(buf, p, a ? t : (1 << 30));
        if (a)
            for (int y = t; y < p.n; y += p.tl) out(y, buf[pad_idx(y)]);
    }
    template <bool INV, bool LO = false, class In>
    __device__ __forceinline__ void run_in(float2* buf, int t, bool act, In&& in) const {
        const bool a = act && t < p.tl;
        if (a)
            for (int y = t; y < p.n; y += p.tl) buf[pad_idx(y)] = in(y);
        __syncthreads();
        line_fft<INV>(buf, p, a ? t : (1 << 30));
    }
};

// A compile-time line of N = 2^a·3^b points. TPL: threads per line (N/16 by default: one
// radix-16 butterfly each; N/8 gives every thread 8 points of the loads and stores around the
// transform, half of them idle in radix-16 stages)
template <int N, int TPL = N / 16>
struct FixedLine {
    const float2* tw;
    __host__ __device__ __forceinline__ static constexpr int n() { return N; }
    __host__ __device__ __forceinline__ static constexpr int tl() { return TPL; }
    template <bool INV>
    __device__ __forceinline__ void run(float2* buf, int t, bool act) const {
        mix_fft<N, TPL, INV>(buf, tw, t, act && t < TPL);
    }
    template <bool INV, bool LO = false, class In, class Out>
    __device__ __forceinline__ void run_io(float2* buf, int t, bool act, In&& in, Out&& out) const {
        mix_fft_io<N, TPL, INV, LO>(buf, tw, t, act && t < TPL, in, out);
    }
    template <bool INV, bool LO = false, class In>
    __device__ __forceinline__ void run_in(float2* buf, int t, bool act, In&& in) const {
        mix_fft_in<N, TPL, INV, LO>(buf, tw, t, act && t < TPL, in);
    }
};

template <int N, int TPL = N / 16>
using Pow2Line = FixedLine<N, TPL>;

}  // namespace zc
