// Block FFTs of length N = 3P (P = 2^k, 128 <= P <= 2048) for sm_100a.
//
// These sizes exist for the reduced-size correlation: its exact size only has to reach
// L + W - 1 per axis, and 3 * 2^k lands closer to that than the next power of two
// (384^2 templates with 1024^2 windows need 1407: 1536 instead of 2048, 56 % of the
// transform grid).  The reference transforms only powers of two; these lengths are
// internal to the batched correlation and never visible in a plan.
//
// One length-3P FFT is computed by T = 3 T' threads (T' = P/16): three sub-FFTs of length
// P (BlockFft<P>; thread (k2, j) = sub-FFT k2, lane j) and one radix-3 step, with
// n = n1 + P n2 and k = 3 k1 + k2 (n1, k1 < P; n2, k2 < 3):
//   forward, decimation in frequency:
//     y_k2[n1] = W_3P^(n1 k2) sum_n2 W_3^(n2 k2) x[n1 + P n2],   X[3 k1 + k2] = DFT_P(y_k2)[k1]
//   inverse, decimation in time:
//     z_k2 = IDFT_P(X[3 k1 + k2]),   x[n1 + P n2] = sum_k2 W_3^(-n2 k2) W_3P^(-n1 k2) z_k2[n1]
// The time domain stays in natural order on both sides: each thread forms its forward
// inputs y_k2[n1] from three natural-order loads (one when the data end before P), and the
// inverse ends with one radix-3 pass through shared memory whose outputs are contiguous in
// n1.  The spectrum lives in registers decimated by 3: thread (k2, j) holds X[k] for
// k = 3 (j + T' q) + k2, which is where a pointwise product (the correlation's conj(T) * I)
// is applied without any exchange.
#pragma once

#include "fft_core.cuh"

namespace ffb {

constexpr int kMinP3 = 128;
constexpr int kMaxP3 = 2048;

__host__ __device__ constexpr bool is_pow2_size(int n) { return n > 0 && (n & (n - 1)) == 0; }
// N = 3P with a supported P
__host__ __device__ constexpr bool is_3p_size(int n) {
    return n > 0 && n % 3 == 0 && is_pow2_size(n / 3) && n / 3 >= kMinP3 && n / 3 <= kMaxP3;
}

// Twiddles of the radix-3 pass: W_3P^m = exp(-2 pi i m / 3P), m < 2P, one block per P.
constexpr int tw3_size_of(int p) { return 2 * p; }
constexpr int tw3_base(int p) {
    int off = 0;
    for (int q = kMinP3; q < p; q *= 2) off += tw3_size_of(q);
    return off;
}
constexpr int kTw3Total = tw3_base(kMaxP3) + tw3_size_of(kMaxP3);

template <int P>
struct Fft3Shape {
    static_assert(P >= kMinP3 && P <= kMaxP3 && (P & (P - 1)) == 0, "P must be a power of two in [128, 2048]");
    static constexpr int N = 3 * P;
    static constexpr int LOGP = ilog2(P);
    static constexpr int TP = P / 16;                  // threads per sub-FFT
    static constexpr int T = 3 * TP;                   // threads per FFT
    static constexpr int SUB = FftShape<P>::SMEM_PAD;  // float2 per sub-FFT region
    // Region and FFT strides of the row C2R, which writes its input spectrum decimated by 3
    // (Z[k] of FFT ff in region k % 3 at phys(k / 3)); a warp's scatter covers 8 consecutive
    // k of each of 4 FFTs (P = 512; 2..16 FFTs per block at the other sizes).  The offsets past
    // a multiple of 16 are the ones a bank model of that scatter finds best for the block
    // shape of each P (at P = 512: 400 instead of 768 wavefronts per block); the sub-FFT
    // exchanges read and write within one region and are conflict-free for any offset.
    static constexpr int C2R_SUB_EXTRA = P == 128 ? 5 : P == 256 ? 1 : P == 512 ? 3 : P == 1024 ? 3 : 11;
    static constexpr int C2R_FFT_EXTRA = P == 128 ? 0 : P == 256 ? 3 : P == 512 ? 3 : P == 1024 ? 15 : 0;
    static constexpr int SUB_C2R = (FftShape<P>::SMEM + 15) / 16 * 16 + C2R_SUB_EXTRA;
    static constexpr int SMEM = 3 * SUB;               // float2 per exchange buffer
    static constexpr int ROUNDS = (P + T - 1) / T;     // radix-3 items per thread (6)
};

// shared-memory position of spectrum index k (natural order) inside one buffer
template <int P>
__device__ __forceinline__ int loc3(int k) {
    return (k >> Fft3Shape<P>::LOGP) * Fft3Shape<P>::SUB + phys(k & (P - 1));
}

// Exchange buffers and barriers of one length-3P FFT inside a block of FPB FFTs.
//   begin()/sync()  : the sub-FFT view handed to BlockFft<P>.  A sub-FFT only exchanges
//                     within its own region, so it synchronises only its own threads:
//                     __syncwarp() when it fits in one warp (P <= 512), else its own named
//                     barrier (1 + FPB + 3 f + k2, T' threads).
//   begin_full()/sync_fft() : the whole FFT (the radix-3 step reads all three regions):
//                     bar.sync 1 + f, T when T is a whole number of warps and the block
//                     holds several FFTs, else __syncthreads().
// Every buffer that the radix-3 step reads across regions is rewritten only after a
// sync_fft() that all its readers passed (the kernels call sync_fft() where a sub-FFT
// exchange follows such reads).  Double buffering (DB) as in FftGroup.
template <int P, int FPB, bool DB, int SUBX = Fft3Shape<P>::SUB, int PADX = 0>
struct Fft3Group {
    using S3 = Fft3Shape<P>;
    static constexpr int T = S3::T;
    static constexpr int TP = S3::TP;
    static_assert(SUBX >= FftShape<P>::SMEM, "a region must hold one sub-FFT's exchange");
    static constexpr int SUB = SUBX;                  // region stride (float2)
    static constexpr int SMEM = 3 * SUBX;             // float2 per exchange buffer
    static constexpr int STRIDE = (DB ? 2 : 1) * SMEM + PADX;  // float2 per FFT
    static constexpr int BYTES = FPB * STRIDE * (int)sizeof(float2);
    static_assert(TP <= 32 || 4 * FPB <= 15, "named barriers: FFT ids 1..FPB, sub-FFT ids FPB+1..4 FPB");
    float2* base;
    int f;
    int r;
    int k;

    __device__ __forceinline__ Fft3Group(float2* smem_block, int group, int sub)
        : base(smem_block + group * STRIDE), f(group), r(sub), k(0) {}

    __device__ __forceinline__ void sync_fft() const {
        if constexpr (T % 32 == 0 && FPB > 1 && FPB <= 15) {
            asm volatile("bar.sync %0, %1;" ::"r"(f + 1), "n"(T) : "memory");
        } else {
            __syncthreads();
        }
    }

    __device__ __forceinline__ void sync() const {
        if constexpr (TP <= 32) {
            __syncwarp();
        } else {
            asm volatile("bar.sync %0, %1;" ::"r"(1 + FPB + 3 * f + r), "n"(TP) : "memory");
        }
    }

    __device__ __forceinline__ float2* next_buffer(bool sub_level) {
        float2* p = base;
        if constexpr (DB) {
            p += (k & 1) * SMEM;
        } else {
            if (sub_level) sync(); else sync_fft();
        }
        k++;
        return p;
    }

    __device__ __forceinline__ float2* begin_full() { return next_buffer(false); }
    __device__ __forceinline__ float2* begin() { return next_buffer(true) + r * SUB; }
    // Whole buffer for a step in which each sub-FFT first writes only its own region: the
    // region's earlier readers in the FFT are that sub-FFT's own threads, so the sub-level
    // wait suffices (the caller's reads across regions follow a sync_fft()).
    __device__ __forceinline__ float2* begin_own() { return next_buffer(true); }
};

constexpr float kH3 = 0.866025403784438646764f;  // sqrt(3)/2

// In-place inverse DFT3 of (a, b, c) (W_3 = exp(+2 pi i / 3)).
__device__ __forceinline__ void idft3(float2& a, float2& b, float2& c) {
    const float2 s = cadd(b, c), d = csub(b, c);
    const float2 m = make_float2(fmaf(-0.5f, s.x, a.x), fmaf(-0.5f, s.y, a.y));
    a = cadd(a, s);
    const float hx = kH3 * d.x, hy = kH3 * d.y;
    b = make_float2(m.x - hy, m.y + hx);
    c = make_float2(m.x + hy, m.y - hx);
}

// Component k2 of the forward DFT3 of (x0, x1, x2): x0 + W_3^k2 x1 + W_3^(2 k2) x2.
__device__ __forceinline__ float2 dft3_component(float2 x0, float2 x1, float2 x2, int k2) {
    const float2 s = cadd(x1, x2);
    if (k2 == 0) return cadd(x0, s);
    const float2 d = csub(x1, x2);
    const float2 m = make_float2(fmaf(-0.5f, s.x, x0.x), fmaf(-0.5f, s.y, x0.y));
    const float hs = k2 == 1 ? -kH3 : kH3;  // -i h d for k2 = 1, +i h d for k2 = 2
    return make_float2(fmaf(-hs, d.y, m.x), fmaf(hs, d.x, m.y));
}

// Forward input y_k2[n1] of thread (k2, .) from x[n1], x[n1 + P], x[n1 + 2P].
template <int P>
__device__ __forceinline__ float2 dif_input(float2 x0, float2 x1, float2 x2, int n1, int k2,
                                            const float2* __restrict__ tw3) {
    const float2 y = dft3_component(x0, x1, x2, k2);
    return k2 == 0 ? y : cmul(y, ld_tw(tw3 + n1 * k2));
}

// Final radix-3 pass of the inverse.  v: z_k2[n1] of thread (k2 = g.r, j), n1 = j + T' q.
// Writes them to region k2 of the next buffer, waits for the FFT's threads, then thread t
// produces x[n1], x[n1 + P], x[n1 + 2P] for n1 = t + T i and hands each to store(n, value).
// Output pruning: only the outputs n < keep are formed (every output needs all three
// sub-FFT values, so the pruning is of this last combination only; keep = 3P forms all).
// The cross-region reads here must be followed by a sync_fft() before any later write to the
// buffer (the batched kernel's next template begins with one).
template <int P, class G, class Store>
__device__ __forceinline__ void dit_output(float2 (&v)[16], G& g, int j, int t, const float2* __restrict__ tw3,
                                           Store store, int keep = 3 * P) {
    using S3 = Fft3Shape<P>;
    float2* buf = g.begin_own();
    {
        float2* s = buf + g.r * G::SUB;
#pragma unroll
        for (int q = 0; q < 16; q++) s[phys(j + S3::TP * q)] = v[q];
    }
    g.sync_fft();
    const int lim = keep < P ? keep : P;
#pragma unroll 2
    for (int i = 0; i < S3::ROUNDS; i++) {
        const int n1 = t + S3::T * i;
        if (n1 < lim) {
            const int p = phys(n1);
            const float2 a = buf[p];
            const float2 w1 = ld_tw(tw3 + n1), w2 = cmul(w1, w1);  // one load: W^2n1 = (W^n1)^2
            const float2 b = cmulc(buf[G::SUB + p], w1);
            const float2 c = cmulc(buf[2 * G::SUB + p], w2);
            // inverse DFT3 of (a, b, c), W_3 = exp(+2 pi i / 3), formed only where kept
            const float2 s = cadd(b, c);
            store(n1, cadd(a, s));
            if (n1 + P < keep) {
                const float2 d = csub(b, c);
                const float2 m = make_float2(fmaf(-0.5f, s.x, a.x), fmaf(-0.5f, s.y, a.y));
                const float hx = kH3 * d.x, hy = kH3 * d.y;
                store(n1 + P, make_float2(m.x - hy, m.y + hx));
                if (n1 + 2 * P < keep) store(n1 + 2 * P, make_float2(m.x + hy, m.y - hx));
            }
        }
    }
}

// Forward in decimation-in-time form, for callers whose input ends well before P and whose
// output goes to shared memory anyway (the row R2C): thread (r, j) loads x[3 m + r],
// m = j + T' q, so the three sub-FFTs share the data instead of each reading all of it;
// the radix-3 step X[k1 + P k2] = sum_r W_3^(r k2) W_3P^(r k1) Y_r[k1] then runs through
// shared memory and leaves X in natural order at loc3<P>(k).  Returns that buffer after a
// barrier of the FFT's threads.
template <int P, class G>
__device__ __forceinline__ float2* forward_dit(float2 (&v)[16], G& g, int j, int t, const float2* __restrict__ tw,
                                               const float2* __restrict__ tw3, int qnz) {
    using S3 = Fft3Shape<P>;
    BlockFft<P, false>::run(v, g, j, tw, qnz);
    float2* buf = g.begin_own();
    {
        float2* s = buf + g.r * G::SUB;
#pragma unroll
        for (int q = 0; q < 16; q++) s[phys(j + S3::TP * q)] = v[q];
    }
    g.sync_fft();
#pragma unroll 2
    for (int i = 0; i < S3::ROUNDS; i++) {
        const int k1 = t + S3::T * i;
        if (k1 < P) {
            const int p = phys(k1);
            const float2 a = buf[p];
            const float2 w1 = ld_tw(tw3 + k1), w2 = cmul(w1, w1);
            const float2 b = cmul(buf[G::SUB + p], w1);
            const float2 c = cmul(buf[2 * G::SUB + p], w2);
            buf[p] = dft3_component(a, b, c, 0);
            buf[G::SUB + p] = dft3_component(a, b, c, 1);
            buf[2 * G::SUB + p] = dft3_component(a, b, c, 2);
        }
    }
    g.sync_fft();
    return buf;
}

// leading q slots of thread (r, j) that can be non-zero when x[3 (j + T' q) + r] is
// loaded only below L
template <int P>
__device__ __forceinline__ int leading_slots_dit(int L, int r, int j) {
    constexpr int TP = Fft3Shape<P>::TP;
    const int Lr = L > r ? (L - r + 2) / 3 : 0;  // count of m with 3 m + r < L
    if (Lr <= j) return 0;
    const int q = (Lr - j + TP - 1) / TP;
    return q > 16 ? 16 : q;
}

// number of leading q slots (n1 = j + T' q) that can be non-zero when only x[n], n < L,
// is loaded: n1 < min(L, P)
template <int P>
__device__ __forceinline__ int leading_slots3(int L, int j) {
    constexpr int TP = Fft3Shape<P>::TP;
    const int Ln = L < P ? L : P;
    if (Ln <= j) return 0;
    const int q = (Ln - j + TP - 1) / TP;
    return q > 16 ? 16 : q;
}

}  // namespace ffb
