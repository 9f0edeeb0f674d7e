// Block FFTs of length N = R P (R = 3, 5 or 7, P = 2^k) for sm_100a.
//
// These sizes exist for the reduced-size correlation and the 2D plans beyond powers of two:
// the correlation's exact size only has to reach L + W - 1 per axis, and R * 2^k lands closer
// to that than the next power of two (384^2 templates with 1024^2 windows need 1407: 1536
// instead of 2048, 56 % of the transform grid; 128^2 templates with 512^2 windows need 639:
// 640 = 5 * 128 instead of 768).  The reference transforms only powers of two.
//
// One length-RP FFT is computed by T = R T' threads (T' = P/16): R sub-FFTs of length P
// (BlockFft<P>; thread (k2, j) = sub-FFT k2, lane j) and one radix-R step, with
// n = n1 + P n2 and k = R k1 + k2 (n1, k1 < P; n2, k2 < R):
//   forward, decimation in frequency:
//     y_k2[n1] = W_RP^(n1 k2) sum_n2 W_R^(n2 k2) x[n1 + P n2],   X[R k1 + k2] = DFT_P(y_k2)[k1]
//   inverse, decimation in time:
//     z_k2 = IDFT_P(X[R k1 + k2]),   x[n1 + P n2] = sum_k2 W_R^(-n2 k2) W_RP^(-n1 k2) z_k2[n1]
// The time domain stays in natural order on both sides: each thread forms its forward
// inputs y_k2[n1] from R natural-order loads (one when the data end before P), and the
// inverse ends with one radix-R pass through shared memory whose outputs are contiguous in
// n1.  The spectrum lives in registers decimated by R: thread (k2, j) holds X[k] for
// k = R (j + T' q) + k2, which is where a pointwise product (the correlation's conj(T) * I)
// is applied without any exchange.
#pragma once

#include "fft_core.cuh"

namespace ffb {

constexpr int kMinP3 = 128;
constexpr int kMaxP3 = 2048;
constexpr int kMaxP5 = 1024;   // 5 * 1024 = 5120 <= 8192, the longest transform of a plan
constexpr int kMaxP7 = 512;    // 7 * 512 = 3584

__host__ __device__ constexpr bool is_pow2_size(int n) { return n > 0 && (n & (n - 1)) == 0; }
// N = 3P with a supported P
__host__ __device__ constexpr bool is_3p_size(int n) {
    return n > 0 && n % 3 == 0 && is_pow2_size(n / 3) && n / 3 >= kMinP3 && n / 3 <= kMaxP3;
}
// N = 5P with a supported P
__host__ __device__ constexpr bool is_5p_size(int n) {
    return n > 0 && n % 5 == 0 && is_pow2_size(n / 5) && n / 5 >= kMinP3 && n / 5 <= kMaxP5;
}
// N = 7P with a supported P
__host__ __device__ constexpr bool is_7p_size(int n) {
    return n > 0 && n % 7 == 0 && is_pow2_size(n / 7) && n / 7 >= kMinP3 && n / 7 <= kMaxP7;
}
__host__ __device__ constexpr bool is_rp_size(int n) { return is_3p_size(n) || is_5p_size(n) || is_7p_size(n); }
// Lengths of the chirp-z (Bluestein) path (kernels_blue.cuh): any other length in [17, 4096],
// on the power-of-two block FFT of length blue_m(n) >= 2n - 1.
constexpr int kMaxBlueN = 4096;
__host__ __device__ constexpr bool is_blue_size(int n) {
    return n >= 17 && n <= kMaxBlueN && !is_pow2_size(n) && !is_rp_size(n);
}
__host__ __device__ constexpr int blue_m(int n) {
    int m = 64;
    while (m < 2 * n - 1) m *= 2;
    return m;
}
// the radix R of a length R * 2^k (1 for a power of two)
__host__ __device__ constexpr int radix_of(int n) {
    return is_3p_size(n) ? 3 : is_5p_size(n) ? 5 : is_7p_size(n) ? 7 : 1;
}

// Twiddles of the radix-R pass: W_RP^m = exp(-2 pi i m / RP), m < (R - 1) P, one block per P.
__host__ __device__ constexpr int kMaxPR(int r) { return r == 3 ? kMaxP3 : r == 5 ? kMaxP5 : kMaxP7; }
__host__ __device__ constexpr int twr_size_of(int r, int p) { return (r - 1) * p; }
__host__ __device__ constexpr int twr_base(int r, int p) {
    int off = 0;
    for (int q = kMinP3; q < p; q *= 2) off += twr_size_of(r, q);
    return off;
}
__host__ __device__ constexpr int twr_total(int r) { return twr_base(r, kMaxPR(r)) + twr_size_of(r, kMaxPR(r)); }
constexpr int kTw3Total = twr_total(3);
constexpr int kTw5Total = twr_total(5);
constexpr int kTw7Total = twr_total(7);

template <int R, int P>
struct FftRShape {
    static_assert(R == 3 || R == 5 || R == 7, "radix 3, 5 or 7");
    static_assert(P >= kMinP3 && P <= kMaxPR(R) && (P & (P - 1)) == 0, "P must be a supported power of two");
    static constexpr int N = R * P;
    static constexpr int LOGP = ilog2(P);
    static constexpr int TP = P / 16;                  // threads per sub-FFT
    static constexpr int T = R * TP;                   // threads per FFT
    static constexpr int SUB = FftShape<P>::SMEM_PAD;  // float2 per sub-FFT region
    // Region and FFT strides of the row C2R, which writes its input spectrum decimated by R
    // (Z[k] of FFT ff in region k % R at phys(k / R)); a warp's scatter covers consecutive k
    // of several FFTs.  For R = 3 the offsets past a multiple of 16 are the ones a bank model
    // of that scatter finds best for the block shape of each P (at P = 512: 400 instead of
    // 768 wavefronts per block); for R = 5 and 7 an odd region offset.  The sub-FFT exchanges read
    // and write within one region and are conflict-free for any offset.
    static constexpr int C2R_SUB_EXTRA =
        R != 3 ? 1 : P == 128 ? 5 : P == 256 ? 1 : P == 512 ? 3 : P == 1024 ? 3 : 11;
    static constexpr int C2R_FFT_EXTRA = R != 3 ? 0 : P == 128 ? 0 : P == 256 ? 3 : P == 512 ? 3 : P == 1024 ? 15 : 0;
    static constexpr int SUB_C2R = (FftShape<P>::SMEM + 15) / 16 * 16 + C2R_SUB_EXTRA;
    static constexpr int SMEM = R * SUB;               // float2 per exchange buffer
    static constexpr int ROUNDS = (P + T - 1) / T;     // radix-R items per thread
};

// shared-memory position of spectrum index k (natural order) inside one buffer
template <int R, int P>
__device__ __forceinline__ int locR(int k) {
    return (k >> FftRShape<R, P>::LOGP) * FftRShape<R, P>::SUB + phys(k & (P - 1));
}

// Exchange buffers and barriers of one length-RP FFT inside a block of FPB FFTs.
//   begin()/sync()  : the sub-FFT view handed to BlockFft<P>.  A sub-FFT only exchanges
//                     within its own region, so it synchronises only its own threads:
//                     __syncwarp() when it fits in one warp (P <= 512), else its own named
//                     barrier (1 + FPB + R f + k2, T' threads).
//   begin_full()/sync_fft() : the whole FFT (the radix-R step reads all regions):
//                     bar.sync 1 + f, T when T is a whole number of warps and the block
//                     holds several FFTs, else __syncthreads().
// Every buffer that the radix-R step reads across regions is rewritten only after a
// sync_fft() that all its readers passed (the kernels call sync_fft() where a sub-FFT
// exchange follows such reads).  Double buffering (DB) as in FftGroup.
template <int R, int P, int FPB, bool DB, int SUBX = FftRShape<R, P>::SUB, int PADX = 0>
struct FftRGroup {
    using S3 = FftRShape<R, P>;
    static constexpr int T = S3::T;
    static constexpr int TP = S3::TP;
    static_assert(SUBX >= FftShape<P>::SMEM, "a region must hold one sub-FFT's exchange");
    static constexpr int SUB = SUBX;                  // region stride (float2)
    static constexpr int SMEM = R * SUBX;             // float2 per exchange buffer
    static constexpr int STRIDE = (DB ? 2 : 1) * SMEM + PADX;  // float2 per FFT
    static constexpr int BYTES = FPB * STRIDE * (int)sizeof(float2);
    static_assert(TP <= 32 || (R + 1) * FPB <= 15, "named barriers: FFT ids 1..FPB, sub-FFT ids FPB+1..(R+1) FPB");
    float2* base;
    int f;
    int r;
    int k;

    __device__ __forceinline__ FftRGroup(float2* smem_block, int group, int sub)
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
            asm volatile("bar.sync %0, %1;" ::"r"(1 + FPB + R * f + r), "n"(TP) : "memory");
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

constexpr float kH3 = 0.866025403784438646764f;   // sqrt(3)/2
constexpr float kC51 = 0.309016994374947424102f;  // cos(2 pi / 5)
constexpr float kC52 = -0.809016994374947424102f; // cos(4 pi / 5)
constexpr float kS51 = 0.951056516295153572116f;  // sin(2 pi / 5)
constexpr float kS52 = 0.587785252292473129169f;  // sin(4 pi / 5)
constexpr float kC71 = 0.623489801858733530525f;  // cos(2 pi / 7)
constexpr float kC72 = -0.222520933956314404289f; // cos(4 pi / 7)
constexpr float kC73 = -0.900968867902419126236f; // cos(6 pi / 7)
constexpr float kS71 = 0.781831482468029808708f;  // sin(2 pi / 7)
constexpr float kS72 = 0.974927912181823607018f;  // sin(4 pi / 7)
constexpr float kS73 = 0.433883739117558120475f;  // sin(6 pi / 7)

// cos and sin of 2 pi m / 7, m = 0..6
__host__ __device__ constexpr float cos7(int m) {
    return m == 0 ? 1.f : (m == 1 || m == 6) ? kC71 : (m == 2 || m == 5) ? kC72 : kC73;
}
__host__ __device__ constexpr float sin7(int m) {
    return m == 0 ? 0.f : m == 1 ? kS71 : m == 2 ? kS72 : m == 3 ? kS73 : m == 4 ? -kS73 : m == 5 ? -kS72 : -kS71;
}

// Component k2 of the forward DFT_R of x[0..R-1]: sum_n x[n] W_R^(n k2), W_R = exp(-2 pi i / R).
template <int R>
__device__ __forceinline__ float2 dftr_component(const float2 (&x)[R], int k2) {
    if constexpr (R == 3) {
        const float2 s = cadd(x[1], x[2]);
        if (k2 == 0) return cadd(x[0], s);
        const float2 d = csub(x[1], x[2]);
        const float2 m = make_float2(fmaf(-0.5f, s.x, x[0].x), fmaf(-0.5f, s.y, x[0].y));
        const float hs = k2 == 1 ? -kH3 : kH3;  // -i h d for k2 = 1, +i h d for k2 = 2
        return make_float2(fmaf(-hs, d.y, m.x), fmaf(hs, d.x, m.y));
    } else if constexpr (R == 7) {
        // pairs j = 1..3: x_j W^(jk) + x_(7-j) W^(-jk) = c (x_j + x_(7-j)) - i s (x_j - x_(7-j)),
        // (c, s) = (cos, sin)(2 pi (j k mod 7) / 7)
        const float2 s1 = cadd(x[1], x[6]), s2 = cadd(x[2], x[5]), s3 = cadd(x[3], x[4]);
        if (k2 == 0) return cadd(x[0], cadd(s1, cadd(s2, s3)));
        const float2 d1 = csub(x[1], x[6]), d2 = csub(x[2], x[5]), d3 = csub(x[3], x[4]);
        const int m1 = k2, m2 = (2 * k2) % 7, m3 = (3 * k2) % 7;
        const float c1 = cos7(m1), c2 = cos7(m2), c3 = cos7(m3);
        const float n1 = sin7(m1), n2 = sin7(m2), n3 = sin7(m3);
        const float2 m = make_float2(fmaf(c3, s3.x, fmaf(c2, s2.x, fmaf(c1, s1.x, x[0].x))),
                                     fmaf(c3, s3.y, fmaf(c2, s2.y, fmaf(c1, s1.y, x[0].y))));
        const float2 t = make_float2(fmaf(n3, d3.x, fmaf(n2, d2.x, n1 * d1.x)), fmaf(n3, d3.y, fmaf(n2, d2.y, n1 * d1.y)));
        return make_float2(m.x + t.y, m.y - t.x);   // m - i t
    } else {
        // X_k = x0 + ca (x1 + x4) + cb (x2 + x3) -+ i [sa (x1 - x4) + sb (x2 - x3)], with
        // (ca, cb, sa, sb) = (c1, c2, s1, s2) for k = 1, 4 and (c2, c1, s2, -s1) for k = 2, 3
        const float2 s1 = cadd(x[1], x[4]), s2 = cadd(x[2], x[3]);
        if (k2 == 0) return cadd(x[0], cadd(s1, s2));
        const float2 d1 = csub(x[1], x[4]), d2 = csub(x[2], x[3]);
        const bool outer = k2 == 1 || k2 == 4;
        const float ca = outer ? kC51 : kC52, cb = outer ? kC52 : kC51;
        const float sa = outer ? kS51 : kS52, sb = outer ? kS52 : -kS51;
        const float2 m = make_float2(fmaf(cb, s2.x, fmaf(ca, s1.x, x[0].x)), fmaf(cb, s2.y, fmaf(ca, s1.y, x[0].y)));
        const float2 t = make_float2(fmaf(sb, d2.x, sa * d1.x), fmaf(sb, d2.y, sa * d1.y));
        // forward: -i t for k = 1, 2; +i t for k = 3, 4
        return k2 <= 2 ? make_float2(m.x + t.y, m.y - t.x) : make_float2(m.x - t.y, m.y + t.x);
    }
}

// Forward input y_k2[n1] of thread (k2, .) from x[n1 + P n2], n2 < R.
template <int R, int P>
__device__ __forceinline__ float2 dif_input(const float2 (&x)[R], int n1, int k2, const float2* __restrict__ twr) {
    const float2 y = dftr_component<R>(x, k2);
    return k2 == 0 ? y : cmul(y, ld_tw(twr + n1 * k2));
}

// The radix-3 form of dif_input with its three inputs as scalars (the form the 1536-point
// fused column pass was tuned with; the array form cost that kernel a register).
template <int P>
__device__ __forceinline__ float2 dif_input3(float2 x0, float2 x1, float2 x2, int n1, int k2,
                                             const float2* __restrict__ tw3) {
    const float2 s = cadd(x1, x2);
    if (k2 == 0) return cadd(x0, s);
    const float2 d = csub(x1, x2);
    const float2 m = make_float2(fmaf(-0.5f, s.x, x0.x), fmaf(-0.5f, s.y, x0.y));
    const float hs = k2 == 1 ? -kH3 : kH3;  // -i h d for k2 = 1, +i h d for k2 = 2
    return cmul(make_float2(fmaf(-hs, d.y, m.x), fmaf(hs, d.x, m.y)), ld_tw(tw3 + n1 * k2));
}

// Inverse DFT_R of z[0..R-1] (W_R = exp(+2 pi i / R)); the outputs n2 < count are handed to
// out(n2, value) (the output pruning of the last pass).
template <int R, class Out>
__device__ __forceinline__ void idftr_head(const float2 (&z)[R], int count, Out out) {
    if constexpr (R == 3) {
        const float2 s = cadd(z[1], z[2]);
        out(0, cadd(z[0], s));
        if (count > 1) {
            const float2 d = csub(z[1], z[2]);
            const float2 m = make_float2(fmaf(-0.5f, s.x, z[0].x), fmaf(-0.5f, s.y, z[0].y));
            const float hx = kH3 * d.x, hy = kH3 * d.y;
            out(1, make_float2(m.x - hy, m.y + hx));
            if (count > 2) out(2, make_float2(m.x + hy, m.y - hx));
        }
    } else if constexpr (R == 7) {
        const float2 s1 = cadd(z[1], z[6]), s2 = cadd(z[2], z[5]), s3 = cadd(z[3], z[4]);
        out(0, cadd(z[0], cadd(s1, cadd(s2, s3))));
        const float2 d1 = csub(z[1], z[6]), d2 = csub(z[2], z[5]), d3 = csub(z[3], z[4]);
        // output n: z0 + sum_j c (z_j + z_(7-j)) + i s (z_j - z_(7-j)), (c, s) at j n mod 7
#pragma unroll
        for (int n = 1; n < 7; n++) {
            if (n < count) {
                const float c1 = cos7(n), c2 = cos7((2 * n) % 7), c3 = cos7((3 * n) % 7);
                const float n1 = sin7(n), n2 = sin7((2 * n) % 7), n3 = sin7((3 * n) % 7);
                const float2 m = make_float2(fmaf(c3, s3.x, fmaf(c2, s2.x, fmaf(c1, s1.x, z[0].x))),
                                             fmaf(c3, s3.y, fmaf(c2, s2.y, fmaf(c1, s1.y, z[0].y))));
                const float2 t = make_float2(fmaf(n3, d3.x, fmaf(n2, d2.x, n1 * d1.x)),
                                             fmaf(n3, d3.y, fmaf(n2, d2.y, n1 * d1.y)));
                out(n, make_float2(m.x - t.y, m.y + t.x));   // m + i t
            }
        }
    } else {
        const float2 s1 = cadd(z[1], z[4]), s2 = cadd(z[2], z[3]);
        out(0, cadd(z[0], cadd(s1, s2)));
        if (count > 1) {
            const float2 d1 = csub(z[1], z[4]), d2 = csub(z[2], z[3]);
            // k = 1, 4 use (c1, c2; s1, s2), k = 2, 3 use (c2, c1; s2, -s1); the inverse adds
            // +i t for k = 1, 2 and -i t for k = 3, 4
            const float2 ma = make_float2(fmaf(kC52, s2.x, fmaf(kC51, s1.x, z[0].x)),
                                          fmaf(kC52, s2.y, fmaf(kC51, s1.y, z[0].y)));
            const float2 ta = make_float2(fmaf(kS52, d2.x, kS51 * d1.x), fmaf(kS52, d2.y, kS51 * d1.y));
            const float2 mb = make_float2(fmaf(kC51, s2.x, fmaf(kC52, s1.x, z[0].x)),
                                          fmaf(kC51, s2.y, fmaf(kC52, s1.y, z[0].y)));
            const float2 tb = make_float2(fmaf(-kS51, d2.x, kS52 * d1.x), fmaf(-kS51, d2.y, kS52 * d1.y));
            out(1, make_float2(ma.x - ta.y, ma.y + ta.x));
            if (count > 2) out(2, make_float2(mb.x - tb.y, mb.y + tb.x));
            if (count > 3) out(3, make_float2(mb.x + tb.y, mb.y - tb.x));
            if (count > 4) out(4, make_float2(ma.x + ta.y, ma.y - ta.x));
        }
    }
}

// W^(n1 k2) for k2 = 0 .. R-1 from the one table value W^n1 (the other powers are products:
// fewer L1 wavefronts than R - 1 loads).
template <int R>
__device__ __forceinline__ void twiddle_powers(float2 (&w)[R], float2 w1) {
    w[0] = make_float2(1.f, 0.f);
    w[1] = w1;
    w[2] = cmul(w1, w1);
    if constexpr (R > 3) {
        w[3] = cmul(w[2], w1);
        w[4] = cmul(w[2], w[2]);
    }
    if constexpr (R > 5) {
        w[5] = cmul(w[4], w1);
        w[6] = cmul(w[3], w[3]);
    }
}

// Final radix-R pass of the inverse.  v: z_k2[n1] of thread (k2 = g.r, j), n1 = j + T' q.
// Writes them to region k2 of the next buffer, waits for the FFT's threads, then thread t
// produces x[n1 + P n2], n2 < R, for n1 = t + T i and hands each to store(n, value).
// Output pruning: only the outputs n < keep are formed (every output needs all R sub-FFT
// values, so the pruning is of this last combination only; keep = RP forms all).
// The cross-region reads here must be followed by a sync_fft() before any later write to the
// buffer (the batched kernel's next template begins with one).
template <int R, int P, class G, class Store>
__device__ __forceinline__ void dit_output(float2 (&v)[16], G& g, int j, int t, const float2* __restrict__ twr,
                                           Store store, int keep = R * P) {
    using S3 = FftRShape<R, P>;
    float2* buf = g.begin_own();
    {
        float2* s = buf + g.r * G::SUB;
#pragma unroll
        for (int q = 0; q < 16; q++) s[phys_idx<S3::TP>(j, q)] = v[q];
    }
    g.sync_fft();
    const int lim = keep < P ? keep : P;
#pragma unroll 2
    for (int i = 0; i < S3::ROUNDS; i++) {
        const int n1 = t + S3::T * i;
        if (n1 < lim) {
            const int p = phys(n1);
            if constexpr (R == 3) {
                const float2 a = buf[p];
                const float2 w1 = ld_tw(twr + n1), w2 = cmul(w1, w1);  // one load: W^2n1 = (W^n1)^2
                const float2 b = cmulc(buf[G::SUB + p], w1);
                const float2 c = cmulc(buf[2 * G::SUB + p], w2);
                // inverse DFT3 of (a, b, c), formed only where kept
                const float2 s = cadd(b, c);
                store(n1, cadd(a, s));
                if (n1 + P < keep) {
                    const float2 d = csub(b, c);
                    const float2 m = make_float2(fmaf(-0.5f, s.x, a.x), fmaf(-0.5f, s.y, a.y));
                    const float hx = kH3 * d.x, hy = kH3 * d.y;
                    store(n1 + P, make_float2(m.x - hy, m.y + hx));
                    if (n1 + 2 * P < keep) store(n1 + 2 * P, make_float2(m.x + hy, m.y - hx));
                }
            } else {
                float2 w[R];
                twiddle_powers<R>(w, ld_tw(twr + n1));
                float2 z[R];
                z[0] = buf[p];
#pragma unroll
                for (int k2 = 1; k2 < R; k2++) z[k2] = cmulc(buf[k2 * G::SUB + p], w[k2]);
                const int count = (keep - n1 + P - 1) / P;   // outputs n1 + P n2 < keep
                idftr_head<R>(z, count < R ? count : R, [&](int n2, float2 x) { store(n1 + P * n2, x); });
            }
        }
    }
}

// Forward in decimation-in-time form, for callers whose input ends well before P and whose
// output goes to shared memory anyway (the row R2C): thread (r, j) loads x[R m + r],
// m = j + T' q, so the R sub-FFTs share the data instead of each reading all of it;
// the radix-R step X[k1 + P k2] = sum_r W_R^(r k2) W_RP^(r k1) Y_r[k1] then runs through
// shared memory and leaves X in natural order at locR<R, P>(k).  Returns that buffer after
// a barrier of the FFT's threads.
template <int R, int P, class G>
__device__ __forceinline__ float2* forward_dit(float2 (&v)[16], G& g, int j, int t, const float2* __restrict__ tw,
                                               const float2* __restrict__ twr, int qnz) {
    using S3 = FftRShape<R, P>;
    BlockFft<P, false>::run(v, g, j, tw, qnz);
    float2* buf = g.begin_own();
    {
        float2* s = buf + g.r * G::SUB;
#pragma unroll
        for (int q = 0; q < 16; q++) s[phys_idx<S3::TP>(j, q)] = v[q];
    }
    g.sync_fft();
#pragma unroll 2
    for (int i = 0; i < S3::ROUNDS; i++) {
        const int k1 = t + S3::T * i;
        if (k1 < P) {
            const int p = phys(k1);
            float2 w[R];
            twiddle_powers<R>(w, ld_tw(twr + k1));
            float2 y[R];
            y[0] = buf[p];
#pragma unroll
            for (int r = 1; r < R; r++) y[r] = cmul(buf[r * G::SUB + p], w[r]);
            float2 out[R];
#pragma unroll
            for (int k2 = 0; k2 < R; k2++) out[k2] = dftr_component<R>(y, k2);
#pragma unroll
            for (int k2 = 0; k2 < R; k2++) buf[k2 * G::SUB + p] = out[k2];
        }
    }
    g.sync_fft();
    return buf;
}

// leading q slots of thread (r, j) that can be non-zero when x[R (j + T' q) + r] is
// loaded only below L
template <int R, int P>
__device__ __forceinline__ int leading_slots_dit(int L, int r, int j) {
    constexpr int TP = FftRShape<R, P>::TP;
    const int Lr = L > r ? (L - r + R - 1) / R : 0;  // count of m with R m + r < L
    if (Lr <= j) return 0;
    const int q = (Lr - j + TP - 1) / TP;
    return q > 16 ? 16 : q;
}

// number of leading q slots (n1 = j + T' q) that can be non-zero when only x[n], n < L,
// is loaded: n1 < min(L, P)
template <int P>
__device__ __forceinline__ int leading_slots_p(int L, int j) {
    constexpr int TP = P / 16;
    const int Ln = L < P ? L : P;
    if (Ln <= j) return 0;
    const int q = (Ln - j + TP - 1) / TP;
    return q > 16 ? 16 : q;
}

}  // namespace ffb
