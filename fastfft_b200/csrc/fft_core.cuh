// Block FFT core for sm_100a: radix-16 register butterflies, Stockham passes with
// shared-memory exchanges, FP64-generated twiddle tables.
//
// One length-N FFT (N = 2^m, 16 <= N <= 8192) is computed by T = N/16 threads.
// Thread j holds v[q] = x[j + T*q] (q = 0..15) on entry and X[j + T*q] on exit, so
// a column or row is read and written with unit stride across the threads.
// The passes are radix-16 passes with growing stride Ns = 1, 16, 256, ... followed by
// an optional closing radix-REM pass (REM = N / 16^k in {2,4,8}) of stride N/REM; between
// passes the values go through shared memory (one float2 of padding per 16 keeps the
// strided writes free of bank conflicts).  The first pass needs no twiddles and the
// closing pass only R-1 per butterfly, which it leaves in the thread's own slots
// (X[b + r N/R] with b = j + T m is slot m + r 16/R): the sizes with REM > 1 spend
// about a third less twiddle arithmetic than with the small pass first.
//
// This replaces the cuFFTDx block FFT that the reference calls through
// FFT().execute(thread_data, shared_mem, workspace) (e.g. src/fastfft/FastFFT.cu:42).
#pragma once

#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <stdint.h>

#ifndef FFB_PACKED_F32X2
#define FFB_PACKED_F32X2 0
#endif

namespace ffb {

constexpr int ilog2(int n) { return n <= 1 ? 0 : 1 + ilog2(n >> 1); }

// ---------------------------------------------------------------------------
// Complex arithmetic on float2.  FFB_PACKED_F32X2=1 maps the component-aligned adds
// to the sm_100 paired FP32 instructions; measured on B200 it made the column passes
// slower (register-pair moves), so the scalar form is the default.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 cadd(float2 a, float2 b) {
#if FFB_PACKED_F32X2
    return __fadd2_rn(a, b);
#else
    return make_float2(a.x + b.x, a.y + b.y);
#endif
}

__device__ __forceinline__ float2 csub(float2 a, float2 b) {
#if FFB_PACKED_F32X2
    return __ffma2_rn(b, make_float2(-1.f, -1.f), a);
#else
    return make_float2(a.x - b.x, a.y - b.y);
#endif
}

__device__ __forceinline__ float2 cscale(float2 a, float s) {
#if FFB_PACKED_F32X2
    return __fmul2_rn(a, make_float2(s, s));
#else
    return make_float2(a.x * s, a.y * s);
#endif
}

// a * w
__device__ __forceinline__ float2 cmul(float2 a, float2 w) {
    return make_float2(fmaf(a.x, w.x, -a.y * w.y), fmaf(a.x, w.y, a.y * w.x));
}

// a * conj(w)
__device__ __forceinline__ float2 cmulc(float2 a, float2 w) {
    return make_float2(fmaf(a.x, w.x, a.y * w.y), fmaf(a.y, w.x, -a.x * w.y));
}

// conj(a) * b : the CONJ_MUL intra-op of the reference, (ax*bx + ay*by, ax*by - ay*bx)
// (include/detail/functors.h:30-40).
__device__ __forceinline__ float2 conj_mul(float2 a, float2 b) {
    return make_float2(fmaf(a.x, b.x, a.y * b.y), fmaf(a.x, b.y, -a.y * b.x));
}

// Multiplication by the constant roots of unity W16^m = exp(-+2 pi i m / 16).
// Forward uses exp(-2 pi i m/16); inverse the conjugate.
constexpr float kC1 = 0.923879532511286756128f;  // cos(pi/8)
constexpr float kS1 = 0.382683432365089771728f;  // sin(pi/8)
constexpr float kR2 = 0.707106781186547524401f;  // sqrt(2)/2

template <bool INV, int M>
__device__ __forceinline__ float2 mul_w16(float2 a) {
    constexpr int m = M & 15;
    if constexpr (m == 0) {
        return a;
    } else if constexpr (m == 4) {
        // forward: -i ; inverse: +i
        return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
    } else if constexpr (m == 8) {
        return make_float2(-a.x, -a.y);
    } else if constexpr (m == 12) {
        return INV ? make_float2(a.y, -a.x) : make_float2(-a.y, a.x);
    } else if constexpr (m == 2) {
        // forward (1 - i)/sqrt2 ; inverse (1 + i)/sqrt2
        return INV ? make_float2(kR2 * (a.x - a.y), kR2 * (a.x + a.y))
                   : make_float2(kR2 * (a.x + a.y), kR2 * (a.y - a.x));
    } else if constexpr (m == 6) {
        // forward (-1 - i)/sqrt2 ; inverse (-1 + i)/sqrt2
        return INV ? make_float2(-kR2 * (a.x + a.y), kR2 * (a.x - a.y))
                   : make_float2(kR2 * (a.y - a.x), -kR2 * (a.x + a.y));
    } else if constexpr (m == 10) {
        return INV ? make_float2(kR2 * (a.y - a.x), -kR2 * (a.x + a.y))
                   : make_float2(-kR2 * (a.x + a.y), kR2 * (a.x - a.y));
    } else if constexpr (m == 14) {
        return INV ? make_float2(kR2 * (a.x + a.y), kR2 * (a.y - a.x))
                   : make_float2(kR2 * (a.x - a.y), kR2 * (a.x + a.y));
    } else {
        // general: angle m*pi/8
        constexpr float c = (m == 1 || m == 15) ? kC1 : (m == 3 || m == 13) ? kS1 : (m == 5 || m == 11) ? -kS1 : -kC1;
        constexpr float s = (m == 1 || m == 7) ? kS1 : (m == 3 || m == 5) ? kC1 : (m == 9 || m == 15) ? -kS1 : -kC1;
        // exp(i*m*pi/8) = (c, s); forward multiplies by (c, -s)
        return INV ? cmul(a, make_float2(c, s)) : cmul(a, make_float2(c, -s));
    }
}

// mul_w16 with the exponent known after unrolling
template <bool INV>
__device__ __forceinline__ float2 mul_w16_k(float2 a, int m) {
    switch (m & 15) {
        case 1: return mul_w16<INV, 1>(a);
        case 2: return mul_w16<INV, 2>(a);
        case 3: return mul_w16<INV, 3>(a);
        case 4: return mul_w16<INV, 4>(a);
        case 5: return mul_w16<INV, 5>(a);
        case 6: return mul_w16<INV, 6>(a);
        case 7: return mul_w16<INV, 7>(a);
        case 8: return mul_w16<INV, 8>(a);
        case 9: return mul_w16<INV, 9>(a);
        case 10: return mul_w16<INV, 10>(a);
        case 11: return mul_w16<INV, 11>(a);
        case 12: return mul_w16<INV, 12>(a);
        case 13: return mul_w16<INV, 13>(a);
        case 14: return mul_w16<INV, 14>(a);
        case 15: return mul_w16<INV, 15>(a);
        default: return a;
    }
}

// ---------------------------------------------------------------------------
// Small DFTs on registers (natural order in, natural order out)
// ---------------------------------------------------------------------------
template <bool INV>
__device__ __forceinline__ void dft2(float2& a0, float2& a1) {
    float2 t = csub(a0, a1);
    a0 = cadd(a0, a1);
    a1 = t;
}

template <bool INV>
__device__ __forceinline__ void dft4(float2& a0, float2& a1, float2& a2, float2& a3) {
    float2 s0 = cadd(a0, a2), e = csub(a0, a2);
    float2 s1 = cadd(a1, a3), d = csub(a1, a3);
    a0 = cadd(s0, s1);
    a2 = csub(s0, s1);
    if (!INV) {
        a1 = make_float2(e.x + d.y, e.y - d.x);
        a3 = make_float2(e.x - d.y, e.y + d.x);
    } else {
        a1 = make_float2(e.x - d.y, e.y + d.x);
        a3 = make_float2(e.x + d.y, e.y - d.x);
    }
}

// DFT8 over v[B + S*r], r = 0..7.
template <bool INV, int B, int S>
__device__ __forceinline__ void dft8(float2 (&v)[16]) {
    // n = n1 + 2 n2 ; first DFT4 over n2 for n1 = 0, 1
    float2 a[8];
#pragma unroll
    for (int r = 0; r < 8; r++) a[r] = v[B + S * r];
    dft4<INV>(a[0], a[2], a[4], a[6]);
    dft4<INV>(a[1], a[3], a[5], a[7]);
    // twiddles W8^(n1 k1) = W16^(2 n1 k1): n1 = 1, k1 = 1,2,3 at a[3], a[5], a[7]
    a[3] = mul_w16<INV, 2>(a[3]);
    a[5] = mul_w16<INV, 4>(a[5]);
    a[7] = mul_w16<INV, 6>(a[7]);
    // DFT2 over n1 for each k1: X[k1 + 4 k2]
    dft2<INV>(a[0], a[1]);
    dft2<INV>(a[2], a[3]);
    dft2<INV>(a[4], a[5]);
    dft2<INV>(a[6], a[7]);
    // a[2 k1 + k2] holds X[k1 + 4 k2]
#pragma unroll
    for (int k1 = 0; k1 < 4; k1++)
#pragma unroll
        for (int k2 = 0; k2 < 2; k2++) v[B + S * (k1 + 4 * k2)] = a[2 * k1 + k2];
}

// Twiddle stage inside the 4x4 decomposition of DFT16: a[n1 + 4 k1] *= W16^(n1 k1)
template <bool INV>
__device__ __forceinline__ void dft16_inner_twiddles(float2 (&a)[16]) {
    a[5] = mul_w16<INV, 1>(a[5]);
    a[9] = mul_w16<INV, 2>(a[9]);
    a[13] = mul_w16<INV, 3>(a[13]);
    a[6] = mul_w16<INV, 2>(a[6]);
    a[10] = mul_w16<INV, 4>(a[10]);
    a[14] = mul_w16<INV, 6>(a[14]);
    a[7] = mul_w16<INV, 3>(a[7]);
    a[11] = mul_w16<INV, 6>(a[11]);
    a[15] = mul_w16<INV, 9>(a[15]);
}

// Final DFT4 over n1 and the 4x4 transpose back to natural order.
template <bool INV>
__device__ __forceinline__ void dft16_outer(float2 (&a)[16], float2 (&v)[16]) {
    // a[n1 + 4 k1] after twiddles; DFT4 over n1 for each k1 -> X[k1 + 4 k2] at a[4 k1 + k2]
    dft4<INV>(a[0], a[1], a[2], a[3]);
    dft4<INV>(a[4], a[5], a[6], a[7]);
    dft4<INV>(a[8], a[9], a[10], a[11]);
    dft4<INV>(a[12], a[13], a[14], a[15]);
#pragma unroll
    for (int k1 = 0; k1 < 4; k1++)
#pragma unroll
        for (int k2 = 0; k2 < 4; k2++) v[k1 + 4 * k2] = a[4 * k1 + k2];
}

// Full DFT16 of v[0..15].
template <bool INV>
__device__ __forceinline__ void dft16(float2 (&v)[16]) {
    // n = n1 + 4 n2: DFT4 over n2 for each n1 -> A[n1][k1] stored at a[n1 + 4 k1]
    float2 a[16];
#pragma unroll
    for (int i = 0; i < 16; i++) a[i] = v[i];
    dft4<INV>(a[0], a[4], a[8], a[12]);
    dft4<INV>(a[1], a[5], a[9], a[13]);
    dft4<INV>(a[2], a[6], a[10], a[14]);
    dft4<INV>(a[3], a[7], a[11], a[15]);
    dft16_inner_twiddles<INV>(a);
    dft16_outer<INV>(a, v);
}

// DFT16 when only v[q], q < qnz, can be non-zero (forward size increase: the
// zero-padded tail of a column is never loaded or transformed).  Only the first
// stage (DFT4 over n2) is specialised, so the three variants share one register
// allocation for the twiddle and outer stages.
template <bool INV>
__device__ __forceinline__ void dft16_pruned(float2 (&v)[16], int qnz) {
    float2 a[16];
    if (qnz <= 4) {
        // only n2 = 0: the first-stage DFT4s are copies
#pragma unroll
        for (int n1 = 0; n1 < 4; n1++) {
            const float2 x = v[n1];
            a[n1] = x; a[n1 + 4] = x; a[n1 + 8] = x; a[n1 + 12] = x;
        }
    } else if (qnz <= 8) {
        // n2 in {0, 1}: DFT4 of (x0, x1, 0, 0) = (x0 + x1, x0 -+ i x1, x0 - x1, x0 +- i x1)
#pragma unroll
        for (int n1 = 0; n1 < 4; n1++) {
            const float2 x0 = v[n1], x1 = v[n1 + 4];
            a[n1] = cadd(x0, x1);
            a[n1 + 8] = csub(x0, x1);
            if (!INV) {
                a[n1 + 4] = make_float2(x0.x + x1.y, x0.y - x1.x);
                a[n1 + 12] = make_float2(x0.x - x1.y, x0.y + x1.x);
            } else {
                a[n1 + 4] = make_float2(x0.x - x1.y, x0.y + x1.x);
                a[n1 + 12] = make_float2(x0.x + x1.y, x0.y - x1.x);
            }
        }
    } else {
#pragma unroll
        for (int i = 0; i < 16; i++) a[i] = v[i];
        dft4<INV>(a[0], a[4], a[8], a[12]);
        dft4<INV>(a[1], a[5], a[9], a[13]);
        dft4<INV>(a[2], a[6], a[10], a[14]);
        dft4<INV>(a[3], a[7], a[11], a[15]);
    }
    dft16_inner_twiddles<INV>(a);
    dft16_outer<INV>(a, v);
}

// The first four outputs X[0..3] of DFT16 (the rest of v is left undefined): the last pass
// of an inverse whose retained window ends within the first quarter of every thread's slots
// (output pruning; e.g. a 4096-point inverse keeping 1024 outputs).  The first stage and the
// twiddles are needed by every output; the last stage keeps only its k2 = 0 sums.
template <bool INV>
__device__ __forceinline__ void dft16_head4(float2 (&v)[16]) {
    float2 a[16];
#pragma unroll
    for (int i = 0; i < 16; i++) a[i] = v[i];
    dft4<INV>(a[0], a[4], a[8], a[12]);
    dft4<INV>(a[1], a[5], a[9], a[13]);
    dft4<INV>(a[2], a[6], a[10], a[14]);
    dft4<INV>(a[3], a[7], a[11], a[15]);
    dft16_inner_twiddles<INV>(a);
#pragma unroll
    for (int k1 = 0; k1 < 4; k1++) v[k1] = cadd(cadd(a[4 * k1], a[4 * k1 + 2]), cadd(a[4 * k1 + 1], a[4 * k1 + 3]));
}

// ---------------------------------------------------------------------------
// Pass structure for one size
// ---------------------------------------------------------------------------
template <int N>
struct FftShape {
    static_assert(N >= 16 && N <= 8192 && (N & (N - 1)) == 0, "N must be a power of two in [16, 8192]");
    static constexpr int LOG = ilog2(N);
    static constexpr int T = N / 16;             // threads per FFT
    static constexpr int REM = 1 << (LOG & 3);   // radix of the optional first pass
    static constexpr int NP16 = LOG >> 2;        // number of radix-16 passes
    static constexpr int SMEM = N + N / 16;      // float2 per FFT exchange buffer
    // Stride between the buffers of consecutive FFT groups of a block: 4 float2 past a
    // multiple of 16, so that accesses that walk across groups (the row kernels' split
    // and gather phases) land in different banks.
    static constexpr int SMEM_PAD = ((SMEM + 15) / 16) * 16 + 4;
    // Twiddle table of one size:
    //   radix-16 pass p = 1 .. NP16-1 (stride ns = 16^p), 16 ns entries:
    //     tw[tw_pass_offset(p) + r ns + t] = W_{16 ns}^(r t)
    //   closing radix-REM pass, (REM-1) N/REM entries:
    //     tw[TW_REM + (r-1) N/REM + b] = W_N^(r b),  r = 1..REM-1, b < N/REM
    static constexpr int tw_pass_offset(int p) {
        int off = 0;
        int ns = 16;
        for (int i = 1; i < p; i++) {
            off += 16 * ns;
            ns *= 16;
        }
        return off;
    }
    static constexpr int TW_REM = tw_pass_offset(NP16);
    static constexpr int TW_SIZE = TW_REM + (REM > 1 ? (REM - 1) * (N / REM) : 0);
};

// Offsets of each size's twiddle table inside the one device-wide table.
constexpr int tw_size_of(int n) {
    int log = ilog2(n), rem = 1 << (log & 3), np16 = log >> 2, off = 0, ns = 16;
    for (int i = 1; i < np16; i++) {
        off += 16 * ns;
        ns *= 16;
    }
    return off + (rem > 1 ? (rem - 1) * (n / rem) : 0);
}
constexpr int tw_base(int n) {
    int off = 0;
    for (int m = 16; m < n; m *= 2) off += tw_size_of(m);
    return off;
}
constexpr int kMinN = 16;
constexpr int kMaxN = 8192;
constexpr int kTwTotal = tw_base(kMaxN) + tw_size_of(kMaxN);

__device__ __forceinline__ int phys(int i) { return i + (i >> 4); }
// Padded-index step of a stride: for i0 and a stride d that is a multiple of 16 (or d = 1 and
// i0 a multiple of 16, with q < 16), phys(i0 + q d) = phys(i0) + q phys_step(d) exactly; the
// exchanges use it so each access is one base plus a constant offset.
__host__ __device__ constexpr int phys_step(int d) { return d == 1 ? 1 : d + d / 16; }
// phys(j + D q) for a compile-time stride D: base plus constant offsets when D % 16 == 0
template <int D>
__device__ __forceinline__ int phys_idx(int j, int q) {
    if constexpr (D % 16 == 0) return phys(j) + q * phys_step(D);
    else return phys(j + D * q);
}

// Twiddle tables (layout in FftShape) are generated in FP64 (sincospi) and rounded to
// FP32 once; W_n^m = exp(-2 pi i m / n).

// Twiddle-table load that the compiler may not hoist out of loops: keeping the
// table values of every pass live across a loop over transforms would double the
// register demand of the fused kernels.
__device__ __forceinline__ float2 ld_tw(const float2* p) {
    float2 r;
    asm volatile("ld.global.nc.v2.f32 {%0, %1}, [%2];" : "=f"(r.x), "=f"(r.y) : "l"(p));
    return r;
}

// Radix-16 pass twiddles v[r] *= W^(r t), r = 1..15, from the four table values
// W^t, W^2t, W^4t, W^8t; the other eleven are products of at most three table values
// (for t = 0 all are exactly 1).  Four loads per pass instead of fifteen keeps the
// shared L1/shared-memory data path, the binding unit of these kernels, free for the
// exchanges.
template <bool INV>
__device__ __forceinline__ void twiddle_pass(float2 (&v)[16], float2 w1, float2 w2, float2 w4, float2 w8) {
#define FFB_TWMUL(r, w) v[r] = INV ? cmulc(v[r], (w)) : cmul(v[r], (w))
    const float2 w3 = cmul(w1, w2);
    FFB_TWMUL(1, w1);
    FFB_TWMUL(2, w2);
    FFB_TWMUL(3, w3);
    FFB_TWMUL(4, w4);
    const float2 w5 = cmul(w1, w4);
    FFB_TWMUL(5, w5);
    const float2 w6 = cmul(w2, w4);
    FFB_TWMUL(6, w6);
    const float2 w7 = cmul(w3, w4);
    FFB_TWMUL(7, w7);
    FFB_TWMUL(8, w8);
    FFB_TWMUL(9, cmul(w1, w8));
    FFB_TWMUL(10, cmul(w2, w8));
    FFB_TWMUL(11, cmul(w3, w8));
    FFB_TWMUL(12, cmul(w4, w8));
    FFB_TWMUL(13, cmul(w5, w8));
    FFB_TWMUL(14, cmul(w6, w8));
    FFB_TWMUL(15, cmul(w7, w8));
#undef FFB_TWMUL
}

// Exchange buffers and barrier of one FFT group (T = N/16 threads) inside a block of
// FPB groups.  Groups of at least one warp synchronise on their own named barrier
// (bar.sync 1 + f, T), so the groups of a block do not wait for each other; smaller
// groups fall back to __syncthreads().  With DB (double buffering) consecutive
// exchanges alternate between two buffers, which makes the write-after-read barrier
// unnecessary: a buffer is rewritten only after a barrier that every thread reaches
// after its last read of it.
template <int N, int FPB, bool DB>
struct FftGroup {
    using S = FftShape<N>;
    static constexpr int T = S::T;
    static constexpr int STRIDE = (DB ? 2 : 1) * S::SMEM_PAD;  // float2 per group
    static constexpr int BYTES = FPB * STRIDE * (int)sizeof(float2);  // per block
    float2* base;
    int f;
    int k;

    __device__ __forceinline__ FftGroup(float2* smem_block, int group) : base(smem_block + group * STRIDE), f(group), k(0) {}

    __device__ __forceinline__ void sync() const {
        if constexpr (T >= 32 && FPB > 1 && FPB <= 15) {
            asm volatile("bar.sync %0, %1;" ::"r"(f + 1), "n"(T) : "memory");
        } else {
            __syncthreads();
        }
    }

    // Buffer for the next exchange (waits for the previous readers when single-buffered).
    __device__ __forceinline__ float2* begin() {
        float2* p = base;
        if constexpr (DB) {
            p += (k & 1) * S::SMEM_PAD;
        } else {
            sync();
        }
        k++;
        return p;
    }
};

template <int N, bool INV>
struct BlockFft {
    using S = FftShape<N>;
    static constexpr int T = S::T;

    // Thread j of the FFT, v holds x[j + T q].  g: this FFT group's exchange buffers and
    // barrier.  tw: the twiddle table for size N.  qnz: number of leading q slots that
    // may be non-zero on input (16 = no pruning).  qout: number of leading output slots
    // X[j + T q], q < qout, the caller keeps (16 = all); the last pass computes only those
    // where the pass structure allows it (the others are left undefined).  Every thread of
    // the group must call this (and, for groups smaller than a warp, every thread of the
    // block).
    template <class G>
    __device__ __forceinline__ static void run(float2 (&v)[16], G& g, int j, const float2* __restrict__ tw, int qnz,
                                               int qout = 16) {
#pragma unroll
        for (int p = 0; p < S::NP16; p++) {
            const int ns = 1 << (4 * p);
            if (p > 0) {
                const float2* __restrict__ t = tw + S::tw_pass_offset(p) + (j & (ns - 1));
                twiddle_pass<INV>(v, ld_tw(t + ns), ld_tw(t + 2 * ns), ld_tw(t + 4 * ns), ld_tw(t + 8 * ns));
            }
            if (p == 0)
                dft16_pruned<INV>(v, qnz);
            else if (S::REM == 1 && p == S::NP16 - 1 && qout <= 4)
                dft16_head4<INV>(v);
            else
                dft16<INV>(v);
            if (p < S::NP16 - 1 || S::REM > 1) {
                float2* s = g.begin();
                const int base = (j / ns) * 16 * ns + (j & (ns - 1));
                // base is a multiple of 16 when ns = 1; ns and T are multiples of 16 otherwise
                float2* const sw = s + phys(base);
#pragma unroll
                for (int r = 0; r < 16; r++) sw[r * phys_step(ns)] = v[r];
                g.sync();
                if constexpr (T % 16 == 0) {
                    const float2* const sr = s + phys(j);
#pragma unroll
                    for (int q = 0; q < 16; q++) v[q] = sr[q * phys_step(T)];
                } else {
#pragma unroll
                    for (int q = 0; q < 16; q++) v[q] = s[phys(j + T * q)];
                }
            }
        }
        if constexpr (S::REM > 1) {
            // closing pass: butterfly b = j + T m over slots m + r M (values X[b + r N/R])
            constexpr int R = S::REM;
            constexpr int M = 16 / R;
            const float2* __restrict__ t = tw + S::TW_REM;
            // W_N^(r (j + T m)) = W_N^(r j) W_16^(r m): R-1 loads, the rest are constant turns
            // (fewer L1 wavefronts, the binding unit of the row passes; measured on B200:
            // C2R 2.97 instead of 3.10 us per template at 1536 points)
            float2 wj[R];
#pragma unroll
            for (int r = 1; r < R; r++) wj[r] = ld_tw(t + (r - 1) * (N / R) + j);
#pragma unroll
            for (int m = 0; m < M; m++) {
#pragma unroll
                for (int r = 1; r < R; r++) {
                    const float2 x = mul_w16_k<INV>(v[m + r * M], r * m);
                    v[m + r * M] = INV ? cmulc(x, wj[r]) : cmul(x, wj[r]);
                }
            }
            if (qout <= M)
                radix_head<R, M>(v);  // only the r = 0 outputs X[j + T m] are kept
            else
                radix_pass<R, M>(v);
        }
    }

    // The r = 0 outputs of the closing pass: v[m] = sum over r of v[m + r M]
    template <int R, int M>
    __device__ __forceinline__ static void radix_head(float2 (&v)[16]) {
#pragma unroll
        for (int m = 0; m < M; m++) {
#pragma unroll
            for (int r = 1; r < R; r++) v[m] = cadd(v[m], v[m + r * M]);
        }
    }

    // DFT_R over the slots m + r M (r = 0..R-1) for each m < M, natural order in and out
    template <int R, int M>
    __device__ __forceinline__ static void radix_pass(float2 (&v)[16]) {
        if constexpr (R == 2) {
#pragma unroll
            for (int m = 0; m < M; m++) dft2<INV>(v[m], v[m + M]);
        } else if constexpr (R == 4) {
#pragma unroll
            for (int m = 0; m < M; m++) dft4<INV>(v[m], v[m + M], v[m + 2 * M], v[m + 3 * M]);
        } else if constexpr (R == 8) {
            dft8<INV, 0, 2>(v);
            dft8<INV, 1, 2>(v);
        }
    }
};

}  // namespace ffb
