// Tensor-core form of the 512-point block FFT (one warp per FFT) for sm_100a: the two
// radix-16 passes run their 16-point DFTs as matrix products Y = F X on the tensor cores
// (F the 16x16 DFT matrix, X the 16 inputs of 32 butterflies), in BF16 split precision:
// F = Fh + Fl and X = Xh + Xl with every part in BF16, Y = Fh Xh + Fh Xl + Fl Xh accumulated
// in FP32 (the dropped Fl Xl term and the BF16 rounding of the low parts leave about 2^-17
// relative error per product; measured against FP64: 4e-6 relative L2 per 512-point FFT,
// 30x the FP32 form's).  Twiddles and the closing radix-2 pass stay in FP32 on the CUDA cores.
//
// Matrix products: mma.sync m16n8k16 (BF16 in, FP32 accumulate) with the complex product as
// four real ones, Yr = Fr Xr - Fi Xi and Yi = Fi Xr + Fr Xi, each in three split terms:
// 12 MMAs per 8 butterflies.  Fragment layout of m16n8k16 (lane = 4 g + t): A rows g and
// g + 8, columns 2t, 2t + 1 (+ 8); B rows (k) 2t, 2t + 1 (+ 8), column (n) g; D rows g and
// g + 8, columns 2t, 2t + 1; the lower half of a 32-bit register holds the lower index.
//
// This is the split-precision tensor-core option of the fused column pass; the FP32
// CUDA-core FFT (fft_core.cuh) stays the default: a 16-point DFT as a 32x32 real product in
// three split terms is about 20x the arithmetic of the radix-16 butterfly, and measured on
// B200 a 512-point round trip takes 2.3x as long this way (mma.sync; 198 instead of 88 ns
// per FFT per SM).
#pragma once

#include "fft_core.cuh"

namespace ffb {

__device__ __forceinline__ uint32_t bf16x2_pack(float lo, float hi) {
    uint32_t r;
    asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
    return r;
}

// (x0, x1) = hi + lo, each a BF16 pair
__device__ __forceinline__ void bf16x2_split(float x0, float x1, uint32_t& hi, uint32_t& lo) {
    hi = bf16x2_pack(x0, x1);
    const float h0 = __uint_as_float(hi << 16), h1 = __uint_as_float(hi & 0xffff0000u);
    lo = bf16x2_pack(x0 - h0, x1 - h1);
}

__device__ __forceinline__ void mma_m16n8k16_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// cos and sin of 2 pi m / 16
__device__ __forceinline__ float cos_16th(int m) {
    switch (m & 15) {
        case 0: return 1.f;
        case 1: return kC1;
        case 2: return kR2;
        case 3: return kS1;
        case 4: return 0.f;
        case 5: return -kS1;
        case 6: return -kR2;
        case 7: return -kC1;
        case 8: return -1.f;
        case 9: return -kC1;
        case 10: return -kR2;
        case 11: return -kS1;
        case 12: return 0.f;
        case 13: return kS1;
        case 14: return kR2;
        default: return kC1;
    }
}
__device__ __forceinline__ float sin_16th(int m) { return cos_16th(m + 12); }

// A fragments of the forward 16-point DFT matrix F[r][q] = exp(-2 pi i r q / 16) held by one
// lane: real and imaginary parts, each as hi and lo BF16 parts, and the negated imaginary
// parts (which are the imaginary parts of the inverse matrix conj F).
struct TcDft16 {
    uint32_t rh[4], rl[4], ih[4], il[4], nih[4], nil[4];

    __device__ __forceinline__ void init(int lane) {
        const int g = lane >> 2, t = lane & 3;
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const int r = g + 8 * (i & 1);
            const int q = 2 * t + 8 * (i >> 1);
            const float c0 = cos_16th(r * q), c1 = cos_16th(r * (q + 1));
            const float s0 = sin_16th(r * q), s1 = sin_16th(r * (q + 1));
            bf16x2_split(c0, c1, rh[i], rl[i]);
            bf16x2_split(-s0, -s1, ih[i], il[i]);
            nih[i] = ih[i] ^ 0x80008000u;
            nil[i] = il[i] ^ 0x80008000u;
        }
    }
};

// One radix-16 Stockham pass of the 512-point FFT held in s (input of butterfly b at
// s[phys(b + 32 q)], q < 16), with the pass twiddles W_{16 NS}^(q (b mod NS)) (tw: that pass's
// table, tw[q NS + t]) applied to the inputs; outputs back into s at the positions of stride
// NS.  Every lane of the warp takes part; reads finish before the first write.
template <bool INV, int NS>
__device__ __forceinline__ void tc_radix16_pass(float2* s, const TcDft16& F, const float2* __restrict__ tw,
                                                int lane) {
    const int g = lane >> 2, t = lane & 3;
    // the inverse transform multiplies by conj F: imaginary parts negated
    const uint32_t(&fih)[4] = INV ? F.nih : F.ih;
    const uint32_t(&fil)[4] = INV ? F.nil : F.il;
    const uint32_t(&nfih)[4] = INV ? F.ih : F.nih;
    const uint32_t(&nfil)[4] = INV ? F.il : F.nil;
    float dr[4][4], di[4][4];
#pragma unroll
    for (int tile = 0; tile < 4; tile++) {
        const int b = g + 8 * tile;
        float2 x[4];
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const int q = 2 * t + (e & 1) + 8 * (e >> 1);
            x[e] = s[phys(b + 32 * q)];
            if constexpr (NS > 1) {
                const float2 w = ld_tw(tw + q * NS + (b & (NS - 1)));
                x[e] = INV ? cmulc(x[e], w) : cmul(x[e], w);
            }
        }
        uint32_t xrh0, xrl0, xrh1, xrl1, xih0, xil0, xih1, xil1;
        bf16x2_split(x[0].x, x[1].x, xrh0, xrl0);
        bf16x2_split(x[2].x, x[3].x, xrh1, xrl1);
        bf16x2_split(x[0].y, x[1].y, xih0, xil0);
        bf16x2_split(x[2].y, x[3].y, xih1, xil1);
#pragma unroll
        for (int e = 0; e < 4; e++) dr[tile][e] = di[tile][e] = 0.f;
        mma_m16n8k16_bf16(dr[tile], F.rh, xrh0, xrh1);
        mma_m16n8k16_bf16(dr[tile], F.rh, xrl0, xrl1);
        mma_m16n8k16_bf16(dr[tile], F.rl, xrh0, xrh1);
        mma_m16n8k16_bf16(dr[tile], nfih, xih0, xih1);
        mma_m16n8k16_bf16(dr[tile], nfih, xil0, xil1);
        mma_m16n8k16_bf16(dr[tile], nfil, xih0, xih1);
        mma_m16n8k16_bf16(di[tile], fih, xrh0, xrh1);
        mma_m16n8k16_bf16(di[tile], fih, xrl0, xrl1);
        mma_m16n8k16_bf16(di[tile], fil, xrh0, xrh1);
        mma_m16n8k16_bf16(di[tile], F.rh, xih0, xih1);
        mma_m16n8k16_bf16(di[tile], F.rh, xil0, xil1);
        mma_m16n8k16_bf16(di[tile], F.rl, xih0, xih1);
    }
    __syncwarp();
#pragma unroll
    for (int tile = 0; tile < 4; tile++) {
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const int r = g + 8 * (e >> 1);
            const int b = 8 * tile + 2 * t + (e & 1);
            s[phys((b / NS) * 16 * NS + (b & (NS - 1)) + r * NS)] = make_float2(dr[tile][e], di[tile][e]);
        }
    }
    __syncwarp();
}

// 512-point FFT of one warp, same contract as BlockFft<512, INV>::run (lane j holds
// x[j + 32 q] in v[q] on entry and X[j + 32 q] on exit); s: the warp's exchange buffer
// (at least phys(511) + 1 float2), which no other warp touches during the call.
template <bool INV>
__device__ __forceinline__ void tc_fft512(float2 (&v)[16], float2* s, const TcDft16& F, const float2* __restrict__ tw,
                                          int j) {
    using S = FftShape<512>;
    __syncwarp();
#pragma unroll
    for (int q = 0; q < 16; q++) s[phys(j + 32 * q)] = v[q];
    __syncwarp();
    tc_radix16_pass<INV, 1>(s, F, tw, j);
    tc_radix16_pass<INV, 16>(s, F, tw + S::tw_pass_offset(1), j);
#pragma unroll
    for (int q = 0; q < 16; q++) v[q] = s[phys(j + 32 * q)];
    // closing radix-2 pass (FP32), as in BlockFft
    const float2 wj = ld_tw(tw + S::TW_REM + j);
#pragma unroll
    for (int m = 0; m < 8; m++) {
        const float2 x = mul_w16_k<INV>(v[m + 8], m);
        v[m + 8] = INV ? cmulc(x, wj) : cmul(x, wj);
        dft2<INV>(v[m], v[m + 8]);
    }
}

}  // namespace ffb
