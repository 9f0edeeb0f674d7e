// Fused cross-correlation column pass, batched over templates (sm_100a).
//
// One block per spectrum column kx serves every template of the batch:
//   - the image-spectrum column (N values) and the template row-pass columns (L values
//     per template) are brought into shared memory by TMA bulk copies
//     (cp.async.bulk ... mbarrier::complete_tx) issued by one thread, so the image
//     column is read once per batch instead of once per template;
//   - each FFT group of the block then runs, per template, the zero-padded forward
//     column FFT, the conj(T) * I intra-op against the shared image column, and the
//     inverse FFT, and stores the first W outputs;
// Replaces block_fft_kernel_C2C_FWD_INCREASE_OP_INV_NONE (src/fastfft/FastFFT.cu:20-56),
// which reloads the image column per template and zero-pads explicitly.
//
// The mbarrier wait is bounded: if the copies have not landed after kWaitLimit polls,
// the block records kErrTimeout in *err and returns without touching the outputs.
#pragma once

#include "kernels_2d.cuh"
#include "tma.cuh"

namespace ffb {

struct XcorrColArgs {
    const float2* t1;          // template g, column c: t1 + g * t1_batch + c * t1_pitch (L valid values)
    long long t1_pitch;
    long long t1_batch;
    int L;
    const void* img;           // image column c: img + c * img_stride (ImgC elements)
    long long img_stride;
    float2* out;               // template g, column c: out + g * out_batch + c * out_pitch (W values)
    long long out_pitch;
    long long out_batch;
    int W;
    int n_cols;
    int n_batch;
    int intra_kind;            // 0 NOOP, 2 CONJ_MUL, 3 CONJ_MUL_THEN_SCALE
    float intra_scale;
    const float2* tw;
    const float2* tw3;         // N = 3P: radix-3 pass twiddles (set by the launcher)
    int* err;
    int L_g[kMaxBatch];        // per-template valid rows of uneven batches (0: use L)
    int tpb;                   // templates per block: block (c, y) serves templates
                               // [y tpb, min((y + 1) tpb, n_batch)) of column c (grid.y blocks)
    int tc;                    // 1: the tensor-core form of the pass where it has one (length 1536,
                               // kernels_tc.cuh); otherwise the FP32 pass runs
};

// Shared-memory plan of the kernel (bytes), shared by the host launcher.
template <int N, class ImgC, int FPB>
struct XcorrSmem {
    static constexpr int kImgBytes = N * (int)sizeof(ImgC);
    static constexpr int kXchBytes = FftGroup<N, FPB, true>::BYTES;
    static __host__ __device__ constexpr int t1_col_elems(int L) { return (L + 1) & ~1; }  // 16-byte multiple
    static __host__ __device__ constexpr int img_off() { return 0; }
    static __host__ __device__ constexpr int xch_off() { return (kImgBytes + 127) & ~127; }
    static __host__ __device__ constexpr int t1_off() { return xch_off() + kXchBytes; }
    static __host__ __device__ constexpr int bar_off(int L, int nb) {
        return (t1_off() + nb * t1_col_elems(L) * 8 + 15) & ~15;
    }
    static __host__ __device__ constexpr int total(int L, int nb) { return bar_off(L, nb) + 16; }
};

// Block size of the batched column pass: 128 threads (several FFTs per block below N = 2048),
// with registers budgeted for 512 resident threads per SM.  Smaller blocks than the former 256
// threads measured faster on B200: 2.06 instead of 2.18 us per template at 1024^2, 0.23
// instead of 0.32 at 256^2 (64 per launch).  Budgets of 640 (92 registers at 1024) and 768
// (80) measured on the uneven batch: 383,887-387,140 and 373,363-373,437 templates/s against
// 385,195-385,889 with 512.
constexpr int kXcorrBlockThreads = 128;
#ifndef FFB_XCORR_SM_THREADS
#define FFB_XCORR_SM_THREADS 512
#endif
constexpr int kXcorrSmThreads = FFB_XCORR_SM_THREADS;

// MUL: apply the conj-multiply intra-op (CONJ_MUL or CONJ_MUL_THEN_SCALE; the scale is
// 1 for CONJ_MUL, an exact multiplication); without it the kernel is a forward/inverse
// round trip (NOOP intra-op).  A compile-time choice keeps the transforms free of a
// run-time branch between them, which costs registers.
template <int N, class ImgC, int FPB, bool MUL>
__global__ void __launch_bounds__(FftShape<N>::T * FPB,
                                  FftShape<N>::T * FPB < kXcorrSmThreads ? kXcorrSmThreads / (FftShape<N>::T * FPB) : 1)
xcorr_cols_kernel(XcorrColArgs a) {
    using S = FftShape<N>;
    using SM = XcorrSmem<N, ImgC, FPB>;
    constexpr int T = S::T;
    extern __shared__ __align__(128) unsigned char sm_raw[];
    const ImgC* img_s = reinterpret_cast<const ImgC*>(sm_raw + SM::img_off());
    float2* xch = reinterpret_cast<float2*>(sm_raw + SM::xch_off());
    float2* t1_s = reinterpret_cast<float2*>(sm_raw + SM::t1_off());
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm_raw + SM::bar_off(a.L, a.tpb));
    const int g0 = blockIdx.y * a.tpb;                              // first template of the block
    const int nb = min(a.tpb, a.n_batch - g0);                      // templates of the block

    const int col = blockIdx.x;
    const int f = threadIdx.x / T;
    const int j = threadIdx.x - f * T;
    const int lcol = SM::t1_col_elems(a.L);

    __shared__ int ok_flag;
    uint32_t bytes = (uint32_t)SM::kImgBytes;
    for (int g = g0; g < g0 + nb; g++) bytes += (uint32_t)SM::t1_col_elems(a.L_g[g] > 0 ? a.L_g[g] : a.L) * 8;
    const bool staged = stage_block(bar, &ok_flag, bytes, a.err, [&]() {
        bulk_g2s(sm_raw + SM::img_off(), static_cast<const ImgC*>(a.img) + (long long)col * a.img_stride,
                 SM::kImgBytes, bar);
        for (int g = 0; g < nb; g++)
            bulk_g2s(t1_s + g * lcol, a.t1 + (g0 + g) * a.t1_batch + (long long)col * a.t1_pitch,
                     SM::t1_col_elems(a.L_g[g0 + g] > 0 ? a.L_g[g0 + g] : a.L) * 8, bar);
    });
    if (!staged) return;

    const float sc = a.intra_kind == 3 ? a.intra_scale : 1.f;
    const int rounds = (nb + FPB - 1) / FPB;
    FftGroup<N, FPB, true> grp(xch, f);
#pragma unroll 1
    for (int it = 0; it < rounds; it++) {
        const int gl = it * FPB + f;                 // template within the block
        const bool live = gl < nb;
        const int g = g0 + (live ? gl : 0);          // template within the launch
        const int Lg = (live && a.L_g[g] > 0) ? a.L_g[g] : a.L;
        // keep the next template's loads from being scheduled into this template's
        // transforms (that would hold twice the values live and spill)
        asm volatile("" ::: "memory");
        float2 v[16];
        const float2* src = t1_s + (live ? gl : 0) * lcol;
#pragma unroll
        for (int q = 0; q < 16; q++) {
            const int n = j + T * q;
            v[q] = (live && n < Lg) ? src[n] : make_float2(0.f, 0.f);
        }
        BlockFft<N, false>::run(v, grp, j, a.tw, live ? leading_slots<T>(Lg, j) : 0);
        if constexpr (MUL) {
            // CONJ_MUL (scale 1) skips the 32 multiplies of the scaling
            if (sc == 1.f) {
#pragma unroll
                for (int q = 0; q < 16; q++) v[q] = conj_mul(v[q], lds_cplx<ImgC>(img_s + j + T * q));
            } else {
#pragma unroll
                for (int q = 0; q < 16; q++) v[q] = cscale(conj_mul(v[q], lds_cplx<ImgC>(img_s + j + T * q)), sc);
            }
        }
        // output pruning: only X[j + T q] < W are kept
        BlockFft<N, true>::run(v, grp, j, a.tw, 16, leading_slots<T>(a.W, j));
        if (live) {
            float2* o = a.out + (long long)g * a.out_batch + (long long)col * a.out_pitch;
#pragma unroll
            for (int q = 0; q < 16; q++) {
                const int n = j + T * q;
                if (n < a.W) o[n] = v[q];
            }
        }
    }
}

}  // namespace ffb
