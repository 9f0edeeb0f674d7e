// Tensor-core form of the fused 1536-point column pass (forward FFT of the zero-padded
// template column, conj(T) * I, inverse FFT, keep W outputs) on the sm_100a tensor cores
// (tcgen05.mma, FP32 accumulators in tensor memory).
//
// Algorithm: the 1536-point DFT as a four-step product 1536 = 48 x 32.  Forward, input
// n = 32 n1 + n2, output k = k1 + 48 k2:
//   F1  Y[n2][k1]  = sum_{n1 < 16} x[32 n1 + n2] W48^(n1 k1)         (templates end before 512)
//       Y'[n2][k1] = Y[n2][k1] W1536^(n2 k1)
//   F2  X[k1 + 48 k2] = sum_{n2} Y'[n2][k1] W32^(n2 k2)
// then Z = conj(X) I (times the scale of CONJ_MUL_THEN_SCALE; the batched path runs the
// correlation functors only), and the inverse with the same factorisation, output
// n = 32 n1 + n2 (n1 < 32 covers W <= 1024, n1 < 48 up to 1536):
//   I1  U[k1][n2]  = sum_{k2} Z[k1 + 48 k2] W32^(-n2 k2)
//   I2  y[32 n1 + n2] = sum_{k1} U[k1][n2] W1536^(-n2 k1) W48^(-n1 k1).
// Every DFT step is a real matrix product on the tensor cores: a complex row vector
// z = (re0, im0, re1, im1, ...) times the real form of a DFT matrix G (rows 2o + c of
// [[Re G, -Im G], [Im G, Re G]] interleaved).  The inverse steps reuse the forward matrices
// through conj(G^-1 z) = G conj(z): I1 is fed conj(Z) and yields conj(U); the I2 input is
// conj(U) W1536^(n2 k1) (the forward twiddle) and I2 yields conj(y).
//
// Precision: BF16 split products.  Every operand is split into two BF16 parts, v = hi + lo
// (hi rounded to nearest, lo the rounded remainder), and A B = Ah Bh + Ah Bl + Al Bh is
// accumulated in FP32 (the dropped Al Bl and the rounding of the low parts leave about 2^-17
// relative error per product; about 7e-6 relative L2 per correlated column in FP64 emulation).
//
// Block: 384 threads = three independent warpgroups sharing the DFT matrices in shared
// memory; each warpgroup takes work items (one image column x 4 templates) from the block's
// contiguous share of the items, so the three work on the same image column at a time.
// Thread r of a warpgroup owns row r of the M = 128 matrix tiles (tensor-memory lane r):
//   F1 rows (n2, t) = n2 + 32 t, K = 2 n1 + c (32), N = 96 (k1 < 48)
//   F2 rows (k1, t) = k1 + 48 t (192 rows: tile 0 rows 0..127, tile 1 128 rows from s1, see
//      below), K = 64, N = 64
//   I1 the same rows, A row-local (each thread writes its own row)
//   I2 rows (n2, t), K = 96 (k1 < 48), N = 64 (or 96 for windows above 1024)
// so F1 -> F2 and I1 -> I2 are transposes through shared memory, the twiddles and the
// correlation product are thread-local, and the tensor-memory loads give each thread its
// own row.  One thread per warpgroup issues the MMAs and commits them to the warpgroup's
// mbarrier; the wait is bounded (%globaltimer), and a timed-out warpgroup sets the error
// word and stops.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "fft_core.cuh"
#include "kernels_xcorr.cuh"
#include "tcgen05.cuh"

namespace ffb {
namespace tc1536 {

constexpr int kN = 1536;
constexpr int kTpi = 4;          // templates per work item
constexpr int kWgs = 3;          // warpgroups per block
constexpr int kThreads = 128 * kWgs;
constexpr int kMaxL = 512;       // F1 reads n1 < 16
// operand layouts (bytes): K-major, no swizzle; LBO 144 (one 16-byte pad per 8 K-chunks'
// row, so that a transposed write of 32 consecutive K pairs hits 32 distinct banks)
constexpr int kLbo = 144;
constexpr int kSbo1 = 4 * kLbo;            // F1: K 32
constexpr int kSbo2 = 8 * kLbo;            // F2 / I1: K 64
constexpr int kSbo4 = 12 * kLbo + 16;      // I2: K 96 (+16: rows 32 apart land on other banks)
constexpr int kHalf = 16 * kSbo4;          // hi part, then lo part at +kHalf
constexpr int kWgBytes = 2 * kHalf;
// DFT matrices in shared memory (and in the same byte image in global memory): real forms of
// W48 (96 x 96) and W32 (64 x 64), BF16 hi and lo parts; LBO 128, SBO one 8-row group.
constexpr int kB48Sbo = 12 * 128;
constexpr int kB32Sbo = 8 * 128;
constexpr int kB48Bytes = 96 * 96 * 2;
constexpr int kB32Bytes = 64 * 64 * 2;
constexpr int kB48h = 0, kB48l = kB48Bytes, kB32h = 2 * kB48Bytes, kB32l = 2 * kB48Bytes + kB32Bytes;
constexpr int kMatBytes = 2 * kB48Bytes + 2 * kB32Bytes;
constexpr int kTwOff = kMatBytes;          // W1536^m, m < 1536 (FP32 pairs), global memory only
constexpr int kConstBytes = kMatBytes + kN * 8;
constexpr int kMatOff = kWgs * kWgBytes;   // shared-memory offset of the matrices
constexpr int kBarOff = kMatOff + kMatBytes;
constexpr int kSmemBytes = kBarOff + 64;
static_assert(kSmemBytes <= 227 * 1024, "shared memory of the tensor-core column pass");
// the unused rows of F2 / I1 tile 1 (row groups 24..31 of the last warpgroup's lo part) stay
// inside the block's shared memory
static_assert(kMatOff - kWgBytes + kHalf + 31 * kSbo2 + 7 * kLbo + 128 <= kSmemBytes, "tile-1 reads");
static_assert(24 * kSbo2 <= kHalf && 16 * kSbo1 <= kHalf, "operand footprints");

template <class T> __device__ __forceinline__ float2 ldg_cplx(const T* p);
template <> __device__ __forceinline__ float2 ldg_cplx<float2>(const float2* p) { return __ldg(p); }
template <> __device__ __forceinline__ float2 ldg_cplx<__half2>(const __half2* p) { return __half22float2(__ldg(p)); }
template <> __device__ __forceinline__ float2 ldg_cplx<__nv_bfloat162>(const __nv_bfloat162* p) {
    return __bfloat1622float2(__ldg(p));
}

__device__ __forceinline__ void sts32(uint32_t a, uint32_t v) {
    asm volatile("st.shared.u32 [%0], %1;" ::"r"(a), "r"(v) : "memory");
}
__device__ __forceinline__ void sts128(uint32_t a, uint32_t x, uint32_t y, uint32_t z, uint32_t w) {
    asm volatile("st.shared.v4.u32 [%0], {%1, %2, %3, %4};" ::"r"(a), "r"(x), "r"(y), "r"(z), "r"(w) : "memory");
}

// Shared-memory descriptor fields other than the start address (LBO, SBO, version 1).
__device__ __forceinline__ uint64_t desc_bits(uint32_t lbo, uint32_t sbo) { return umma_desc(0, lbo, sbo); }

// Issue D = A B^T over KSTEPS K steps in three split terms (Ah Bh + Ah Bl + Al Bh) for tile 0
// of A at descriptor a0 and, with TILES = 2, tile 1 at a0 + a1 (descriptor units of 16 bytes),
// tile j into tensor-memory columns d + 64 j.  bh / bl: descriptors of the matrix parts.
template <int TILES, int KSTEPS>
__device__ __forceinline__ void issue_split_gemm(uint32_t d, uint64_t a0, uint32_t a1, uint64_t bh, uint64_t bl,
                                                 uint32_t idesc) {
#pragma unroll
    for (int j = 0; j < TILES; j++) {
        const uint64_t at = a0 + (j ? a1 : 0u);
#pragma unroll
        for (int s = 0; s < KSTEPS; s++) {
            const uint64_t ao = at + (uint64_t)(s * 2 * kLbo / 16), bo = (uint64_t)(s * 2 * 128 / 16);
            umma_bf16(d + 64 * j, ao, bh + bo, idesc, s > 0);
            umma_bf16(d + 64 * j, ao, bl + bo, idesc, 1);
            umma_bf16(d + 64 * j, ao + kHalf / 16, bh + bo, idesc, 1);
        }
    }
}

}  // namespace tc1536

// grid: persistent, at most one block per SM (the shared memory allows no second);
// consts: the byte image of the DFT matrices followed by the W1536 table.
template <class ImgC>
__global__ void __launch_bounds__(tc1536::kThreads, 1)
xcorr1536_tc_kernel(XcorrColArgs a, const uint8_t* __restrict__ consts, int n_items) {
    using namespace tc1536;
    extern __shared__ __align__(128) uint8_t sm[];
    const int wg = threadIdx.x >> 7;
    const int lt = threadIdx.x & 127;
    const int wq = lt >> 5;                 // warp within the warpgroup (= its tensor-memory lane quarter)
    const int lane = lt & 31;
    uint64_t* bars = reinterpret_cast<uint64_t*>(sm + kBarOff);
    int* flags = reinterpret_cast<int*>(sm + kBarOff + 32);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm + kBarOff + 48);

    // DFT matrices into shared memory (read by the tensor cores: async proxy)
    {
        const uint4* src = reinterpret_cast<const uint4*>(consts);
        uint4* dst = reinterpret_cast<uint4*>(sm + kMatOff);
        for (int i = threadIdx.x; i < kMatBytes / 16; i += kThreads) dst[i] = __ldg(src + i);
    }
    if (threadIdx.x < 32) tmem_alloc(tmem_slot, 512);
    if (threadIdx.x == 0) {
        for (int i = 0; i < kWgs; i++) mbar_init(bars + i, 1);
        fence_barrier_init();
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tm = *tmem_slot + (uint32_t)(wg * 128);   // this warpgroup's 128 columns
    const uint32_t tl = (uint32_t)(wq * 32) << 16;           // this warp's lane quarter

    const uint32_t s0 = smem_addr(sm);
    const uint32_t rg = s0 + wg * kWgBytes;                  // operand region (hi; lo at +kHalf)
    const float2* __restrict__ tw = reinterpret_cast<const float2*>(consts + kTwOff);
    uint64_t* bar = bars + wg;
    int* flag = flags + wg;
    const int bid = 1 + wg;                                  // named barrier of the warpgroup
    // F2 / I1 tile 1 covers rows s1 .. s1 + 127: its new rows 128..191 sit in lanes 0..63 for
    // s1 = 128 (rows 192..255 read other shared memory and are ignored) or in lanes 64..127
    // for s1 = 64 (rows 64..127 are computed twice); the warpgroups alternate, so the extra
    // rows fall on different warp schedulers
    const int s1 = wg == 1 ? 64 : 128;
    const bool t1_rows = (lt >= 128 - s1) && (lt < 192 - s1);    // warp-uniform
    // the thread that issues the MMAs: in a warp without tile-1 rows
    const int issuer = wg == 1 ? 0 : 32 * (2 + (wg >> 1));
    const bool n4_96 = a.W > 1024;
    const float sc = a.intra_kind == 3 ? a.intra_scale : 1.f;
    const int ngroups = (a.n_batch + kTpi - 1) / kTpi;
    const int per = (n_items + gridDim.x - 1) / gridDim.x;
    const int i_end = min(n_items, (int)(blockIdx.x + 1) * per);
    uint32_t phase = 0;

    // descriptors (start address in the low 14 bits, units of 16 bytes)
    const uint64_t dA1 = desc_bits(kLbo, kSbo1) + (rg >> 4);
    const uint64_t dA2 = desc_bits(kLbo, kSbo2) + (rg >> 4);
    const uint64_t dA4 = desc_bits(kLbo, kSbo4) + (rg >> 4);
    const uint32_t a2t1 = (uint32_t)((s1 / 8) * kSbo2 / 16);
    const uint64_t d48 = desc_bits(128, kB48Sbo), d32 = desc_bits(128, kB32Sbo);
    const uint64_t b48h = d48 + ((s0 + kMatOff + kB48h) >> 4), b48l = d48 + ((s0 + kMatOff + kB48l) >> 4);
    const uint64_t b32h = d32 + ((s0 + kMatOff + kB32h) >> 4), b32l = d32 + ((s0 + kMatOff + kB32l) >> 4);

    // all threads: shared-memory operands written and tensor-memory reads done
    auto pre_issue = [&]() {
        fence_async_smem();
        tc_fence_before();
        named_sync(bid, 128);
    };
    // the issuer waits for the warpgroup's MMAs (bounded, suspending); the outcome reaches
    // every thread of the warpgroup through the named barrier
    auto mma_done = [&]() -> bool {
        if (lt == issuer) {
            bool ok = mbar_wait_suspend(bar, phase);
            if (!ok) {
                if (a.err) atomicExch(a.err, kErrTimeout);
                mbar_wait_suspend(bar, phase);
            }
            *flag = ok ? 1 : 0;
        }
        named_sync(bid, 128);
        const bool ok = *reinterpret_cast<volatile int*>(flag) != 0;
        if (ok) mbar_wait(bar, phase);   // completed: acquire for this thread
        tc_fence_after();
        phase ^= 1;
        return ok;
    };

    // F1 input of an item: thread (n2 = lane, t = wq) holds x[32 n1 + n2], n1 < 16
    float2 xin[16];
    auto load_input = [&](int item) {
        const int col = item / ngroups;
        const int g = (item - col * ngroups) * kTpi + wq;
        const bool live = g < a.n_batch;
        const int Lg = live ? (a.L_g[g] > 0 ? a.L_g[g] : a.L) : 0;
        const float2* src = a.t1 + (long long)(live ? g : 0) * a.t1_batch + (long long)col * a.t1_pitch;
#pragma unroll
        for (int n1 = 0; n1 < 16; n1++) {
            const int n = 32 * n1 + lane;
            xin[n1] = n < Lg ? src[n] : make_float2(0.f, 0.f);
        }
    };
    const int it0 = blockIdx.x * per + wg;
    if (it0 < i_end) load_input(it0);

#pragma unroll 1
    for (int it = it0; it < i_end; it += kWgs) {
        const int col = it / ngroups;
        const int g0 = (it - col * ngroups) * kTpi;

        // ---- F1 input: rows n2 + 32 t, K = 2 n1 + c ----
        {
            uint32_t hi[16], lo[16];
#pragma unroll
            for (int n1 = 0; n1 < 16; n1++) split_bf16x2(xin[n1].x, xin[n1].y, hi[n1], lo[n1]);
            const uint32_t row = rg + (lt >> 3) * kSbo1 + (lt & 7) * 16;
#pragma unroll
            for (int c = 0; c < 4; c++) {
                sts128(row + c * kLbo, hi[4 * c], hi[4 * c + 1], hi[4 * c + 2], hi[4 * c + 3]);
                sts128(row + kHalf + c * kLbo, lo[4 * c], lo[4 * c + 1], lo[4 * c + 2], lo[4 * c + 3]);
            }
        }
        pre_issue();
        if (lt == issuer) {
            tc_fence_after();
            issue_split_gemm<1, 2>(tm, dA1, 0, b48h, b48l, umma_idesc_bf16(128, 96));
            umma_commit(bar);
        }
        if (!mma_done()) break;

        // ---- F1 -> F2: twiddle W1536^(n2 k1), transpose to rows k1 + 48 t, K = 2 n2 + c ----
        {
            const int n2 = lane;
            const float2 w1 = __ldg(tw + n2);
            const uint32_t base = rg + (n2 >> 2) * kLbo + (n2 & 3) * 4;
            float2 cur = make_float2(1.f, 0.f);
#pragma unroll 1
            for (int q = 0; q < 3; q++) {
                uint32_t v[32];
                tmem_ld32(tm + tl + 32 * q, v);
                tmem_wait(v);
#pragma unroll
                for (int i = 0; i < 16; i++) {
                    const int k1 = 16 * q + i;
                    cur = (i & 7) == 0 ? __ldg(tw + n2 * k1) : cmul(cur, w1);
                    const float2 y = cmul(make_float2(__uint_as_float(v[2 * i]), __uint_as_float(v[2 * i + 1])), cur);
                    uint32_t hi, lo;
                    split_bf16x2(y.x, y.y, hi, lo);
                    const int r = k1 + 48 * wq;
                    const uint32_t ad = base + (r >> 3) * kSbo2 + (r & 7) * 16;
                    sts32(ad, hi);
                    sts32(ad + kHalf, lo);
                }
            }
        }
        pre_issue();
        if (lt == issuer) {
            tc_fence_after();
            issue_split_gemm<2, 4>(tm, dA2, a2t1, b32h, b32l, umma_idesc_bf16(128, 64));
            umma_commit(bar);
        }
        // image values of this thread's tile-0 row, first half, while the MMAs run
        const ImgC* img = static_cast<const ImgC*>(a.img) + (long long)col * a.img_stride;
        float2 im[16];
#pragma unroll
        for (int i = 0; i < 16; i++) im[i] = ldg_cplx<ImgC>(img + lt % 48 + 48 * i);
        if (!mma_done()) break;

        // ---- F2 -> I1: Z = conj(X) I (x scale), I1 input conj(Z), row-local ----
#pragma unroll 1
        for (int j = 0; j < 2; j++) {
            if (j == 1 && !t1_rows) break;
            const int r = j ? s1 + lt : lt;
            const int k1 = r % 48;
            const uint32_t row = rg + (r >> 3) * kSbo2 + (r & 7) * 16;
            uint32_t v0[32], v1[32];
            tmem_ld32(tm + tl + 64 * j, v0);
            tmem_ld32(tm + tl + 64 * j + 32, v1);
#pragma unroll
            for (int h = 0; h < 2; h++) {
                if (j == 1 || h == 1) {
#pragma unroll
                    for (int i = 0; i < 16; i++) im[i] = ldg_cplx<ImgC>(img + k1 + 48 * (16 * h + i));
                }
                uint32_t(&v)[32] = h ? v1 : v0;
                tmem_wait(v);
                uint32_t hi[16], lo[16];
#pragma unroll
                for (int i = 0; i < 16; i++) {
                    float2 z = conj_mul(make_float2(__uint_as_float(v[2 * i]), __uint_as_float(v[2 * i + 1])), im[i]);
                    if (sc != 1.f) z = cscale(z, sc);
                    split_bf16x2(z.x, -z.y, hi[i], lo[i]);
                }
#pragma unroll
                for (int c = 0; c < 4; c++) {
                    sts128(row + (4 * h + c) * kLbo, hi[4 * c], hi[4 * c + 1], hi[4 * c + 2], hi[4 * c + 3]);
                    sts128(row + kHalf + (4 * h + c) * kLbo, lo[4 * c], lo[4 * c + 1], lo[4 * c + 2], lo[4 * c + 3]);
                }
            }
        }
        pre_issue();
        if (lt == issuer) {
            tc_fence_after();
            issue_split_gemm<2, 4>(tm, dA2, a2t1, b32h, b32l, umma_idesc_bf16(128, 64));
            umma_commit(bar);
        }
        if (!mma_done()) break;

        // ---- I1 -> I2: conj(U) W1536^(n2 k1), transpose to rows n2 + 32 t, K = 2 k1 + c ----
#pragma unroll 1
        for (int j = 0; j < 2; j++) {
            if (j == 1 && !t1_rows) break;
            const int r = j ? s1 + lt : lt;
            const int t = r / 48;
            const int k1 = r - 48 * t;
            const float2 v1 = __ldg(tw + k1);
            const uint32_t base = rg + (k1 >> 2) * kLbo + (k1 & 3) * 4;
            float2 cur = make_float2(1.f, 0.f);
            uint32_t va[32], vb[32];
            tmem_ld32(tm + tl + 64 * j, va);
            tmem_ld32(tm + tl + 64 * j + 32, vb);
#pragma unroll
            for (int h = 0; h < 2; h++) {
                uint32_t(&v)[32] = h ? vb : va;
                tmem_wait(v);
#pragma unroll
                for (int i = 0; i < 16; i++) {
                    const int n2 = 16 * h + i;
                    cur = (i & 7) == 0 ? __ldg(tw + n2 * k1) : cmul(cur, v1);
                    const float2 y = cmul(make_float2(__uint_as_float(v[2 * i]), __uint_as_float(v[2 * i + 1])), cur);
                    uint32_t hi, lo;
                    split_bf16x2(y.x, y.y, hi, lo);
                    const int r4 = n2 + 32 * t;
                    const uint32_t ad = base + (r4 >> 3) * kSbo4 + (r4 & 7) * 16;
                    sts32(ad, hi);
                    sts32(ad + kHalf, lo);
                }
            }
        }
        pre_issue();
        if (lt == issuer) {
            tc_fence_after();
            if (n4_96)
                issue_split_gemm<1, 6>(tm, dA4, 0, b48h, b48l, umma_idesc_bf16(128, 96));
            else
                issue_split_gemm<1, 6>(tm, dA4, 0, b48h, b48l, umma_idesc_bf16(128, 64));
            umma_commit(bar);
        }
        // the next item's template values, while the MMAs run
        if (it + kWgs < i_end) load_input(it + kWgs);
        if (!mma_done()) break;

        // ---- output: thread (n2 = lane, t = wq) holds conj y[32 n1 + n2] ----
        {
            const int g = g0 + wq;
            const bool live = g < a.n_batch;
            float2* o = a.out + (long long)(live ? g : 0) * a.out_batch + (long long)col * a.out_pitch;
#pragma unroll 1
            for (int h = 0; h < (n4_96 ? 3 : 2); h++) {
                uint32_t v[32];
                tmem_ld32(tm + tl + 32 * h, v);
                tmem_wait(v);
                if (live) {
#pragma unroll
                    for (int i = 0; i < 16; i++) {
                        const int n = 32 * (16 * h + i) + lane;
                        if (n < a.W) o[n] = make_float2(__uint_as_float(v[2 * i]), -__uint_as_float(v[2 * i + 1]));
                    }
                }
            }
        }
        // the next item's F1 MMAs overwrite these tensor-memory columns: its pre_issue
        // barrier follows every thread's loads (tcgen05.wait::ld) and fence
    }
    tc_fence_before();
    __syncthreads();
    if (threadIdx.x < 32) tmem_dealloc(*tmem_slot, 512);
}

}  // namespace ffb
