// Pass kernels at the lengths N = RP (R = 3 or 5) of the reduced-size correlation and of the
// 2D plans beyond powers of two (sm_100a).
//
// Same argument structures, data layouts and outputs as the power-of-two kernels in
// kernels_2d.cuh / kernels_xcorr.cuh; only the FFT inside differs (length RP, fft3.cuh):
//   r2c3_rows_kernel   : row R2C, two real rows per complex FFT, transposed [kx][y] output
//   c2r3_rows_kernel   : row C2R from [kx][y], two rows per complex FFT, fused peak search
//   cols3_kernel       : column FFT (2D layout), forward / inverse / fused correlation, keep W
//   xcorr3_cols_kernel : batched fused column pass (TMA-staged image and template columns,
//                        forward, conj(T) * I, inverse), keep W
// Time-domain data are loaded and stored in natural order; the spectrum side is decimated
// by R (thread (k2, j) holds X[R (j + T' q) + k2]).  R = 3 or 5 (lengths 3 * 2^k, 5 * 2^k).
#pragma once

#include "fft3.cuh"
#include "kernels_xcorr.cuh"

namespace ffb {

// Resident threads per SM the register budget of the column passes (batched and single) is
// sized for: 480 (at most 136 registers; 128 used at 1536 points without spills), as 5 blocks
// of one 1536-point FFT (96 threads) each.  Small blocks beat 2 blocks of 2 FFTs (named
// barriers per FFT) on B200: 5.66 instead of 5.94 us per template at 1536 points in the
// batched pass, 1.41 instead of 1.58 at 768.  Budgets measured side by side at 1536 points
// (batched pass, us per template): 384 threads (156 registers, 4 blocks) 5.41-5.53, 480 (128
// registers, 5 blocks) 5.12, 576 (96 registers, a few spills in other instantiations) 5.15-5.16.
#ifndef FFB_XCORR3_SM_THREADS
#define FFB_XCORR3_SM_THREADS 480
#endif
constexpr int kXcorr3SmThreads = FFB_XCORR3_SM_THREADS;

// ---------------------------------------------------------------------------
// Row R2C (forward)
// ---------------------------------------------------------------------------
#ifndef FFB_ROWS3_MIN_BLOCKS
#define FFB_ROWS3_MIN_BLOCKS 2
#endif

template <int R, int P, class InT, int FPB>
__global__ void __launch_bounds__(FftRShape<R, P>::T * FPB, FFB_ROWS3_MIN_BLOCKS)
r2c3_rows_kernel(RowFwdArgs a) {
    using S3 = FftRShape<R, P>;
    constexpr int N = S3::N;
    constexpr int T = S3::T;
    constexpr int TP = S3::TP;
    extern __shared__ float2 smem[];
    using G = FftRGroup<R, P, FPB, false>;
    const int f = threadIdx.x / T;
    const int t = threadIdx.x - f * T;
    const int k2 = t / TP;
    const int j = t - k2 * TP;
    G g(smem, f, k2);
    // batch entries in reverse order: the fused column pass that follows starts with entry 0,
    // whose rows are then the last written and still in L2 (measured on B200 with the C2R's
    // reversal: 9.76 instead of 9.79 us per template at 1536^2, 2.91 instead of 2.96 at 768^2)
    const int gb = gridDim.y - 1 - blockIdx.y;
    const int n_rows = a.rows_g[gb] > 0 ? a.rows_g[gb] : a.n_rows;
    const int L = a.L_g[gb] > 0 ? a.L_g[gb] : a.L;
    const long long in_pitch = a.pitch_g[gb] > 0 ? a.pitch_g[gb] : a.in_pitch;
    const int ra = 2 * (blockIdx.x * FPB + f);
    const bool has_a = ra < n_rows, has_b = ra + 1 < n_rows;
    const InT* in_g = static_cast<const InT*>(a.in[gb]);
    const InT* pa = in_g + input_row(ra, a.rows_y, a.rows_z) * in_pitch;
    const InT* pb = in_g + input_row(ra + 1, a.rows_y, a.rows_z) * in_pitch;
    float2* const out_g = a.out + (long long)gb * a.out_batch_stride;
    // two real rows as one complex sequence z[n] = a[n] + i b[n]; thread (r, j) holds
    // z[R (j + T' q) + r] (decimation in time: the sub-FFTs share the row's samples)
    float2 v[16];
#pragma unroll
    for (int q = 0; q < 16; q++) {
        const int n = R * (j + TP * q) + k2;
        float xa = 0.f, xb = 0.f;
        if (n < L) {
            if (has_a) xa = ld_real<InT>(pa + n);
            if (has_b) xb = ld_real<InT>(pb + n);
        }
        v[q] = make_float2(xa * a.scale, xb * a.scale);
    }
    forward_dit<R, P>(v, g, j, t, a.tw, a.tw3, leading_slots_dit<R, P>(L, k2, j));

    // Split Z = A + iB into the two real-row spectra (every FFT's buffer is read by the
    // whole block): A[k] = (Z[k] + conj Z[N-k]) / 2, B[k] = -i (Z[k] - conj Z[N-k]) / 2.
    __syncthreads();
    // item it of this thread: spectrum index k = k0 + T it of FFT ff0
    constexpr int kItemsPerThread = (FPB * (N / 2 + 1) + T * FPB - 1) / (T * FPB);
    const int ff0 = threadIdx.x % FPB;
    const int k0 = threadIdx.x / FPB;
    const float2* sf = smem + ff0 * G::STRIDE;
    const int rr0 = 2 * (blockIdx.x * FPB + ff0);
    const bool two = rr0 + 1 < n_rows, one = rr0 < n_rows;
    float2* o = out_g + (long long)k0 * a.out_pitch + rr0;
    const long long step = (long long)T * a.out_pitch;
#pragma unroll
    for (int it = 0; it < kItemsPerThread; it++, o += step) {
        const int k = k0 + T * it;
        if (k >= a.kmax) continue;
        const float2 z1 = sf[locR<R, P>(k)];
        const float2 z2 = sf[locR<R, P>(k == 0 ? 0 : N - k)];
        const float2 A = make_float2(0.5f * (z1.x + z2.x), 0.5f * (z1.y - z2.y));
        const float2 B = make_float2(0.5f * (z1.y + z2.y), 0.5f * (z2.x - z1.x));
        if (two) {
            *reinterpret_cast<float4*>(o) = make_float4(A.x, A.y, B.x, B.y);
        } else if (one) {
            *o = A;
        }
    }
}

// ---------------------------------------------------------------------------
// Row C2R (inverse), optional fused peak search
// ---------------------------------------------------------------------------
// The C2R gathers its input from L2/HBM with all of a thread's loads in flight at once, so it
// gains from a third resident block per SM (56 registers; measured on B200 at 1536 points:
// 4.2 instead of 4.6 us per template); the R2C does not, and keeps two.  Measured again with
// the 1536-point step (us per template): R2C at 3 blocks (56 registers, 48 bytes spilled)
// 2.086 against 2.093 at 2, within noise; C2R at 4 blocks (40 registers, 104 bytes spilled)
// 3.96 against 2.81 at 3.
#ifndef FFB_C2R3_MIN_BLOCKS
#define FFB_C2R3_MIN_BLOCKS 3
#endif

// PLAIN: windows written at origin 0, no peak search, no projection (the epilogue is then
// only the bounds check and the stores).
template <int R, int P, class OutT, int FPB, bool PLAIN>
__global__ void __launch_bounds__(FftRShape<R, P>::T * FPB, FFB_C2R3_MIN_BLOCKS)
c2r3_rows_kernel(RowInvArgs a) {
    using S3 = FftRShape<R, P>;
    constexpr int N = S3::N;
    constexpr int T = S3::T;
    constexpr int TP = S3::TP;
    constexpr int H = N / 2;
    extern __shared__ float2 smem[];
    using G = FftRGroup<R, P, FPB, false, S3::SUB_C2R, S3::C2R_FFT_EXTRA>;
    // Z[k] of FFT ff goes to region k % R at phys(k / R) (decimated by R, so that sub-FFT k2
    // finds its inputs Z[3 m + k2] contiguous in its own region)
    const int f = threadIdx.x / T;
    const int t = threadIdx.x - f * T;
    const int k2 = t / TP;
    const int j = t - k2 * TP;
    G g(smem, f, k2);
    // batch entries in reverse order: the fused column pass wrote the last entries last, so
    // theirs are the columns still in L2
    const int gb = gridDim.y - 1 - blockIdx.y;
    // Gather rows (2 per FFT) and build Z[k] = A[k] + i B[k] over the full circle from the
    // half spectra; the imaginary parts of the k = 0 and k = N/2 bins are dropped.
    // Item it of this thread is spectrum index k = k0 + T it of FFT ff0 (the block's item
    // stride T FPB is a multiple of FPB): one pointer, advanced by T rows per item.
    constexpr int kItemsPerThread = (FPB * (H + 1) + T * FPB - 1) / (T * FPB);
    const int ff0 = threadIdx.x % FPB;
    const int k0 = threadIdx.x / FPB;
    float4 ld[kItemsPerThread];
    {
        const int rr0 = 2 * (blockIdx.x * FPB + ff0);
        const bool two = rr0 + 1 < a.n_rows, one = rr0 < a.n_rows;
        const float2* p = a.in + (long long)gb * a.in_batch_stride + (long long)k0 * a.in_pitch + rr0;
        const long long step = (long long)T * a.in_pitch;
#pragma unroll
        for (int it = 0; it < kItemsPerThread; it++, p += step) {
            ld[it] = make_float4(0.f, 0.f, 0.f, 0.f);
            if (k0 + T * it <= H) {
                if (two) {
                    ld[it] = *reinterpret_cast<const float4*>(p);
                } else if (one) {
                    const float2 x = *p;
                    ld[it] = make_float4(x.x, x.y, 0.f, 0.f);
                }
            }
        }
    }
    // k % R and (N - k) % R stay fixed over the items (T = R T') and k / R moves by T' per
    // item, so the divisions by R are done once.
    float2* const sf = smem + ff0 * G::STRIDE;
    const int kq0 = k0 / R, kr0 = k0 - R * (k0 / R);
    const int nq0 = (N - k0) / R, nr0 = (N - k0) - R * ((N - k0) / R);
    float2* const s_k = sf + kr0 * G::SUB;
    float2* const s_nk = sf + nr0 * G::SUB;
    static_assert((T * FPB) % FPB == 0 && T % R == 0, "item stride");
#pragma unroll
    for (int it = 0; it < kItemsPerThread; it++) {
        const int k = k0 + T * it;
        if (k <= H) {
            const float2 A = make_float2(ld[it].x, ld[it].y), B = make_float2(ld[it].z, ld[it].w);
            if (k == 0 || k == H) {
                s_k[phys(kq0 + TP * it)] = make_float2(A.x, B.x);
            } else {
                s_k[phys(kq0 + TP * it)] = make_float2(A.x - B.y, A.y + B.x);
                s_nk[phys(nq0 - TP * it)] = make_float2(A.x + B.y, B.x - A.y);
            }
        }
    }
    __syncthreads();
    float2 v[16];
    {
        const float2* z = g.base + k2 * G::SUB;
#pragma unroll
        for (int q = 0; q < 16; q++) v[q] = z[phys(j + TP * q)];
    }
    // (each sub-FFT read only its own region, which its first exchange rewrites after its
    // own barrier)
    BlockFft<P, true>::run(v, g, j, a.tw, 16);
    const int ra = 2 * (blockIdx.x * FPB + f);
    OutT* oa = static_cast<OutT*>(a.out[gb]) + (long long)ra * a.out_pitch;
    OutT* ob = oa + a.out_pitch;
    const bool has_a = ra < a.n_rows, has_b = ra + 1 < a.n_rows;
    if constexpr (PLAIN) {
        dit_output<R, P>(v, g, j, t, a.tw3, [&](int n, float2 x) {
            if (n < a.W) {
                if (has_a) st_real<OutT>(oa + n, x.x * a.scale);
                if (has_b) st_real<OutT>(ob + n, x.y * a.scale);
            }
        }, a.W);
        return;
    } else {
        const bool write = !a.peaks_only;
        unsigned long long best = 0;
        const unsigned int tmpl = (unsigned)(a.mip_base + a.peak_slot[gb]);
        unsigned long long* ma = a.mip ? a.mip + (long long)ra * a.W : nullptr;
        dit_output<R, P>(v, g, j, t, a.tw3, [&](int n0, float2 x) {
            const int n = n0 - a.X0;
            if (n >= 0 && n < a.W) {
                const float va = x.x * a.scale, vb = x.y * a.scale;
                if (write) {
                    if (has_a) st_real<OutT>(oa + n, va);
                    if (has_b) st_real<OutT>(ob + n, vb);
                }
                if (ma) {
                    if (has_a) atomicMax(ma + n, peak_key(va, tmpl));
                    if (has_b) atomicMax(ma + a.W + n, peak_key(vb, tmpl));
                }
                if (a.peaks) {
                    if (has_a) {
                        const unsigned long long k = peak_key(va, (unsigned)(ra * a.W + n));
                        best = k > best ? k : best;
                    }
                    if (has_b) {
                        const unsigned long long k = peak_key(vb, (unsigned)((ra + 1) * a.W + n));
                        best = k > best ? k : best;
                    }
                }
            }
        }, a.X0 + a.W);
        if (a.peaks) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const unsigned long long other = __shfl_xor_sync(0xffffffffu, best, o);
                best = other > best ? other : best;
            }
            if ((threadIdx.x & 31) == 0 && best != 0) atomicMax(a.peaks + a.peak_slot[gb], best);
        }
    }
}

// ---------------------------------------------------------------------------
// Column passes over the 2D [kx][y] layout (modes as cols_kernel): FWD (the image
// preparation of the reduced-size correlation and FwdFFT at these lengths), INV and the
// single-template XCORR.  Output window [W0, W0 + W); the general 3D addressing of
// cols_kernel is not supported at these lengths (3D transforms are powers of two).
// ---------------------------------------------------------------------------
// OutC: storage type of the forward spectrum (FWD mode; the other modes write float2)
template <int R, int P, int MODE, class InC, class ImgC, int FPB, class OutC = float2>
__global__ void __launch_bounds__(FftRShape<R, P>::T * FPB, FftRShape<R, P>::T * FPB < kXcorr3SmThreads
                                                                ? kXcorr3SmThreads / (FftRShape<R, P>::T * FPB) : 1)
cols3_kernel(ColArgs a) {
    using S3 = FftRShape<R, P>;
    constexpr int T = S3::T;
    constexpr int TP = S3::TP;
    extern __shared__ float2 smem[];
    using G = FftRGroup<R, P, FPB, true>;
    const int f = threadIdx.x / T;
    const int t = threadIdx.x - f * T;
    const int k2 = t / TP;
    const int j = t - k2 * TP;
    G g(smem, f, k2);
    const int col = blockIdx.x * FPB + f;
    const bool valid = col < a.n_cols;
    const long long bz = blockIdx.y;
    const InC* pin = static_cast<const InC*>(a.in) + bz * a.in_batch_stride + (long long)col * a.in_stride;
    float2* pout = static_cast<float2*>(a.out) + bz * a.out_batch_stride + (long long)col * a.out_stride;
    float2 v[16];
    if constexpr (MODE == COL_INV) {
        // spectrum X[k], k < L, natural order in the column: thread (k2, j) takes X[3 m + k2]
#pragma unroll
        for (int q = 0; q < 16; q++) {
            const int k = R * (j + TP * q) + k2;
            const float2 x = (valid && k < a.L) ? ld_cplx<InC>(pin + k) : make_float2(0.f, 0.f);
            v[q] = (a.in_scale != 1.f) ? cscale(x, a.in_scale) : x;
        }
        BlockFft<P, true>::run(v, g, j, a.tw, 16);
    } else {
        auto ld = [&](int n) {
            const float2 x = (valid && n < a.L) ? ld_cplx<InC>(pin + n) : make_float2(0.f, 0.f);
            return (a.in_scale != 1.f) ? cscale(x, a.in_scale) : x;
        };
#pragma unroll
        for (int q = 0; q < 16; q++) {
            const int n1 = j + TP * q;
            float2 x[R];
#pragma unroll
            for (int n2 = 0; n2 < R; n2++) x[n2] = ld(n1 + P * n2);
            v[q] = dif_input<R, P>(x, n1, k2, a.tw3);
        }
        BlockFft<P, false>::run(v, g, j, a.tw, valid ? leading_slots_p<P>(a.L, j) : 0);
        if constexpr (MODE == COL_FWD) {
            // spectrum side: X[3 m + k2] straight from the registers
            if (valid) {
                OutC* po = static_cast<OutC*>(a.out) + bz * a.out_batch_stride + (long long)col * a.out_stride;
#pragma unroll
                for (int q = 0; q < 16; q++) {
                    const int n = R * (j + TP * q) + k2 - a.W0;
                    if (n >= 0 && n < a.W) st_cplx<OutC>(po + n, (a.out_scale != 1.f) ? cscale(v[q], a.out_scale) : v[q]);
                }
            }
            return;
        } else {
            if (a.intra_kind != 0) {
                const ImgC* pimg =
                    static_cast<const ImgC*>(a.img) + bz * a.img_batch_stride + (long long)col * a.img_stride;
                const float sc = a.intra_kind == 3 ? a.intra_scale : 1.f;
#pragma unroll
                for (int q = 0; q < 16; q++) {
                    float2 im = make_float2(0.f, 0.f);
                    if (valid) im = ld_cplx_stream<ImgC>(pimg + R * (j + TP * q) + k2);
                    const float2 pr = conj_mul(v[q], im);
                    v[q] = (sc != 1.f) ? cscale(pr, sc) : pr;
                }
            }
            BlockFft<P, true>::run(v, g, j, a.tw, 16);
        }
    }
    // INV and XCORR: radix-3 output pass, natural order
    const int W = valid ? a.W : 0;
    dit_output<R, P>(v, g, j, t, a.tw3, [&](int n0, float2 x) {
        const int n = n0 - a.W0;
        if (n >= 0 && n < W) pout[n] = (a.out_scale != 1.f) ? cscale(x, a.out_scale) : x;
    }, a.W0 + W);
}

// ---------------------------------------------------------------------------
// Batched fused correlation column pass (as xcorr_cols_kernel)
// ---------------------------------------------------------------------------
// One exchange buffer per FFT: the sub-FFT exchanges synchronise one warp (P = 512) or
// their own T' threads, so double buffering saves little, while the 26 KB it costs at
// P = 512 decides whether two blocks fit on an SM with 16 templates staged (measured on
// B200: 8.5 instead of 9.4 us per template for the 1536-point pass).
constexpr bool kXcorr3DB = false;

template <int R, int P, class ImgC, int FPB>
struct Xcorr3Smem {
    static constexpr int kImgBytes = R * P * (int)sizeof(ImgC);
    static constexpr int kXchBytes = FftRGroup<R, P, FPB, kXcorr3DB>::BYTES;
    static __host__ __device__ constexpr int t1_col_elems(int L) { return (L + 1) & ~1; }  // 16-byte multiple
    static __host__ __device__ constexpr int img_off() { return 0; }
    static __host__ __device__ constexpr int xch_off() { return (kImgBytes + 127) & ~127; }
    static __host__ __device__ constexpr int t1_off() { return xch_off() + kXchBytes; }
    static __host__ __device__ constexpr int bar_off(int L, int nb) {
        return (t1_off() + nb * t1_col_elems(L) * 8 + 15) & ~15;
    }
    static __host__ __device__ constexpr int total(int L, int nb) { return bar_off(L, nb) + 16; }
};


template <int R, int P, class ImgC, int FPB, bool MUL>
__global__ void __launch_bounds__(FftRShape<R, P>::T * FPB,
                                  FftRShape<R, P>::T * FPB < kXcorr3SmThreads ? kXcorr3SmThreads / (FftRShape<R, P>::T * FPB) : 1)
xcorr3_cols_kernel(XcorrColArgs a) {
    using S3 = FftRShape<R, P>;
    using SM = Xcorr3Smem<R, P, ImgC, FPB>;
    constexpr int T = S3::T;
    constexpr int TP = S3::TP;
    extern __shared__ __align__(128) unsigned char sm_raw[];
    const ImgC* img_s = reinterpret_cast<const ImgC*>(sm_raw + SM::img_off());
    float2* xch = reinterpret_cast<float2*>(sm_raw + SM::xch_off());
    float2* t1_s = reinterpret_cast<float2*>(sm_raw + SM::t1_off());
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm_raw + SM::bar_off(a.L, a.tpb));
    const int g0 = blockIdx.y * a.tpb;                              // first template of the block
    const int nb = min(a.tpb, a.n_batch - g0);                      // templates of the block

    const int col = blockIdx.x;
    const int f = threadIdx.x / T;
    const int t = threadIdx.x - f * T;
    const int k2 = t / TP;
    const int j = t - k2 * TP;
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
    FftRGroup<R, P, FPB, kXcorr3DB> grp(xch, f, k2);
#pragma unroll 1
    for (int it = 0; it < rounds; it++) {
        const int gl = it * FPB + f;                 // template within the block
        const bool live = gl < nb;
        const int g = g0 + (live ? gl : 0);          // template within the launch
        const int Lg = (live && a.L_g[g] > 0) ? a.L_g[g] : a.L;
        // keep the next template's loads out of this template's transforms
        asm volatile("" ::: "memory");
        // the previous round's output pass read all three regions of one buffer, which the
        // sub-FFT exchanges below rewrite
        if (it > 0) grp.sync_fft();
        float2 v[16];
        const float2* src = t1_s + (live ? gl : 0) * lcol;
        // Templates that end before P (the usual case: L + W - 1 <= 3P with W >= L) need
        // only x[n1]; this block-uniform branch skips the other two loads and the radix-3
        // sums (measured on B200 at 1536 points: 7.2 instead of 7.8 us per template).
        if (Lg <= P) {
            // y_k2[n1] = W_3P^(n1 k2) x[n1]
#pragma unroll
            for (int q = 0; q < 16; q++) {
                const int n1 = j + TP * q;
                const float2 x0 = (live && n1 < Lg) ? src[n1] : make_float2(0.f, 0.f);
                v[q] = k2 == 0 ? x0 : cmul(x0, ld_tw(a.tw3 + n1 * k2));
            }
        } else {
#pragma unroll
            for (int q = 0; q < 16; q++) {
                const int n1 = j + TP * q;
                if constexpr (R == 3) {
                    const float2 x0 = (live && n1 < Lg) ? src[n1] : make_float2(0.f, 0.f);
                    const float2 x1 = (live && n1 + P < Lg) ? src[n1 + P] : make_float2(0.f, 0.f);
                    const float2 x2 = (live && n1 + 2 * P < Lg) ? src[n1 + 2 * P] : make_float2(0.f, 0.f);
                    v[q] = dif_input3<P>(x0, x1, x2, n1, k2, a.tw3);
                } else {
                    float2 x[R];
#pragma unroll
                    for (int n2 = 0; n2 < R; n2++)
                        x[n2] = (live && n1 + P * n2 < Lg) ? src[n1 + P * n2] : make_float2(0.f, 0.f);
                    v[q] = dif_input<R, P>(x, n1, k2, a.tw3);
                }
            }
        }
        BlockFft<P, false>::run(v, grp, j, a.tw, live ? leading_slots_p<P>(Lg, j) : 0);
        if constexpr (MUL) {
            // CONJ_MUL (scale 1) skips the 32 multiplies of the scaling
            if (sc == 1.f) {
#pragma unroll
                for (int q = 0; q < 16; q++) v[q] = conj_mul(v[q], lds_cplx<ImgC>(img_s + R * (j + TP * q) + k2));
            } else {
#pragma unroll
                for (int q = 0; q < 16; q++) {
                    const float2 im = lds_cplx<ImgC>(img_s + R * (j + TP * q) + k2);
                    v[q] = cscale(conj_mul(v[q], im), sc);
                }
            }
        }
        BlockFft<P, true>::run(v, grp, j, a.tw, 16);
        float2* o = a.out + (long long)g * a.out_batch + (long long)col * a.out_pitch;
        const int W = live ? a.W : 0;
        dit_output<R, P>(v, grp, j, t, a.tw3, [&](int n, float2 x) {
            if (n < W) o[n] = x;
        }, a.W);
    }
}

}  // namespace ffb
