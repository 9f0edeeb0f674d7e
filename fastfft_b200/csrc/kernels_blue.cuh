// Transforms of any length N (2D real-input plans whose lengths are neither powers of two nor
// R * 2^k): Bluestein's chirp-z form of the N-point DFT on the power-of-two block FFT of length
// M >= 2N - 1.  With c_n = exp(-i pi n^2 / N), n k = (n^2 + k^2 - (k - n)^2) / 2 gives
//   X[k] = c_k sum_n (x_n c_n) conj(c_(k-n)),
// a circular convolution of a_n = x_n c_n (n < N, zero above) with b_m = conj(c_|m|) (|m| < N,
// placed at m and M - m), done as IFFT_M(FFT_M(a) FFT_M(b)); FFT_M(b) / M is a table per N.
// The inverse uses conj(DFT(conj X)).  Kernels (one FFT group of T = M / 16 threads per block,
// the same argument structures and layouts as the power-of-two passes in kernels_2d.cuh):
//   blue_r2c_rows_kernel : row R2C, two real rows per complex DFT, transposed [kx][y] output
//   blue_c2r_rows_kernel : row C2R from [kx][y], two rows per complex DFT, window [X0, X0 + W)
//   blue_cols_kernel     : column DFT, forward / inverse / correlation, window (the general
//                          column addressing of ColArgs: 2D and 3D passes)
//   blue_c2c_rows_fwd_kernel, blue_c2c_rows_inv_kernel : complex-input rows (C2C plans), one row
//                          per block, transposed [kx][y] output / gather over every kx
#pragma once

#include "kernels_2d.cuh"

namespace ffb {

struct BlueArgs {
    const float2* chirp;   // c_n, n < N
    const float2* filt;    // FFT_M(b)[m] / M, m < M
    int n;                 // N
};

// Length-N DFT (inverse: the unnormalised inverse) of x held as thread j's x[j + T q] (entries at
// or above N are ignored), on the M-point block FFT; on return thread j holds X[j + T q] for
// j + T q < N (zero above).  qnz: leading input slots that may be non-zero; keep: outputs below
// it are needed (the last pass of the inverse FFT_M forms only those where it can).
template <int M, class G>
__device__ __forceinline__ void bluestein_dft(float2 (&v)[16], G& g, int j, const float2* __restrict__ tw,
                                              const BlueArgs& b, bool inv, int qnz, int keep) {
    constexpr int T = M / 16;
#pragma unroll
    for (int q = 0; q < 16; q++) {
        const int n = j + T * q;
        float2 x = v[q];
        if (inv) x.y = -x.y;
        v[q] = n < b.n ? cmul(x, __ldg(b.chirp + n)) : make_float2(0.f, 0.f);
    }
    BlockFft<M, false>::run(v, g, j, tw, qnz);
#pragma unroll
    for (int q = 0; q < 16; q++) v[q] = cmul(v[q], __ldg(b.filt + j + T * q));
    BlockFft<M, true>::run(v, g, j, tw, 16, leading_slots<T>(keep, j));
#pragma unroll
    for (int q = 0; q < 16; q++) {
        const int k = j + T * q;
        float2 y = k < b.n ? cmul(v[q], __ldg(b.chirp + k)) : make_float2(0.f, 0.f);
        if (inv) y.y = -y.y;
        v[q] = y;
    }
}

template <int M, class InT>
__global__ void __launch_bounds__(M / 16)
blue_r2c_rows_kernel(RowFwdArgs a, BlueArgs b) {
    constexpr int T = M / 16;
    extern __shared__ float2 smem[];
    using G = FftGroup<M, 1, true>;
    const int j = threadIdx.x;
    G g(smem, 0);
    const int gb = blockIdx.y;
    const int N = b.n;
    const int n_rows = a.rows_g[gb] > 0 ? a.rows_g[gb] : a.n_rows;
    const int L = min(a.L_g[gb] > 0 ? a.L_g[gb] : a.L, N);
    const long long in_pitch = a.pitch_g[gb] > 0 ? a.pitch_g[gb] : a.in_pitch;
    const int ra = 2 * blockIdx.x;
    const bool has_a = ra < n_rows, has_b = ra + 1 < n_rows;
    const InT* in_g = static_cast<const InT*>(a.in[gb]);
    const InT* pa = in_g + input_row(ra, a.rows_y, a.rows_z) * in_pitch;
    const InT* pb = in_g + input_row(ra + 1, a.rows_y, a.rows_z) * in_pitch;
    float2 v[16];
#pragma unroll
    for (int q = 0; q < 16; q++) {
        const int n = j + T * q;
        float xa = 0.f, xb = 0.f;
        if (n < L) {
            if (has_a) xa = ld_real<InT>(pa + n);
            if (has_b) xb = ld_real<InT>(pb + n);
        }
        v[q] = make_float2(xa * a.scale, xb * a.scale);
    }
    bluestein_dft<M>(v, g, j, a.tw, b, false, leading_slots<T>(L, j), N);
    // split Z = A + iB into the two real rows' spectra through shared memory
    __syncthreads();
    float2* s = smem;
#pragma unroll
    for (int q = 0; q < 16; q++) s[phys(j + T * q)] = v[q];
    __syncthreads();
    float2* const out_g = a.out + (long long)gb * a.out_batch_stride;
    for (int k = j; k < a.kmax; k += T) {
        const float2 z1 = s[phys(k)];
        const float2 z2 = s[phys(k == 0 ? 0 : N - k)];
        const float2 A = make_float2(0.5f * (z1.x + z2.x), 0.5f * (z1.y - z2.y));
        const float2 B = make_float2(0.5f * (z1.y + z2.y), 0.5f * (z2.x - z1.x));
        float2* o = out_g + (long long)k * a.out_pitch + ra;
        if (has_b) {
            *reinterpret_cast<float4*>(o) = make_float4(A.x, A.y, B.x, B.y);
        } else if (has_a) {
            *o = A;
        }
    }
}

template <int M, class OutT>
__global__ void __launch_bounds__(M / 16)
blue_c2r_rows_kernel(RowInvArgs a, BlueArgs b) {
    constexpr int T = M / 16;
    extern __shared__ float2 smem[];
    using G = FftGroup<M, 1, true>;
    const int j = threadIdx.x;
    G g(smem, 0);
    const int gb = blockIdx.y;
    const int N = b.n;
    const int H = N / 2;
    const int ra = 2 * blockIdx.x;
    const bool has_a = ra < a.n_rows, has_b = ra + 1 < a.n_rows;
    // Z[k] = A[k] + i B[k] over the full circle from the two rows' half spectra (the imaginary
    // parts of the self-conjugate bins k = 0 and, for even N, k = N/2 are dropped)
    float2* s = smem;
    const float2* p = a.in + (long long)gb * a.in_batch_stride + ra;
    for (int k = j; k <= H; k += T) {
        float2 A = make_float2(0.f, 0.f), B = make_float2(0.f, 0.f);
        if (has_b) {
            const float4 t = *reinterpret_cast<const float4*>(p + (long long)k * a.in_pitch);
            A = make_float2(t.x, t.y);
            B = make_float2(t.z, t.w);
        } else if (has_a) {
            A = p[(long long)k * a.in_pitch];
        }
        if (k == 0 || 2 * k == N) {
            s[phys(k)] = make_float2(A.x, B.x);
        } else {
            s[phys(k)] = make_float2(A.x - B.y, A.y + B.x);
            s[phys(N - k)] = make_float2(A.x + B.y, B.x - A.y);
        }
    }
    __syncthreads();
    float2 v[16];
#pragma unroll
    for (int q = 0; q < 16; q++) {
        const int k = j + T * q;
        v[q] = k < N ? s[phys(k)] : make_float2(0.f, 0.f);
    }
    __syncthreads();   // the DFT's exchanges reuse this buffer
    bluestein_dft<M>(v, g, j, a.tw, b, true, 16, min(N, a.X0 + a.W));
    OutT* oa = static_cast<OutT*>(a.out[gb]) + (long long)ra * a.out_pitch;
    OutT* ob = oa + a.out_pitch;
#pragma unroll
    for (int q = 0; q < 16; q++) {
        const int n = j + T * q - a.X0;
        if (n >= 0 && n < a.W && j + T * q < N) {
            if (has_a) st_real<OutT>(oa + n, v[q].x * a.scale);
            if (has_b) st_real<OutT>(ob + n, v[q].y * a.scale);
        }
    }
}

// MODE: COL_FWD, COL_INV or COL_XCORR (forward, conj(T) x image, inverse).
template <int M, int MODE, class InC, class ImgC, class OutC>
__global__ void __launch_bounds__(M / 16)
blue_cols_kernel(ColArgs a, BlueArgs b) {
    constexpr int T = M / 16;
    extern __shared__ float2 smem[];
    using G = FftGroup<M, 1, true>;
    const int j = threadIdx.x;
    G g(smem, 0);
    const int col = blockIdx.x;
    const long long bz = blockIdx.y;
    const int N = b.n;
    const int L = min(a.L, N);
    const int in_div = a.in_div > 0 ? a.in_div : 1;
    const InC* pin = static_cast<const InC*>(a.in) + bz * a.in_batch_stride + (long long)(col / in_div) * a.in_stride +
                     (long long)(col % in_div) * a.in_stride2;
    float2 v[16];
#pragma unroll
    for (int q = 0; q < 16; q++) {
        const int n = j + T * q;
        const float2 x = n < L ? ld_cplx<InC>(pin + n) : make_float2(0.f, 0.f);
        v[q] = (a.in_scale != 1.f) ? cscale(x, a.in_scale) : x;
    }
    const int keep = min(N, a.W0 + a.W);
    if constexpr (MODE == COL_FWD) {
        bluestein_dft<M>(v, g, j, a.tw, b, false, leading_slots<T>(L, j), keep);
    } else if constexpr (MODE == COL_INV) {
        bluestein_dft<M>(v, g, j, a.tw, b, true, leading_slots<T>(L, j), keep);
    } else {
        bluestein_dft<M>(v, g, j, a.tw, b, false, leading_slots<T>(L, j), N);
        if (a.intra_kind != 0) {
            const ImgC* pimg = static_cast<const ImgC*>(a.img) + bz * a.img_batch_stride + (long long)col * a.img_stride;
            const float sc = a.intra_kind == 3 ? a.intra_scale : 1.f;
#pragma unroll
            for (int q = 0; q < 16; q++) {
                const int k = j + T * q;
                const float2 im = k < N ? ld_cplx<ImgC>(pimg + k) : make_float2(0.f, 0.f);
                const float2 p = conj_mul(v[q], im);
                v[q] = (sc != 1.f) ? cscale(p, sc) : p;
            }
        }
        bluestein_dft<M>(v, g, j, a.tw, b, true, 16, keep);
    }
    const int out_div = a.out_div > 0 ? a.out_div : 1;
    OutC* pout = static_cast<OutC*>(a.out) + bz * a.out_batch_stride + (long long)(col / out_div) * a.out_stride +
                 (long long)(col % out_div) * a.out_stride2;
    const long long es = a.out_elem_stride > 0 ? a.out_elem_stride : 1;
#pragma unroll
    for (int q = 0; q < 16; q++) {
        const int n = j + T * q - a.W0;
        if (n >= 0 && n < a.W && j + T * q < N) {
            const float2 x = (a.out_scale != 1.f) ? cscale(v[q], a.out_scale) : v[q];
            st_cplx<OutC>(pout + n * es, x);
        }
    }
}

// Complex-input row forward: row blockIdx.x of batch entry blockIdx.y, X[k] for k < kmax at
// out[k * out_pitch + row].
template <int M, class InC>
__global__ void __launch_bounds__(M / 16)
blue_c2c_rows_fwd_kernel(RowFwdArgs a, BlueArgs b) {
    constexpr int T = M / 16;
    extern __shared__ float2 smem[];
    using G = FftGroup<M, 1, true>;
    const int j = threadIdx.x;
    G g(smem, 0);
    const int gb = blockIdx.y;
    const int row = blockIdx.x;
    const int N = b.n;
    const int L = min(a.L, N);
    const InC* p = static_cast<const InC*>(a.in[gb]) + input_row(row, a.rows_y, a.rows_z) * a.in_pitch;
    float2 v[16];
#pragma unroll
    for (int q = 0; q < 16; q++) {
        const int n = j + T * q;
        const float2 x = n < L ? ld_cplx<InC>(p + n) : make_float2(0.f, 0.f);
        v[q] = (a.scale != 1.f) ? cscale(x, a.scale) : x;
    }
    bluestein_dft<M>(v, g, j, a.tw, b, false, leading_slots<T>(L, j), min(N, a.kmax));
    float2* const o = a.out + (long long)gb * a.out_batch_stride + row;
#pragma unroll
    for (int q = 0; q < 16; q++) {
        const int k = j + T * q;
        if (k < a.kmax && k < N) o[(long long)k * a.out_pitch] = v[q];
    }
}

// Complex-output row inverse: row blockIdx.x gathers X[k], k < N, from in[k * in_pitch + row]
// and keeps the outputs [X0, X0 + W).
template <int M, class OutC>
__global__ void __launch_bounds__(M / 16)
blue_c2c_rows_inv_kernel(RowInvArgs a, BlueArgs b) {
    constexpr int T = M / 16;
    extern __shared__ float2 smem[];
    using G = FftGroup<M, 1, true>;
    const int j = threadIdx.x;
    G g(smem, 0);
    const int gb = blockIdx.y;
    const int row = blockIdx.x;
    const int N = b.n;
    const float2* p = a.in + (long long)gb * a.in_batch_stride + row;
    float2 v[16];
#pragma unroll
    for (int q = 0; q < 16; q++) {
        const int k = j + T * q;
        v[q] = k < N ? p[(long long)k * a.in_pitch] : make_float2(0.f, 0.f);
    }
    bluestein_dft<M>(v, g, j, a.tw, b, true, 16, min(N, a.X0 + a.W));
    OutC* o = static_cast<OutC*>(a.out[gb]) + (long long)row * a.out_pitch;
#pragma unroll
    for (int q = 0; q < 16; q++) {
        const int n = j + T * q - a.X0;
        if (n >= 0 && n < a.W && j + T * q < N) st_cplx<OutC>(o + n, (a.scale != 1.f) ? cscale(v[q], a.scale) : v[q]);
    }
}

}  // namespace ffb
