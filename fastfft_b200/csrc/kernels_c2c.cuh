// Row passes of the complex-input (C2C) transforms (sm_100a).
//
// The reference's FourierTransformer declares complex InputType (float2, __half2) but its
// complex paths are stubs ("Complex input images are not yet supported",
// src/fastfft/FastFFT.cu:369-391; 3D cross-correlation variants :722-793).  These kernels
// give complex-input plans the same structure as the real ones, with the same transposed
// spectrum layout [kx][ky] (ky contiguous), kx now over all N_x frequencies:
//   c2c_rows_fwd : one complex row per FFT, zero padding x >= L implicit, transposed
//                  output out[kx * out_pitch + row] for kx < kmax (forward decrease keeps
//                  the first kmax)
//   c2c_rows_inv : gathers in[kx * in_pitch + row] for every kx < N, inverse FFT, keeps
//                  x in [X0, X0 + W) of each row (complex output, pitch out_pitch)
// The column passes are the real path's (cols_kernel), over N_x columns instead of N_x/2+1.
// A block holds FPB rows; its transposed accesses walk the rows fastest, so each kx touches
// FPB consecutive complex values.
#pragma once

#include "kernels_2d.cuh"

namespace ffb {

template <int N, class InC, int FPB>
__global__ void __launch_bounds__(FftShape<N>::T * FPB, (FftShape<N>::T * FPB <= 256) ? 4 : 2)
c2c_rows_fwd_kernel(RowFwdArgs a) {
    using S = FftShape<N>;
    constexpr int T = S::T;
    extern __shared__ float2 smem[];
    using G = FftGroup<N, FPB, false>;
    const int f = threadIdx.x / T;
    const int j = threadIdx.x - f * T;
    G g(smem, f);
    const int gb = blockIdx.y;
    const int r0 = blockIdx.x * FPB;
    const int row = r0 + f;
    const bool has = row < a.n_rows;
    const InC* p = static_cast<const InC*>(a.in[gb]) + input_row(row, a.rows_y, a.rows_z) * a.in_pitch;
    float2 v[16];
#pragma unroll
    for (int q = 0; q < 16; q++) {
        const int n = j + T * q;
        const float2 x = (has && n < a.L) ? ld_cplx<InC>(p + n) : make_float2(0.f, 0.f);
        v[q] = (a.scale != 1.f) ? cscale(x, a.scale) : x;
    }
    BlockFft<N, false>::run(v, g, j, a.tw, has ? leading_slots<T>(a.L, j) : 0);
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 16; q++) g.base[phys(j + T * q)] = v[q];
    __syncthreads();
    // transposed store: item i of the block is (kx = i / FPB, row r0 + i % FPB)
    float2* const out_g = a.out + (long long)gb * a.out_batch_stride;
    const int rows_here = min(FPB, a.n_rows - r0);
    for (int i = threadIdx.x; i < a.kmax * FPB; i += T * FPB) {
        const int k = i / FPB, ff = i - k * FPB;
        if (ff < rows_here) out_g[(long long)k * a.out_pitch + r0 + ff] = smem[ff * G::STRIDE + phys(k)];
    }
}

template <int N, class OutC, int FPB>
__global__ void __launch_bounds__(FftShape<N>::T * FPB, (FftShape<N>::T * FPB <= 256) ? 4 : 2)
c2c_rows_inv_kernel(RowInvArgs a) {
    using S = FftShape<N>;
    constexpr int T = S::T;
    extern __shared__ float2 smem[];
    using G = FftGroup<N, FPB, false>;
    const int f = threadIdx.x / T;
    const int j = threadIdx.x - f * T;
    G g(smem, f);
    const int gb = blockIdx.y;
    const int r0 = blockIdx.x * FPB;
    const int rows_here = min(FPB, a.n_rows - r0);
    // gather: item i of the block is (kx = i / FPB, row r0 + i % FPB)
    const float2* in_g = a.in + (long long)gb * a.in_batch_stride;
    for (int i = threadIdx.x; i < N * FPB; i += T * FPB) {
        const int k = i / FPB, ff = i - k * FPB;
        smem[ff * G::STRIDE + phys(k)] = ff < rows_here ? in_g[(long long)k * a.in_pitch + r0 + ff] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    float2 v[16];
#pragma unroll
    for (int q = 0; q < 16; q++) v[q] = g.base[phys(j + T * q)];
    // output pruning: a window at the origin keeps X[j + T q] for q < qout only
    BlockFft<N, true>::run(v, g, j, a.tw, 16, a.X0 == 0 ? leading_slots<T>(a.W, j) : 16);
    const int row = r0 + f;
    if (row >= a.n_rows) return;
    OutC* o = static_cast<OutC*>(a.out[gb]) + (long long)row * a.out_pitch;
#pragma unroll
    for (int q = 0; q < 16; q++) {
        const int n = j + T * q - a.X0;
        if (n >= 0 && n < a.W) st_cplx<OutC>(o + n, (a.scale != 1.f) ? cscale(v[q], a.scale) : v[q]);
    }
}

}  // namespace ffb
