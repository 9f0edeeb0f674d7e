// Launchers for the length-RP pass kernels (kernels_fft3.cuh, R = 3, 5 or 7), templated on R;
// launch_fft3.cu, launch_fft5.cu and launch_fft7.cu each instantiate one radix (separate
// translation units so they compile in parallel) and launch_fft3.cu holds the public
// launchers, which pick the radix of N.  The caller's `tw` is replaced by the two tables these kernels read (sub-FFT
// size P, radix-R pass).
#pragma once

#include "kernels_fft3.cuh"
#include "launch_common.cuh"

namespace ffb {


// Runtime N = R P -> compile-time (R, P) for the radix R of this translation unit.
#define FFB_SIZE_R_SWITCH(R, n, FN, ...)                                        \
    switch ((n) / (R)) {                                                        \
        case 128: return FN<R, 128>(__VA_ARGS__);                               \
        case 256: return FN<R, 256>(__VA_ARGS__);                               \
        case 512: return FN<R, 512>(__VA_ARGS__);                               \
        case 1024:                                                              \
            if constexpr (1024 <= kMaxPR(R)) return FN<R, (R == 7 ? 512 : 1024)>(__VA_ARGS__); \
            return cudaErrorInvalidValue;                                       \
        case 2048:                                                              \
            if constexpr (2048 <= kMaxPR(R)) return FN<R, (R == 3 ? 2048 : 1024)>(__VA_ARGS__); \
            return cudaErrorInvalidValue;                                       \
        default: return cudaErrorInvalidValue;                                  \
    }

// FFTs per block: up to 384 threads for the row passes and 256 for the column passes, in
// whole warps (the peak search shuffles over full warps).  Row blocks of 384 threads hold a
// power-of-two number of FFTs (4 at 1536 points), whose buffers the gather and split phases
// interleave without bank conflicts (5 FFTs of 96 threads cost 47 % extra shared-memory
// wavefronts there); measured on B200: 15.6 instead of 15.8 us per template at 1536^2.
// (the most FFTs up to the target whose threads fill whole warps; if none does, the fewest
// above it that do, e.g. 4 FFTs of 40 threads at length 640)
constexpr int fpb3_for(int t, int target) {
    int f = target / t;
    if (f < 1) f = 1;
    while (f > 1 && (t * f) % 32 != 0) f--;
    while ((t * f) % 32 != 0) f++;
    return f;
}
template <int R, int P>
constexpr int row_fpb3() {
    return fpb3_for(FftRShape<R, P>::T, 384);
}
// column passes: blocks of about 96 threads (one FFT from P = 512 up), as the batched pass;
// measured on B200 in the image preparation of the 384^2 -> 4096^2 -> 1024^2 step: 647.7
// instead of 650.3 us per step with the 1536-point forward columns in 192-thread blocks
template <int R, int P>
constexpr int col_fpb3() {
    return fpb3_for(FftRShape<R, P>::T, 96);
}
// batched fused column pass: blocks of about 96 threads (one FFT from P = 512 up; 2 and 4
// FFTs of 48 and 24 threads below)
template <int R, int P>
constexpr int xcorr3_fpb() {
    return fpb3_for(FftRShape<R, P>::T, 96);
}
static_assert(FftRShape<3, 128>::T * row_fpb3<3, 128>() % 32 == 0 && FftRShape<3, 128>::T * col_fpb3<3, 128>() % 32 == 0,
              "warps");
static_assert(FftRShape<5, 128>::T * row_fpb3<5, 128>() % 32 == 0 && FftRShape<5, 128>::T * col_fpb3<5, 128>() % 32 == 0,
              "warps");
static_assert(FftRShape<5, 256>::T * xcorr3_fpb<5, 256>() % 32 == 0, "warps");

static cudaError_t tables3(int r, int p, const float2** tw, const float2** tw3) {
    cudaError_t e = twiddles_for(p, tw);
    if (e != cudaSuccess) return e;
    return twiddles_for(r * p, tw3);
}

// ---------------------------------------------------------------------------
template <int R, int P, class InT>
static cudaError_t r2c3_impl(const RowFwdArgs& a0, cudaStream_t st) {
    constexpr int FPB = row_fpb3<R, P>();
    constexpr int THREADS = FftRShape<R, P>::T * FPB;
    const size_t smem = (size_t)FftRGroup<R, P, FPB, false>::BYTES;
    RowFwdArgs a = a0;
    cudaError_t e = tables3(R, P, &a.tw, &a.tw3);
    if (e != cudaSuccess) return e;
    static std::atomic<unsigned long long> mask{0};
    auto fn = r2c3_rows_kernel<R, P, InT, FPB>;
    if ((e = ensure_smem_attr((const void*)fn, smem, &mask)) != cudaSuccess) return e;
    const int grid = (a.n_rows + 2 * FPB - 1) / (2 * FPB);
    if (grid == 0) return cudaSuccess;
    if (a.n_batch < 1 || a.n_batch > kMaxBatch) return cudaErrorInvalidValue;
    fn<<<dim3(grid, a.n_batch), THREADS, smem, st>>>(a);
    return cudaGetLastError();
}

template <int R, int P>
static cudaError_t r2c3_dispatch(int in_dtype, const RowFwdArgs& a, cudaStream_t st) {
    switch (in_dtype) {
        case 0: return r2c3_impl<R, P, float>(a, st);
        case 1: return r2c3_impl<R, P, __half>(a, st);
        case 2: return r2c3_impl<R, P, __nv_bfloat16>(a, st);
        default: return cudaErrorInvalidValue;
    }
}

template <int R>
cudaError_t launch_r2c_r(int n, int in_dtype, const RowFwdArgs& a, cudaStream_t st) {
    FFB_SIZE_R_SWITCH(R, n, r2c3_dispatch, in_dtype, a, st)
}

// ---------------------------------------------------------------------------
template <int R, int P, class OutT>
static cudaError_t c2r3_impl(const RowInvArgs& a0, cudaStream_t st) {
    constexpr int FPB = row_fpb3<R, P>();
    constexpr int THREADS = FftRShape<R, P>::T * FPB;
    const size_t smem = (size_t)FftRGroup<R, P, FPB, false, FftRShape<R, P>::SUB_C2R, FftRShape<R, P>::C2R_FFT_EXTRA>::BYTES;
    RowInvArgs a = a0;
    cudaError_t e = tables3(R, P, &a.tw, &a.tw3);
    if (e != cudaSuccess) return e;
    static std::atomic<unsigned long long> mask_plain{0}, mask_full{0};
    // plain windows (no peak search, no projection, origin 0): the short epilogue
    const bool plain = !a.peaks && !a.mip && !a.peaks_only && a.X0 == 0;
    auto fn = plain ? c2r3_rows_kernel<R, P, OutT, FPB, true> : c2r3_rows_kernel<R, P, OutT, FPB, false>;
    if ((e = ensure_smem_attr((const void*)fn, smem, plain ? &mask_plain : &mask_full)) != cudaSuccess) return e;
    const int grid = (a.n_rows + 2 * FPB - 1) / (2 * FPB);
    if (grid == 0) return cudaSuccess;
    if (a.n_batch < 1 || a.n_batch > kMaxBatch) return cudaErrorInvalidValue;
    fn<<<dim3(grid, a.n_batch), THREADS, smem, st>>>(a);
    return cudaGetLastError();
}

template <int R, int P>
static cudaError_t c2r3_dispatch(int out_dtype, const RowInvArgs& a, cudaStream_t st) {
    switch (out_dtype) {
        case 0: return c2r3_impl<R, P, float>(a, st);
        case 1: return c2r3_impl<R, P, __half>(a, st);
        case 2: return c2r3_impl<R, P, __nv_bfloat16>(a, st);
        default: return cudaErrorInvalidValue;
    }
}

template <int R>
cudaError_t launch_c2r_r(int n, int out_dtype, const RowInvArgs& a, cudaStream_t st) {
    FFB_SIZE_R_SWITCH(R, n, c2r3_dispatch, out_dtype, a, st)
}

// ---------------------------------------------------------------------------
template <int R, int P, int MODE, class InC, class ImgC, class OutC = float2>
static cudaError_t cols3_impl(const ColArgs& a0, cudaStream_t st) {
    // 2D layout only (3D transforms are powers of two)
    if (a0.in_div > 1 || a0.out_div > 1 || a0.out_elem_stride > 1) return cudaErrorInvalidValue;
    constexpr int FPB = col_fpb3<R, P>();
    constexpr int THREADS = FftRShape<R, P>::T * FPB;
    const size_t smem = (size_t)FftRGroup<R, P, FPB, true>::BYTES;
    ColArgs a = a0;
    cudaError_t e = tables3(R, P, &a.tw, &a.tw3);
    if (e != cudaSuccess) return e;
    static std::atomic<unsigned long long> mask{0};
    auto fn = cols3_kernel<R, P, MODE, InC, ImgC, FPB, OutC>;
    if ((e = ensure_smem_attr((const void*)fn, smem, &mask)) != cudaSuccess) return e;
    const int grid = (a.n_cols + FPB - 1) / FPB;
    if (grid == 0) return cudaSuccess;
    if (a.n_batch < 1 || a.n_batch > kMaxBatch) return cudaErrorInvalidValue;
    fn<<<dim3(grid, a.n_batch), THREADS, smem, st>>>(a);
    return cudaGetLastError();
}

template <int R, int P>
static cudaError_t cols3_fwd_dispatch(int out_dtype, const ColArgs& a, cudaStream_t st) {
    switch (out_dtype) {
        case 3: return cols3_impl<R, P, COL_FWD, float2, float2, float2>(a, st);
        case 4: return cols3_impl<R, P, COL_FWD, float2, float2, __half2>(a, st);
        case 5: return cols3_impl<R, P, COL_FWD, float2, float2, __nv_bfloat162>(a, st);
        default: return cudaErrorInvalidValue;
    }
}
template <int R, int P>
static cudaError_t cols3_inv_dispatch(int in_dtype, const ColArgs& a, cudaStream_t st) {
    switch (in_dtype) {
        case 3: return cols3_impl<R, P, COL_INV, float2, float2>(a, st);
        case 4: return cols3_impl<R, P, COL_INV, __half2, float2>(a, st);
        case 5: return cols3_impl<R, P, COL_INV, __nv_bfloat162, float2>(a, st);
        default: return cudaErrorInvalidValue;
    }
}
template <int R, int P>
static cudaError_t cols3_xcorr_dispatch(int img_dtype, const ColArgs& a, cudaStream_t st) {
    switch (img_dtype) {
        case 3: return cols3_impl<R, P, COL_XCORR, float2, float2>(a, st);
        case 4: return cols3_impl<R, P, COL_XCORR, float2, __half2>(a, st);
        case 5: return cols3_impl<R, P, COL_XCORR, float2, __nv_bfloat162>(a, st);
        default: return cudaErrorInvalidValue;
    }
}

template <int R>
cudaError_t launch_cols_fwd_r(int n, int out_dtype, const ColArgs& a, cudaStream_t st) {
    FFB_SIZE_R_SWITCH(R, n, cols3_fwd_dispatch, out_dtype, a, st)
}
template <int R>
cudaError_t launch_cols_inv_r(int n, int in_dtype, const ColArgs& a, cudaStream_t st) {
    FFB_SIZE_R_SWITCH(R, n, cols3_inv_dispatch, in_dtype, a, st)
}
template <int R>
cudaError_t launch_cols_xcorr_r(int n, int img_dtype, const ColArgs& a, cudaStream_t st) {
    FFB_SIZE_R_SWITCH(R, n, cols3_xcorr_dispatch, img_dtype, a, st)
}

// ---------------------------------------------------------------------------
// dynamic shared memory available to one block (227 KB, less a little static shared memory)
constexpr int kMaxDynSmem3 = 227 * 1024 - 1024;

template <int R, int P, class ImgC>
static cudaError_t xcorr3_impl(const XcorrColArgs& a0, cudaStream_t st) {
    constexpr int FPB = xcorr3_fpb<R, P>();
    using SM = Xcorr3Smem<R, P, ImgC, FPB>;
    if (a0.n_batch < 1 || a0.n_batch > kMaxBatch || a0.n_cols < 1) return cudaErrorInvalidValue;
    if (a0.tpb < 1 || a0.tpb > a0.n_batch) return cudaErrorInvalidValue;
    const int smem = SM::total(a0.L, a0.tpb);
    if (smem > kMaxDynSmem3) return cudaErrorInvalidValue;
    XcorrColArgs a = a0;
    cudaError_t e = tables3(R, P, &a.tw, &a.tw3);
    if (e != cudaSuccess) return e;
    static std::atomic<int> set_attr[2][64];
    const bool mul = a.intra_kind != 0;
    auto fn = mul ? xcorr3_cols_kernel<R, P, ImgC, FPB, true> : xcorr3_cols_kernel<R, P, ImgC, FPB, false>;
    if ((e = ensure_smem_at_least((const void*)fn, (size_t)smem, set_attr[mul])) != cudaSuccess) return e;
    fn<<<dim3(a.n_cols, (a.n_batch + a.tpb - 1) / a.tpb), FftRShape<R, P>::T * FPB, smem, st>>>(a);
    return cudaGetLastError();
}

template <int R, int P>
static cudaError_t xcorr3_dispatch(int img_dtype, const XcorrColArgs& a, cudaStream_t st) {
    switch (img_dtype) {
        case 3: return xcorr3_impl<R, P, float2>(a, st);
        case 4: return xcorr3_impl<R, P, __half2>(a, st);
        case 5: return xcorr3_impl<R, P, __nv_bfloat162>(a, st);
        default: return cudaErrorInvalidValue;
    }
}

template <int R>
cudaError_t launch_xcorr_r(int n, int img_dtype, const XcorrColArgs& a, cudaStream_t st) {
    FFB_SIZE_R_SWITCH(R, n, xcorr3_dispatch, img_dtype, a, st)
}

template <int R, int P>
static size_t xcorr3_smem_p(int img_dtype, int L, int n_batch) {
    constexpr int FPB = xcorr3_fpb<R, P>();
    if (img_dtype == 3) return (size_t)Xcorr3Smem<R, P, float2, FPB>::total(L, n_batch);
    return (size_t)Xcorr3Smem<R, P, __half2, FPB>::total(L, n_batch);
}

template <int R>
size_t xcorr_smem_r(int n, int img_dtype, int L, int n_batch) {
    switch (n / R) {
        case 128: return xcorr3_smem_p<R, 128>(img_dtype, L, n_batch);
        case 256: return xcorr3_smem_p<R, 256>(img_dtype, L, n_batch);
        case 512: return xcorr3_smem_p<R, 512>(img_dtype, L, n_batch);
        case 1024:
            if constexpr (1024 <= kMaxPR(R)) return xcorr3_smem_p<R, (R == 7 ? 512 : 1024)>(img_dtype, L, n_batch);
            return ~(size_t)0;
        case 2048:
            if constexpr (R == 3) return xcorr3_smem_p<R, 2048>(img_dtype, L, n_batch);
            return ~(size_t)0;
        default: return ~(size_t)0;
    }
}


// The radix-R entry points (explicitly instantiated in launch_fft3.cu, launch_fft5.cu and
// launch_fft7.cu).
#define FFB_DECLARE_RADIX_LAUNCHERS(EXT, R)                                                       \
    EXT template cudaError_t launch_r2c_r<R>(int, int, const RowFwdArgs&, cudaStream_t);            \
    EXT template cudaError_t launch_c2r_r<R>(int, int, const RowInvArgs&, cudaStream_t);            \
    EXT template cudaError_t launch_cols_fwd_r<R>(int, int, const ColArgs&, cudaStream_t);          \
    EXT template cudaError_t launch_cols_inv_r<R>(int, int, const ColArgs&, cudaStream_t);          \
    EXT template cudaError_t launch_cols_xcorr_r<R>(int, int, const ColArgs&, cudaStream_t);        \
    EXT template cudaError_t launch_xcorr_r<R>(int, int, const XcorrColArgs&, cudaStream_t);        \
    EXT template size_t xcorr_smem_r<R>(int, int, int, int);

}  // namespace ffb
