// Launchers for the column passes (forward, inverse, fused cross-correlation).
#include "launch_common.cuh"

namespace ffb {

template <int N, int MODE, class ImgC, class InC = float2, class OutC = float2>
static cudaError_t cols_impl(const ColArgs& a, cudaStream_t st) {
    constexpr int FPB = col_fpb<N>();
    constexpr int THREADS = FftShape<N>::T * FPB;
    const size_t smem = (size_t)FftGroup<N, FPB, true>::BYTES;
    static std::atomic<unsigned long long> mask{0};
    auto fn = cols_kernel<N, MODE, InC, ImgC, OutC, FPB>;
    cudaError_t e = ensure_smem_attr((const void*)fn, smem, &mask);
    if (e != cudaSuccess) return e;
    const int grid = (a.n_cols + FPB - 1) / FPB;
    if (grid == 0) return cudaSuccess;
    if (a.n_batch < 1 || a.n_batch > kMaxBatch) return cudaErrorInvalidValue;
    fn<<<dim3(grid, a.n_batch), THREADS, smem, st>>>(a);
    return cudaGetLastError();
}

template <int N>
static cudaError_t fwd_dispatch(int out_dtype, const ColArgs& a, cudaStream_t st) {
    switch (out_dtype) {
        case 3: return cols_impl<N, COL_FWD, float2, float2, float2>(a, st);
        case 4: return cols_impl<N, COL_FWD, float2, float2, __half2>(a, st);
        case 5: return cols_impl<N, COL_FWD, float2, float2, __nv_bfloat162>(a, st);
        default: return cudaErrorInvalidValue;
    }
}
template <int N>
static cudaError_t inv_dispatch(int in_dtype, const ColArgs& a, cudaStream_t st) {
    switch (in_dtype) {
        case 3: return cols_impl<N, COL_INV, float2, float2>(a, st);
        case 4: return cols_impl<N, COL_INV, float2, __half2>(a, st);
        case 5: return cols_impl<N, COL_INV, float2, __nv_bfloat162>(a, st);
        default: return cudaErrorInvalidValue;
    }
}
template <int N>
static cudaError_t xcorr_dispatch(int img_dtype, const ColArgs& a, cudaStream_t st) {
    switch (img_dtype) {
        case 3: return cols_impl<N, COL_XCORR, float2>(a, st);
        case 4: return cols_impl<N, COL_XCORR, __half2>(a, st);
        case 5: return cols_impl<N, COL_XCORR, __nv_bfloat162>(a, st);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_cols_fwd(int n, int out_dtype, const ColArgs& a, cudaStream_t st) {
    if (is_3p_size(n)) return launch_cols3_fwd(n, out_dtype, a, st);
    FFB_SIZE_SWITCH(n, fwd_dispatch, out_dtype, a, st)
}
cudaError_t launch_cols_inv(int n, int in_dtype, const ColArgs& a, cudaStream_t st) {
    if (is_3p_size(n)) return launch_cols3_inv(n, in_dtype, a, st);
    FFB_SIZE_SWITCH(n, inv_dispatch, in_dtype, a, st)
}
cudaError_t launch_cols_xcorr(int n, int img_dtype, const ColArgs& a, cudaStream_t st) {
    if (is_3p_size(n)) return launch_cols3_xcorr(n, img_dtype, a, st);
    FFB_SIZE_SWITCH(n, xcorr_dispatch, img_dtype, a, st)
}

}  // namespace ffb
