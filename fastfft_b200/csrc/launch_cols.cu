// Launchers for the column passes (forward, inverse, fused cross-correlation).
#include "launch_common.cuh"

namespace ffb {

template <int N, int MODE, class ImgC, class InC = float2, class OutC = float2>
static cudaError_t cols_impl(const ColArgs& args, cudaStream_t st) {
    constexpr int FPB = col_fpb<N>();
    constexpr int THREADS = FftShape<N>::T * FPB;
    using CS = ColSmem<N, ImgC, FPB>;
    ColArgs a = args;
    // The fused pass with one column per block stages its image column by a bulk copy when
    // every column starts on a 16-byte boundary (cp.async.bulk needs 16-byte aligned
    // addresses and sizes; N * sizeof(ImgC) is a multiple of 16 for N >= 16).
    const size_t isz = sizeof(ImgC);
    a.stage_img = MODE == COL_XCORR && FPB == 1 && a.intra_kind != 0 && a.img != nullptr &&
                  reinterpret_cast<uintptr_t>(a.img) % 16 == 0 && (a.img_stride * isz) % 16 == 0 &&
                  (a.img_batch_stride * isz) % 16 == 0;
    // transposed output through shared memory when the block's FPB columns are consecutive in
    // memory for every element: out_stride2 == 1 within a block that does not cross an
    // out_div boundary, or consecutive columns one element apart (out_div 1, out_stride 1)
    const int out_div = a.out_div > 0 ? a.out_div : 1;
    a.out_coalesce = FPB > 1 && a.out_elem_stride > 1 &&
                     ((out_div % FPB == 0 && a.out_stride2 == 1) || (out_div == 1 && a.out_stride == 1));
    const size_t smem = a.stage_img ? (size_t)CS::kStagedBytes : (size_t)CS::kXchBytes;
    static std::atomic<int> high_water[64];
    auto fn = cols_kernel<N, MODE, InC, ImgC, OutC, FPB>;
    cudaError_t e = ensure_smem_at_least((const void*)fn, smem, high_water);
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
    if (is_rp_size(n)) return launch_cols3_fwd(n, out_dtype, a, st);
    if (is_blue_size(n)) return launch_blue_cols(n, COL_FWD, out_dtype, a, st);
    FFB_SIZE_SWITCH(n, fwd_dispatch, out_dtype, a, st)
}
cudaError_t launch_cols_inv(int n, int in_dtype, const ColArgs& a, cudaStream_t st) {
    if (is_rp_size(n)) return launch_cols3_inv(n, in_dtype, a, st);
    if (is_blue_size(n)) return launch_blue_cols(n, COL_INV, in_dtype, a, st);
    FFB_SIZE_SWITCH(n, inv_dispatch, in_dtype, a, st)
}
cudaError_t launch_cols_xcorr(int n, int img_dtype, const ColArgs& a, cudaStream_t st) {
    if (is_rp_size(n)) return launch_cols3_xcorr(n, img_dtype, a, st);
    if (is_blue_size(n)) return launch_blue_cols(n, COL_XCORR, img_dtype, a, st);
    FFB_SIZE_SWITCH(n, xcorr_dispatch, img_dtype, a, st)
}

}  // namespace ffb
