// Launchers for the row passes (R2C forward, C2R inverse).
#include "kernels_c2c.cuh"
#include "launch_common.cuh"

namespace ffb {

template <int N, class InT>
static cudaError_t r2c_impl(const RowFwdArgs& a, cudaStream_t st) {
    constexpr int FPB = r2c_fpb<N>();
    constexpr int THREADS = FftShape<N>::T * FPB;
    const size_t smem = (size_t)FftGroup<N, FPB, false>::BYTES;
    static std::atomic<unsigned long long> mask{0};
    auto fn = r2c_rows_kernel<N, InT, FPB>;
    cudaError_t e = ensure_smem_attr((const void*)fn, smem, &mask);
    if (e != cudaSuccess) return e;
    const int grid = (a.n_rows + 2 * FPB - 1) / (2 * FPB);
    if (grid == 0) return cudaSuccess;
    if (a.n_batch < 1 || a.n_batch > kMaxBatch) return cudaErrorInvalidValue;
    fn<<<dim3(grid, a.n_batch), THREADS, smem, st>>>(a);
    return cudaGetLastError();
}

template <int N>
static cudaError_t r2c_dispatch(int in_dtype, const RowFwdArgs& a, cudaStream_t st) {
    switch (in_dtype) {
        case 0: return r2c_impl<N, float>(a, st);
        case 1: return r2c_impl<N, __half>(a, st);
        case 2: return r2c_impl<N, __nv_bfloat16>(a, st);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_r2c_rows(int n, int in_dtype, const RowFwdArgs& a, cudaStream_t st) {
    if (is_rp_size(n)) return launch_r2c3(n, in_dtype, a, st);
    if (is_blue_size(n)) return launch_blue_r2c(n, in_dtype, a, st);
    FFB_SIZE_SWITCH(n, r2c_dispatch, in_dtype, a, st)
}

template <int N, class OutT>
static cudaError_t c2r_impl(const RowInvArgs& a, cudaStream_t st) {
    constexpr int FPB = c2r_fpb<N>();
    constexpr int THREADS = FftShape<N>::T * FPB;
    const size_t smem = (size_t)FftGroup<N, FPB, false>::BYTES;
    static std::atomic<unsigned long long> mask{0};
    auto fn = c2r_rows_kernel<N, OutT, FPB>;
    cudaError_t e = ensure_smem_attr((const void*)fn, smem, &mask);
    if (e != cudaSuccess) return e;
    const int grid = (a.n_rows + 2 * FPB - 1) / (2 * FPB);
    if (grid == 0) return cudaSuccess;
    if (a.n_batch < 1 || a.n_batch > kMaxBatch) return cudaErrorInvalidValue;
    fn<<<dim3(grid, a.n_batch), THREADS, smem, st>>>(a);
    return cudaGetLastError();
}

template <int N>
static cudaError_t c2r_dispatch(int out_dtype, const RowInvArgs& a, cudaStream_t st) {
    switch (out_dtype) {
        case 0: return c2r_impl<N, float>(a, st);
        case 1: return c2r_impl<N, __half>(a, st);
        case 2: return c2r_impl<N, __nv_bfloat16>(a, st);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_c2r_rows(int n, int out_dtype, const RowInvArgs& a, cudaStream_t st) {
    if (is_rp_size(n)) return launch_c2r3(n, out_dtype, a, st);
    if (is_blue_size(n)) return launch_blue_c2r(n, out_dtype, a, st);
    FFB_SIZE_SWITCH(n, c2r_dispatch, out_dtype, a, st)
}

// Complex-input (C2C) row passes: one complex row per FFT, 512-thread blocks.
template <int N, class InC>
static cudaError_t c2c_fwd_impl(const RowFwdArgs& a, cudaStream_t st) {
    constexpr int FPB = row_fpb<N>();
    constexpr int THREADS = FftShape<N>::T * FPB;
    const size_t smem = (size_t)FftGroup<N, FPB, false>::BYTES;
    static std::atomic<unsigned long long> mask{0};
    auto fn = c2c_rows_fwd_kernel<N, InC, FPB>;
    cudaError_t e = ensure_smem_attr((const void*)fn, smem, &mask);
    if (e != cudaSuccess) return e;
    const int grid = (a.n_rows + FPB - 1) / FPB;
    if (grid == 0) return cudaSuccess;
    if (a.n_batch < 1 || a.n_batch > kMaxBatch || a.kmax > N) return cudaErrorInvalidValue;
    fn<<<dim3(grid, a.n_batch), THREADS, smem, st>>>(a);
    return cudaGetLastError();
}

template <int N>
static cudaError_t c2c_fwd_dispatch(int in_dtype, const RowFwdArgs& a, cudaStream_t st) {
    switch (in_dtype) {
        case 3: return c2c_fwd_impl<N, float2>(a, st);
        case 4: return c2c_fwd_impl<N, __half2>(a, st);
        case 5: return c2c_fwd_impl<N, __nv_bfloat162>(a, st);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_c2c_rows_fwd(int n, int in_dtype, const RowFwdArgs& a, cudaStream_t st) {
    if (is_blue_size(n)) return launch_blue_c2c_fwd(n, in_dtype, a, st);
    FFB_SIZE_SWITCH(n, c2c_fwd_dispatch, in_dtype, a, st)
}

template <int N, class OutC>
static cudaError_t c2c_inv_impl(const RowInvArgs& a, cudaStream_t st) {
    constexpr int FPB = row_fpb<N>();
    constexpr int THREADS = FftShape<N>::T * FPB;
    const size_t smem = (size_t)FftGroup<N, FPB, false>::BYTES;
    static std::atomic<unsigned long long> mask{0};
    auto fn = c2c_rows_inv_kernel<N, OutC, FPB>;
    cudaError_t e = ensure_smem_attr((const void*)fn, smem, &mask);
    if (e != cudaSuccess) return e;
    const int grid = (a.n_rows + FPB - 1) / FPB;
    if (grid == 0) return cudaSuccess;
    if (a.n_batch < 1 || a.n_batch > kMaxBatch) return cudaErrorInvalidValue;
    fn<<<dim3(grid, a.n_batch), THREADS, smem, st>>>(a);
    return cudaGetLastError();
}

template <int N>
static cudaError_t c2c_inv_dispatch(int out_dtype, const RowInvArgs& a, cudaStream_t st) {
    switch (out_dtype) {
        case 3: return c2c_inv_impl<N, float2>(a, st);
        case 4: return c2c_inv_impl<N, __half2>(a, st);
        case 5: return c2c_inv_impl<N, __nv_bfloat162>(a, st);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_c2c_rows_inv(int n, int out_dtype, const RowInvArgs& a, cudaStream_t st) {
    if (is_blue_size(n)) return launch_blue_c2c_inv(n, out_dtype, a, st);
    FFB_SIZE_SWITCH(n, c2c_inv_dispatch, out_dtype, a, st)
}

}  // namespace ffb
