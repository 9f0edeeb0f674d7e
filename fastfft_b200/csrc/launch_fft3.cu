// Radix-3 instantiation of the length-RP launchers (lengths 3 * 2^k; see launch_fftr.cuh) and
// the public launchers of these lengths, which pick the radix of N (the radix-5 and radix-7
// instances are compiled in launch_fft5.cu and launch_fft7.cu).
#include "launch_fftr.cuh"

namespace ffb {

FFB_DECLARE_RADIX_LAUNCHERS(, 3)
FFB_DECLARE_RADIX_LAUNCHERS(extern, 5)
FFB_DECLARE_RADIX_LAUNCHERS(extern, 7)

// FN<R>(args...) for the radix R of the length n
#define FFB_BY_RADIX(n, FN, ...) \
    (is_7p_size(n) ? FN<7>(__VA_ARGS__) : is_5p_size(n) ? FN<5>(__VA_ARGS__) : FN<3>(__VA_ARGS__))

cudaError_t launch_r2c3(int n, int in_dtype, const RowFwdArgs& a, cudaStream_t st) {
    return FFB_BY_RADIX(n, launch_r2c_r, n, in_dtype, a, st);
}
cudaError_t launch_c2r3(int n, int out_dtype, const RowInvArgs& a, cudaStream_t st) {
    return FFB_BY_RADIX(n, launch_c2r_r, n, out_dtype, a, st);
}
cudaError_t launch_cols3_fwd(int n, int out_dtype, const ColArgs& a, cudaStream_t st) {
    return FFB_BY_RADIX(n, launch_cols_fwd_r, n, out_dtype, a, st);
}
cudaError_t launch_cols3_inv(int n, int in_dtype, const ColArgs& a, cudaStream_t st) {
    return FFB_BY_RADIX(n, launch_cols_inv_r, n, in_dtype, a, st);
}
cudaError_t launch_cols3_xcorr(int n, int img_dtype, const ColArgs& a, cudaStream_t st) {
    return FFB_BY_RADIX(n, launch_cols_xcorr_r, n, img_dtype, a, st);
}
cudaError_t launch_xcorr3(int n, int img_dtype, const XcorrColArgs& a, cudaStream_t st) {
    if (n == 3 * 512 && a.tc && xcorr1536_tc_supported(a)) return launch_xcorr1536_tc(img_dtype, a, st);
    return FFB_BY_RADIX(n, launch_xcorr_r, n, img_dtype, a, st);
}
size_t xcorr3_smem(int n, int img_dtype, int L, int n_batch) {
    return FFB_BY_RADIX(n, xcorr_smem_r, n, img_dtype, L, n_batch);
}

}  // namespace ffb
