// Host-side launchers for the pass kernels (one translation unit per kernel family,
// so the sm_100a build compiles in parallel).  Each launcher picks the compile-time
// FFT size from the runtime N (power of two in [16, 8192], or 3P for the passes of the
// reduced-size correlation) and the data types.
#pragma once

#include <cuda_runtime.h>

#include <atomic>

namespace ffb {

struct RowFwdArgs;
struct ColArgs;
struct RowInvArgs;
struct XcorrColArgs;

// dtype codes follow fastfft_dtype in include/fastfft_capi.h
cudaError_t launch_r2c_rows(int n, int in_dtype, const RowFwdArgs& a, cudaStream_t st);
cudaError_t launch_c2r_rows(int n, int out_dtype, const RowInvArgs& a, cudaStream_t st);
// Complex-input row passes (in_dtype / out_dtype: 3 complex64, 4 complex32, 5 complex bf16).
cudaError_t launch_c2c_rows_fwd(int n, int in_dtype, const RowFwdArgs& a, cudaStream_t st);
cudaError_t launch_c2c_rows_inv(int n, int out_dtype, const RowInvArgs& a, cudaStream_t st);
// out_dtype: storage of the spectrum written (3 complex64, 4 complex32, 5 complex bf16)
cudaError_t launch_cols_fwd(int n, int out_dtype, const ColArgs& a, cudaStream_t st);
cudaError_t launch_cols_inv(int n, int in_dtype, const ColArgs& a, cudaStream_t st);
cudaError_t launch_cols_xcorr(int n, int img_dtype, const ColArgs& a, cudaStream_t st);
// Batched fused column pass (TMA-staged image and template columns), n <= 4096.
cudaError_t launch_xcorr_cols(int n, int img_dtype, const XcorrColArgs& a, cudaStream_t st);
size_t xcorr_cols_smem(int n, int img_dtype, int L, int n_batch);

// Lengths N = 3P (128 <= P <= 2048): the reduced-size correlation's internal sizes and the
// 2D plans at these sizes; the public launchers above forward them here.
cudaError_t launch_r2c3(int n, int in_dtype, const RowFwdArgs& a, cudaStream_t st);
cudaError_t launch_c2r3(int n, int out_dtype, const RowInvArgs& a, cudaStream_t st);
cudaError_t launch_cols3_fwd(int n, int out_dtype, const ColArgs& a, cudaStream_t st);
cudaError_t launch_cols3_inv(int n, int in_dtype, const ColArgs& a, cudaStream_t st);
cudaError_t launch_cols3_xcorr(int n, int img_dtype, const ColArgs& a, cudaStream_t st);
cudaError_t launch_xcorr3(int n, int img_dtype, const XcorrColArgs& a, cudaStream_t st);
size_t xcorr3_smem(int n, int img_dtype, int L, int n_batch);
// Tensor-core form of the batched fused column pass at length 1536 (kernels_tc.cuh): templates
// of up to 512 rows, windows of up to 1536; launch_xcorr3 routes calls with a.tc set here.
bool xcorr1536_tc_supported(const XcorrColArgs& a);
cudaError_t launch_xcorr1536_tc(int img_dtype, const XcorrColArgs& a, cudaStream_t st);

// Any other length in [17, 4096] (kernels_blue.cuh, chirp-z on a power-of-two FFT): row R2C,
// row C2R (no peak search or projection), complex rows, column passes (2D and 3D addressing).  The caller's `tw`
// is the table twiddles_for(n) returns (of the power-of-two length the path runs on).
cudaError_t launch_blue_r2c(int n, int in_dtype, const RowFwdArgs& a, cudaStream_t st);
cudaError_t launch_blue_c2r(int n, int out_dtype, const RowInvArgs& a, cudaStream_t st);
cudaError_t launch_blue_cols(int n, int mode, int dtype, const ColArgs& a, cudaStream_t st);
cudaError_t launch_blue_c2c_fwd(int n, int in_dtype, const RowFwdArgs& a, cudaStream_t st);
cudaError_t launch_blue_c2c_inv(int n, int out_dtype, const RowInvArgs& a, cudaStream_t st);
// Builds (once per device and length, synchronously) the chirp and filter tables of length n.
cudaError_t prepare_blue_tables(int n);

// Radial operations on square 2D half spectra (spectrum_ops.cu).
struct RadialArgs;
cudaError_t launch_radial_filter(int out_dtype, const RadialArgs& a, cudaStream_t st);
cudaError_t launch_radial_power(const RadialArgs& a, float* power, cudaStream_t st);

// Device-wide FP64-generated twiddle tables (generated once per device): for a power of
// two n the radix-16 pass table, for n = 3P the radix-3 pass table W_n^m, m < 2P.
cudaError_t twiddles_for(int n, const float2** out);

// Message returned by fastfft_last_error(NULL), for entry points without a handle.
void set_unbound_error(const char* msg);

// Raises cudaFuncAttributeMaxDynamicSharedMemorySize of func on the current device to at
// least `bytes` (per_device: 64 per-device high-water marks owned by the caller).
cudaError_t ensure_smem_at_least(const void* func, size_t bytes, std::atomic<int>* per_device);

// Sets cudaFuncAttributeMaxDynamicSharedMemorySize once per (kernel, device).
cudaError_t ensure_smem_attr(const void* func, size_t bytes, std::atomic<unsigned long long>* done_mask);

}  // namespace ffb
