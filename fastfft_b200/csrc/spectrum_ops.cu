// Radial operations on square 2D half spectra in the [kx][ky] layout (ky contiguous, kx in
// [0, N/2], ky in [0, N)): the rotationally averaged power spectrum, and the multiplication by
// a radial filter (band-pass, or whitening with 1 / sqrt of that power), with the filtered
// spectrum written in FP32, FP16 or BF16 storage.  These prepare an image spectrum before the
// correlation; they are memory-bound passes over the spectrum.
//
// Radius of element (kx, ky): r = floor(sqrt(kx^2 + sy^2)), sy = ky for ky <= N/2 else ky - N,
// in frequency-index units, computed exactly in integers; radii at or beyond n_bins - 1 use
// the last bin.  In the half spectrum, columns 0 < kx < N/2 stand for two conjugate elements
// of the full spectrum and count twice in the averages.
#include "launch_common.cuh"
#include "spectrum_ops.h"

namespace ffb {

__device__ __forceinline__ int radial_bin(int kx, int ky, int n, int n_bins) {
    const int sy = ky <= n / 2 ? ky : ky - n;
    const int v = kx * kx + sy * sy;  // < 2^26 for n <= 8192: the float estimate is corrected
    int r = (int)sqrtf((float)v);
    while (r * r > v) r--;
    while ((r + 1) * (r + 1) <= v) r++;
    return r < n_bins ? r : n_bins - 1;
}

template <class OutC>
__global__ void __launch_bounds__(256) radial_filter_kernel(RadialArgs a) {
    const int kx = blockIdx.y;
    const float2* in = a.in + (long long)kx * a.n;
    OutC* out = static_cast<OutC*>(a.out) + (long long)kx * a.n;
    for (int ky = blockIdx.x * blockDim.x + threadIdx.x; ky < a.n; ky += gridDim.x * blockDim.x) {
        const float f = a.filter[radial_bin(kx, ky, a.n, a.n_bins)] * a.scale;
        const float2 v = in[ky];
        st_cplx<OutC>(out + ky, make_float2(v.x * f, v.y * f));
    }
}

// Block-wise histogram in shared memory (float), folded into the global double sums.
__global__ void __launch_bounds__(256) radial_power_kernel(RadialArgs a) {
    extern __shared__ float hist[];  // 2 * n_bins: sums, weights
    for (int b = threadIdx.x; b < 2 * a.n_bins; b += blockDim.x) hist[b] = 0.f;
    __syncthreads();
    const int nkx = a.n / 2 + 1;
    const long long total = (long long)nkx * a.n;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int kx = (int)(i / a.n), ky = (int)(i - (long long)kx * a.n);
        const float2 v = a.in[i];
        const float w = (kx == 0 || 2 * kx == a.n) ? 1.f : 2.f;
        const int b = radial_bin(kx, ky, a.n, a.n_bins);
        atomicAdd(&hist[b], w * (v.x * v.x + v.y * v.y));
        atomicAdd(&hist[a.n_bins + b], w);
    }
    __syncthreads();
    for (int b = threadIdx.x; b < a.n_bins; b += blockDim.x) {
        if (hist[a.n_bins + b] != 0.f) {
            atomicAdd(a.sums + b, (double)hist[b]);
            atomicAdd(a.weights + b, (double)hist[a.n_bins + b]);
        }
    }
}

__global__ void radial_power_finish_kernel(const double* sums, const double* weights, float* power, int n_bins) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < n_bins) power[b] = weights[b] > 0.0 ? (float)(sums[b] / weights[b]) : 0.f;
}

cudaError_t launch_radial_filter(int out_dtype, const RadialArgs& a, cudaStream_t st) {
    if (a.n < 2 || a.n_bins < 1) return cudaErrorInvalidValue;
    const dim3 grid((a.n + 255) / 256, a.n / 2 + 1);
    switch (out_dtype) {
        case 3: radial_filter_kernel<float2><<<grid, 256, 0, st>>>(a); break;
        case 4: radial_filter_kernel<__half2><<<grid, 256, 0, st>>>(a); break;
        case 5: radial_filter_kernel<__nv_bfloat162><<<grid, 256, 0, st>>>(a); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

// sums and weights: 2 * n_bins doubles of scratch, zeroed here
cudaError_t launch_radial_power(const RadialArgs& a, float* power, cudaStream_t st) {
    if (a.n < 2 || a.n_bins < 1) return cudaErrorInvalidValue;
    const size_t smem = (size_t)2 * a.n_bins * sizeof(float);
    static std::atomic<int> set[64];
    cudaError_t e = ensure_smem_at_least((const void*)radial_power_kernel, smem, set);
    if (e != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(a.sums, 0, (size_t)a.n_bins * sizeof(double), st)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(a.weights, 0, (size_t)a.n_bins * sizeof(double), st)) != cudaSuccess) return e;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    radial_power_kernel<<<2 * sms, 256, smem, st>>>(a);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    radial_power_finish_kernel<<<(a.n_bins + 255) / 256, 256, 0, st>>>(a.sums, a.weights, power, a.n_bins);
    return cudaGetLastError();
}

}  // namespace ffb
