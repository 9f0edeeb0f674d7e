// Launchers of the chirp-z (Bluestein) passes (kernels_blue.cuh) and their tables: per length N
// the chirp c_n = exp(-i pi n^2 / N) and the filter spectrum FFT_M(b) / M of
// b_m = conj(c_|m|), |m| < N, both evaluated in FP64 (n^2 reduced mod 2N, the filter as a
// direct sum over the 2N - 1 non-zero b_m) and rounded once; generated on first use per device.
#include <map>
#include <mutex>
#include <utility>

#include "kernels_blue.cuh"
#include "launch_common.cuh"

namespace ffb {

namespace {

// chirp (FP64 and FP32) and the FP64 roots W_M^t, t < M
__global__ void blue_chirp_kernel(int n, int m, double2* cd, float2* cf, double2* wm) {
    const int gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid < n) {
        const long long e = ((long long)gid * gid) % (2LL * n);
        double s, c;
        sincospi(-(double)e / (double)n, &s, &c);
        cd[gid] = make_double2(c, s);
        cf[gid] = make_float2((float)c, (float)s);
    }
    if (gid < m) {
        double s, c;
        sincospi(-2.0 * (double)gid / (double)m, &s, &c);
        wm[gid] = make_double2(c, s);
    }
}

// FFT_M(b)[k] / M with b_0 = 1, b_m = b_(M-m) = conj(c_m) for 0 < m < N:
// (1 + sum_m conj(c_m) (W^(mk) + W^(-mk))) / M = (1 + sum_m 2 cos(2 pi m k / M) conj(c_m)) / M
__global__ void blue_filter_kernel(int n, int m, const double2* __restrict__ cd, const double2* __restrict__ wm,
                                   float2* filt) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= m) return;
    double re = 1.0, im = 0.0;
    for (int j = 1; j < n; j++) {
        const double w = 2.0 * wm[(int)(((long long)j * k) % m)].x;
        re += w * cd[j].x;
        im -= w * cd[j].y;
    }
    filt[k] = make_float2((float)(re / m), (float)(im / m));
}

struct BlueTables {
    float2* chirp = nullptr;
    float2* filt = nullptr;
};

std::mutex g_blue_mutex;
std::map<std::pair<int, int>, BlueTables> g_blue;   // (device, N)

cudaError_t blue_tables(int n, BlueArgs* b) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(g_blue_mutex);
    auto it = g_blue.find({dev, n});
    if (it == g_blue.end()) {
        const int m = blue_m(n);
        BlueTables t;
        double2 *cd = nullptr, *wm = nullptr;
        if ((e = cudaMalloc(&t.chirp, sizeof(float2) * n)) != cudaSuccess) return e;
        if ((e = cudaMalloc(&t.filt, sizeof(float2) * m)) != cudaSuccess) {
            cudaFree(t.chirp);
            return e;
        }
        if ((e = cudaMalloc(&cd, sizeof(double2) * n)) == cudaSuccess &&
            (e = cudaMalloc(&wm, sizeof(double2) * m)) == cudaSuccess) {
            cudaStream_t s;
            if ((e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)) == cudaSuccess) {
                const int top = n > m ? n : m;
                blue_chirp_kernel<<<(top + 255) / 256, 256, 0, s>>>(n, m, cd, t.chirp, wm);
                blue_filter_kernel<<<(m + 127) / 128, 128, 0, s>>>(n, m, cd, wm, t.filt);
                e = cudaGetLastError();
                const cudaError_t e2 = cudaStreamSynchronize(s);
                if (e == cudaSuccess) e = e2;
                cudaStreamDestroy(s);
            }
        }
        cudaFree(cd);
        cudaFree(wm);
        if (e != cudaSuccess) {
            cudaFree(t.chirp);
            cudaFree(t.filt);
            return e;
        }
        it = g_blue.emplace(std::make_pair(dev, n), t).first;
    }
    b->chirp = it->second.chirp;
    b->filt = it->second.filt;
    b->n = n;
    return cudaSuccess;
}

template <int M>
constexpr size_t blue_smem() {
    return (size_t)FftGroup<M, 1, true>::BYTES;
}

template <int M, class InT>
cudaError_t r2c_impl(const RowFwdArgs& a, const BlueArgs& b, cudaStream_t st) {
    static std::atomic<int> hw[64];
    auto fn = blue_r2c_rows_kernel<M, InT>;
    cudaError_t e = ensure_smem_at_least((const void*)fn, blue_smem<M>(), hw);
    if (e != cudaSuccess) return e;
    const int grid = (a.n_rows + 1) / 2;
    if (grid == 0) return cudaSuccess;
    fn<<<dim3(grid, a.n_batch), M / 16, blue_smem<M>(), st>>>(a, b);
    return cudaGetLastError();
}

template <int M, class OutT>
cudaError_t c2r_impl(const RowInvArgs& a, const BlueArgs& b, cudaStream_t st) {
    static std::atomic<int> hw[64];
    auto fn = blue_c2r_rows_kernel<M, OutT>;
    cudaError_t e = ensure_smem_at_least((const void*)fn, blue_smem<M>(), hw);
    if (e != cudaSuccess) return e;
    const int grid = (a.n_rows + 1) / 2;
    if (grid == 0) return cudaSuccess;
    fn<<<dim3(grid, a.n_batch), M / 16, blue_smem<M>(), st>>>(a, b);
    return cudaGetLastError();
}

template <int M, class InC>
cudaError_t c2c_fwd_impl(const RowFwdArgs& a, const BlueArgs& b, cudaStream_t st) {
    static std::atomic<int> hw[64];
    auto fn = blue_c2c_rows_fwd_kernel<M, InC>;
    cudaError_t e = ensure_smem_at_least((const void*)fn, blue_smem<M>(), hw);
    if (e != cudaSuccess) return e;
    if (a.n_rows == 0) return cudaSuccess;
    fn<<<dim3(a.n_rows, a.n_batch), M / 16, blue_smem<M>(), st>>>(a, b);
    return cudaGetLastError();
}

template <int M, class OutC>
cudaError_t c2c_inv_impl(const RowInvArgs& a, const BlueArgs& b, cudaStream_t st) {
    static std::atomic<int> hw[64];
    auto fn = blue_c2c_rows_inv_kernel<M, OutC>;
    cudaError_t e = ensure_smem_at_least((const void*)fn, blue_smem<M>(), hw);
    if (e != cudaSuccess) return e;
    if (a.n_rows == 0) return cudaSuccess;
    fn<<<dim3(a.n_rows, a.n_batch), M / 16, blue_smem<M>(), st>>>(a, b);
    return cudaGetLastError();
}

template <int M, int MODE, class InC, class ImgC, class OutC>
cudaError_t cols_impl(const ColArgs& a, const BlueArgs& b, cudaStream_t st) {
    static std::atomic<int> hw[64];
    auto fn = blue_cols_kernel<M, MODE, InC, ImgC, OutC>;
    cudaError_t e = ensure_smem_at_least((const void*)fn, blue_smem<M>(), hw);
    if (e != cudaSuccess) return e;
    if (a.n_cols == 0) return cudaSuccess;
    fn<<<dim3(a.n_cols, a.n_batch), M / 16, blue_smem<M>(), st>>>(a, b);
    return cudaGetLastError();
}

template <int M>
cudaError_t r2c_m(int in_dtype, const RowFwdArgs& a, const BlueArgs& b, cudaStream_t st) {
    switch (in_dtype) {
        case 0: return r2c_impl<M, float>(a, b, st);
        case 1: return r2c_impl<M, __half>(a, b, st);
        case 2: return r2c_impl<M, __nv_bfloat16>(a, b, st);
        default: return cudaErrorInvalidValue;
    }
}
template <int M>
cudaError_t c2r_m(int out_dtype, const RowInvArgs& a, const BlueArgs& b, cudaStream_t st) {
    switch (out_dtype) {
        case 0: return c2r_impl<M, float>(a, b, st);
        case 1: return c2r_impl<M, __half>(a, b, st);
        case 2: return c2r_impl<M, __nv_bfloat16>(a, b, st);
        default: return cudaErrorInvalidValue;
    }
}
// complex storage: 3 float2, 4 __half2, 5 __nv_bfloat162
template <int M>
cudaError_t c2c_fwd_m(int in_dtype, const RowFwdArgs& a, const BlueArgs& b, cudaStream_t st) {
    switch (in_dtype) {
        case 3: return c2c_fwd_impl<M, float2>(a, b, st);
        case 4: return c2c_fwd_impl<M, __half2>(a, b, st);
        case 5: return c2c_fwd_impl<M, __nv_bfloat162>(a, b, st);
        default: return cudaErrorInvalidValue;
    }
}
template <int M>
cudaError_t c2c_inv_m(int out_dtype, const RowInvArgs& a, const BlueArgs& b, cudaStream_t st) {
    switch (out_dtype) {
        case 3: return c2c_inv_impl<M, float2>(a, b, st);
        case 4: return c2c_inv_impl<M, __half2>(a, b, st);
        case 5: return c2c_inv_impl<M, __nv_bfloat162>(a, b, st);
        default: return cudaErrorInvalidValue;
    }
}
// dtype: the output storage (FWD), the input storage (INV) or the image storage (XCORR), as the
// power-of-two column launchers take it
template <int M>
cudaError_t cols_m(int mode, int dtype, const ColArgs& a, const BlueArgs& b, cudaStream_t st) {
    if (mode == COL_FWD) {
        switch (dtype) {
            case 3: return cols_impl<M, COL_FWD, float2, float2, float2>(a, b, st);
            case 4: return cols_impl<M, COL_FWD, float2, float2, __half2>(a, b, st);
            case 5: return cols_impl<M, COL_FWD, float2, float2, __nv_bfloat162>(a, b, st);
            default: return cudaErrorInvalidValue;
        }
    }
    if (mode == COL_INV) {
        switch (dtype) {
            case 3: return cols_impl<M, COL_INV, float2, float2, float2>(a, b, st);
            case 4: return cols_impl<M, COL_INV, __half2, float2, float2>(a, b, st);
            case 5: return cols_impl<M, COL_INV, __nv_bfloat162, float2, float2>(a, b, st);
            default: return cudaErrorInvalidValue;
        }
    }
    switch (dtype) {
        case 3: return cols_impl<M, COL_XCORR, float2, float2, float2>(a, b, st);
        case 4: return cols_impl<M, COL_XCORR, float2, __half2, float2>(a, b, st);
        case 5: return cols_impl<M, COL_XCORR, float2, __nv_bfloat162, float2>(a, b, st);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace

cudaError_t prepare_blue_tables(int n) {
    if (!is_blue_size(n)) return cudaErrorInvalidValue;
    BlueArgs b;
    return blue_tables(n, &b);
}

#define FFB_BLUE_M_SWITCH(n, FN, ...)                  \
    switch (blue_m(n)) {                               \
        case 64: return FN<64>(__VA_ARGS__);           \
        case 128: return FN<128>(__VA_ARGS__);         \
        case 256: return FN<256>(__VA_ARGS__);         \
        case 512: return FN<512>(__VA_ARGS__);         \
        case 1024: return FN<1024>(__VA_ARGS__);       \
        case 2048: return FN<2048>(__VA_ARGS__);       \
        case 4096: return FN<4096>(__VA_ARGS__);       \
        case 8192: return FN<8192>(__VA_ARGS__);       \
        default: return cudaErrorInvalidValue;         \
    }

cudaError_t launch_blue_r2c(int n, int in_dtype, const RowFwdArgs& a, cudaStream_t st) {
    if (!is_blue_size(n) || a.n_batch < 1 || a.n_batch > kMaxBatch) return cudaErrorInvalidValue;
    BlueArgs b;
    cudaError_t e = blue_tables(n, &b);
    if (e != cudaSuccess) return e;
    FFB_BLUE_M_SWITCH(n, r2c_m, in_dtype, a, b, st)
}

cudaError_t launch_blue_c2r(int n, int out_dtype, const RowInvArgs& a, cudaStream_t st) {
    // the chirp-z row inverse has no fused peak search or projection
    if (!is_blue_size(n) || a.peaks || a.mip || a.n_batch < 1 || a.n_batch > kMaxBatch) return cudaErrorInvalidValue;
    BlueArgs b;
    cudaError_t e = blue_tables(n, &b);
    if (e != cudaSuccess) return e;
    FFB_BLUE_M_SWITCH(n, c2r_m, out_dtype, a, b, st)
}

cudaError_t launch_blue_c2c_fwd(int n, int in_dtype, const RowFwdArgs& a, cudaStream_t st) {
    if (!is_blue_size(n) || a.n_batch < 1 || a.n_batch > kMaxBatch) return cudaErrorInvalidValue;
    BlueArgs b;
    cudaError_t e = blue_tables(n, &b);
    if (e != cudaSuccess) return e;
    FFB_BLUE_M_SWITCH(n, c2c_fwd_m, in_dtype, a, b, st)
}

cudaError_t launch_blue_c2c_inv(int n, int out_dtype, const RowInvArgs& a, cudaStream_t st) {
    if (!is_blue_size(n) || a.peaks || a.mip || a.n_batch < 1 || a.n_batch > kMaxBatch) return cudaErrorInvalidValue;
    BlueArgs b;
    cudaError_t e = blue_tables(n, &b);
    if (e != cudaSuccess) return e;
    FFB_BLUE_M_SWITCH(n, c2c_inv_m, out_dtype, a, b, st)
}

cudaError_t launch_blue_cols(int n, int mode, int dtype, const ColArgs& a, cudaStream_t st) {
    if (!is_blue_size(n) || a.n_batch < 1 || a.n_batch > kMaxBatch) return cudaErrorInvalidValue;
    BlueArgs b;
    cudaError_t e = blue_tables(n, &b);
    if (e != cudaSuccess) return e;
    FFB_BLUE_M_SWITCH(n, cols_m, mode, dtype, a, b, st)
}

}  // namespace ffb
