// Launcher for the batched fused correlation column pass (kernels_xcorr.cuh).
#include "kernels_xcorr.cuh"
#include "launch_common.cuh"

namespace ffb {

// dynamic shared memory available to one block (227 KB, less a little static shared memory)
constexpr int kMaxDynSmem = 227 * 1024 - 1024;

template <int N>
constexpr int xcorr_fpb() {
    return FftShape<N>::T >= kXcorrBlockThreads ? 1 : kXcorrBlockThreads / FftShape<N>::T;
}

template <int N, class ImgC>
static cudaError_t xcorr_v2_impl(const XcorrColArgs& a, cudaStream_t st) {
    if constexpr (N > 4096) {
        return cudaErrorInvalidValue;
    } else {
        constexpr int FPB = xcorr_fpb<N>();
        using SM = XcorrSmem<N, ImgC, FPB>;
        if (a.n_batch < 1 || a.n_batch > kMaxBatch || a.n_cols < 1) return cudaErrorInvalidValue;
        if (a.tpb < 1 || a.tpb > a.n_batch) return cudaErrorInvalidValue;
        const int smem = SM::total(a.L, a.tpb);
        if (smem > kMaxDynSmem) return cudaErrorInvalidValue;
        static std::atomic<int> set_mul[64], set_nomul[64];
        const bool mul = a.intra_kind != 0;
        auto fn = mul ? xcorr_cols_kernel<N, ImgC, FPB, true> : xcorr_cols_kernel<N, ImgC, FPB, false>;
        cudaError_t e = ensure_smem_at_least((const void*)fn, (size_t)smem, mul ? set_mul : set_nomul);
        if (e != cudaSuccess) return e;
        fn<<<dim3(a.n_cols, (a.n_batch + a.tpb - 1) / a.tpb), FftShape<N>::T * FPB, smem, st>>>(a);
        return cudaGetLastError();
    }
}

template <int N>
static cudaError_t xcorr_v2_dispatch(int img_dtype, const XcorrColArgs& a, cudaStream_t st) {
    switch (img_dtype) {
        case 3: return xcorr_v2_impl<N, float2>(a, st);
        case 4: return xcorr_v2_impl<N, __half2>(a, st);
        case 5: return xcorr_v2_impl<N, __nv_bfloat162>(a, st);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_xcorr_cols(int n, int img_dtype, const XcorrColArgs& a, cudaStream_t st) {
    if (is_rp_size(n)) return launch_xcorr3(n, img_dtype, a, st);
    FFB_SIZE_SWITCH(n, xcorr_v2_dispatch, img_dtype, a, st)
}

size_t xcorr_cols_smem(int n, int img_dtype, int L, int n_batch) {
    if (is_rp_size(n)) return xcorr3_smem(n, img_dtype, L, n_batch);
    const int isz = img_dtype == 3 ? 8 : 4;
    const int fpb = (n / 16) >= kXcorrBlockThreads ? 1 : kXcorrBlockThreads / (n / 16);
    const size_t img = ((size_t)n * isz + 127) & ~(size_t)127;
    const size_t smem_fft = (size_t)(((n + n / 16) + 15) / 16) * 16 + 4;  // FftShape::SMEM_PAD
    const size_t xch = (size_t)fpb * 2 * smem_fft * 8;                    // double-buffered groups
    const size_t t1 = (size_t)n_batch * (size_t)((L + 1) & ~1) * 8;
    return ((img + xch + t1 + 15) & ~(size_t)15) + 16;
}

}  // namespace ffb
