// Launcher of the tensor-core fused 1536-point column pass (kernels_tc.cuh) and the
// generation of its constants: the BF16 hi / lo real forms of the 48- and 32-point DFT
// matrices in their shared-memory byte image, and the W1536 table (FP64 sincospi, rounded
// once).
#include <mutex>

#include "kernels_tc.cuh"
#include "launch.h"

namespace ffb {

__device__ __align__(16) uint8_t g_tc1536[tc1536::kConstBytes];

namespace {

// element (r, k) of the real form of the n-point DFT matrix W_n^(o i), o = r / 2, i = k / 2:
// [[Re, -Im], [Im, Re]] per complex entry
__device__ double dft_real_form(int n, int r, int k) {
    const int o = r >> 1, i = k >> 1;
    const int e = (o * i) % n;
    double s, c;
    sincospi(-2.0 * (double)e / (double)n, &s, &c);
    if ((r & 1) == 0) return (k & 1) == 0 ? c : -s;
    return (k & 1) == 0 ? s : c;
}

__global__ void init_tc1536_kernel(uint8_t* out) {
    using namespace tc1536;
    const int gid = blockIdx.x * blockDim.x + threadIdx.x;
    constexpr int n48 = 96 * 96, n32 = 64 * 64;
    if (gid < n48 + n32) {
        const bool big = gid < n48;
        const int id = big ? gid : gid - n48;
        const int dim = big ? 96 : 64;
        const int r = id / dim, k = id - (id / dim) * dim;
        const double v = dft_real_form(big ? 48 : 32, r, k);
        const __nv_bfloat16 hi = __float2bfloat16_rn((float)v);
        const __nv_bfloat16 lo = __float2bfloat16_rn((float)(v - (double)__bfloat162float(hi)));
        const int off = (r >> 3) * (big ? kB48Sbo : kB32Sbo) + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2;
        *reinterpret_cast<__nv_bfloat16*>(out + (big ? kB48h : kB32h) + off) = hi;
        *reinterpret_cast<__nv_bfloat16*>(out + (big ? kB48l : kB32l) + off) = lo;
    } else if (gid < n48 + n32 + kN) {
        const int m = gid - n48 - n32;
        double s, c;
        sincospi(-2.0 * (double)m / (double)kN, &s, &c);
        reinterpret_cast<float2*>(out + kTwOff)[m] = make_float2((float)c, (float)s);
    }
}

std::mutex g_tc_mutex;
const uint8_t* g_tc_ptr[64] = {nullptr};
int g_sms[64] = {0};

cudaError_t tc1536_consts(const uint8_t** out, int* sms) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_tc_mutex);
    if (!g_tc_ptr[dev]) {
        void* p = nullptr;
        if ((e = cudaGetSymbolAddress(&p, g_tc1536)) != cudaSuccess) return e;
        if ((e = cudaDeviceGetAttribute(&g_sms[dev], cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
        cudaStream_t s;
        if ((e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)) != cudaSuccess) return e;
        constexpr int total = 96 * 96 + 64 * 64 + tc1536::kN;
        init_tc1536_kernel<<<(total + 255) / 256, 256, 0, s>>>(static_cast<uint8_t*>(p));
        e = cudaGetLastError();
        const cudaError_t e2 = cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
        if (e != cudaSuccess) return e;
        if (e2 != cudaSuccess) return e2;
        g_tc_ptr[dev] = static_cast<const uint8_t*>(p);
    }
    *out = g_tc_ptr[dev];
    *sms = g_sms[dev];
    return cudaSuccess;
}

template <class ImgC>
cudaError_t launch_tc_typed(const XcorrColArgs& a, const uint8_t* consts, int sms, cudaStream_t st) {
    static std::atomic<int> set_attr[64];
    auto fn = xcorr1536_tc_kernel<ImgC>;
    cudaError_t e = ensure_smem_at_least((const void*)fn, (size_t)tc1536::kSmemBytes, set_attr);
    if (e != cudaSuccess) return e;
    const int n_items = a.n_cols * ((a.n_batch + tc1536::kTpi - 1) / tc1536::kTpi);
    const int want = (n_items + tc1536::kWgs - 1) / tc1536::kWgs;
    const int grid = want < sms ? want : sms;
    fn<<<grid, tc1536::kThreads, tc1536::kSmemBytes, st>>>(a, consts, n_items);
    return cudaGetLastError();
}

}  // namespace

bool xcorr1536_tc_supported(const XcorrColArgs& a) {
    if (a.n_batch < 1 || a.n_batch > kMaxBatch || a.n_cols < 1) return false;
    if (a.intra_kind != 2 && a.intra_kind != 3) return false;   // CONJ_MUL, CONJ_MUL_THEN_SCALE
    if (a.L < 1 || a.L > tc1536::kMaxL || a.W < 1 || a.W > tc1536::kN) return false;
    for (int g = 0; g < a.n_batch; g++)
        if (a.L_g[g] > tc1536::kMaxL) return false;
    return true;
}

cudaError_t launch_xcorr1536_tc(int img_dtype, const XcorrColArgs& a, cudaStream_t st) {
    if (!xcorr1536_tc_supported(a)) return cudaErrorInvalidValue;
    const uint8_t* consts = nullptr;
    int sms = 0;
    cudaError_t e = tc1536_consts(&consts, &sms);
    if (e != cudaSuccess) return e;
    switch (img_dtype) {
        case 3: return launch_tc_typed<float2>(a, consts, sms, st);
        case 4: return launch_tc_typed<__half2>(a, consts, sms, st);
        case 5: return launch_tc_typed<__nv_bfloat162>(a, consts, sms, st);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace ffb
