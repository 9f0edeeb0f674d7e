// Device-wide twiddle table and per-device/per-kernel one-time set-up.
#include <mutex>

#include "launch_common.cuh"

namespace ffb {

// ---------------------------------------------------------------------------
// Twiddle table generation: FP64 sincospi, rounded once to FP32
// ---------------------------------------------------------------------------
static __global__ void init_twiddles_kernel(float2* tw) {
    const int gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= kTwTotal) return;
    // locate (size n, pass, r, t) of entry gid; layout in FftShape
    int base = 0;
    for (int n = kMinN; n <= kMaxN; n *= 2) {
        const int sz = tw_size_of(n);
        if (gid < base + sz) {
            int local = gid - base;
            const int log = ilog2(n);
            const int rem = 1 << (log & 3);
            const int np16 = log >> 2;
            // exponent e of W_d^e = exp(-2 pi i e / d) = cospi(-x) + i sinpi(-x), x = 2 e / d
            long long e = 0, d = 1;
            int ns = 16;
            int p = 1;
            for (; p < np16; p++) {
                if (local < 16 * ns) {
                    const int r = local / ns;
                    e = (long long)r * (local - r * ns);
                    d = 16LL * ns;
                    break;
                }
                local -= 16 * ns;
                ns *= 16;
            }
            if (p == np16) {
                // closing radix-rem pass: (r-1) n/rem + b  ->  W_n^(r b)
                const int nr = n / rem;
                const int r = 1 + local / nr;
                e = (long long)r * (local - (r - 1) * nr);
                d = n;
            }
            const double x = -2.0 * (double)e / (double)d;
            double sv, cv;
            sincospi(x, &sv, &cv);
            tw[gid] = make_float2((float)cv, (float)sv);
            return;
        }
        base += sz;
    }
}


// Radix-R pass tables of the lengths N = RP: W_N^m = exp(-2 pi i m / N), m < (R - 1) P.
static __global__ void init_twiddles_r_kernel(float2* tw, int r) {
    const int gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= twr_total(r)) return;
    for (int p = kMinP3; p <= kMaxPR(r); p *= 2) {
        const int base = twr_base(r, p);
        if (gid < base + twr_size_of(r, p)) {
            const int m = gid - base;
            // exp(-2 pi i m / rp) = cospi(-x) + i sinpi(-x), x = 2 m / rp
            const double x = -2.0 * (double)m / ((double)r * (double)p);
            double sv, cv;
            sincospi(x, &sv, &cv);
            tw[gid] = make_float2((float)cv, (float)sv);
            return;
        }
    }
}

// One table for every supported size, generated on the device in FP64 and rounded
// once to FP32 (the reference evaluates __sincosf per element instead,
// include/detail/device_functions.h:17-27).
__device__ float2 g_twiddles[kTwTotal];
__device__ float2 g_twiddles3[kTw3Total];
__device__ float2 g_twiddles5[kTw5Total];
__device__ float2 g_twiddles7[kTw7Total];

namespace {
std::mutex g_tw_mutex;
const float2* g_tw_ptr[64] = {nullptr};
const float2* g_tw3_ptr[64] = {nullptr};
const float2* g_tw5_ptr[64] = {nullptr};
const float2* g_tw7_ptr[64] = {nullptr};
}  // namespace

cudaError_t twiddles_for(int n, const float2** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_tw_mutex);
    if (!g_tw_ptr[dev]) {
        void* p = nullptr;
        void* p3 = nullptr;
        void* p5 = nullptr;
        void* p7 = nullptr;
        e = cudaGetSymbolAddress(&p, g_twiddles);
        if (e != cudaSuccess) return e;
        e = cudaGetSymbolAddress(&p3, g_twiddles3);
        if (e != cudaSuccess) return e;
        e = cudaGetSymbolAddress(&p5, g_twiddles5);
        if (e != cudaSuccess) return e;
        e = cudaGetSymbolAddress(&p7, g_twiddles7);
        if (e != cudaSuccess) return e;
        cudaStream_t s;
        e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
        if (e != cudaSuccess) return e;
        init_twiddles_kernel<<<(kTwTotal + 255) / 256, 256, 0, s>>>(static_cast<float2*>(p));
        e = cudaGetLastError();
        if (e == cudaSuccess) {
            init_twiddles_r_kernel<<<(kTw3Total + 255) / 256, 256, 0, s>>>(static_cast<float2*>(p3), 3);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) {
            init_twiddles_r_kernel<<<(kTw5Total + 255) / 256, 256, 0, s>>>(static_cast<float2*>(p5), 5);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) {
            init_twiddles_r_kernel<<<(kTw7Total + 255) / 256, 256, 0, s>>>(static_cast<float2*>(p7), 7);
            e = cudaGetLastError();
        }
        cudaError_t e2 = cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
        if (e != cudaSuccess) return e;
        if (e2 != cudaSuccess) return e2;
        g_tw_ptr[dev] = static_cast<const float2*>(p);
        g_tw3_ptr[dev] = static_cast<const float2*>(p3);
        g_tw5_ptr[dev] = static_cast<const float2*>(p5);
        g_tw7_ptr[dev] = static_cast<const float2*>(p7);
    }
    if (is_3p_size(n)) {
        *out = g_tw3_ptr[dev] + twr_base(3, n / 3);
        return cudaSuccess;
    }
    if (is_5p_size(n)) {
        *out = g_tw5_ptr[dev] + twr_base(5, n / 5);
        return cudaSuccess;
    }
    if (is_7p_size(n)) {
        *out = g_tw7_ptr[dev] + twr_base(7, n / 7);
        return cudaSuccess;
    }
    if (is_blue_size(n)) n = blue_m(n);   // the chirp-z path runs on the power-of-two FFT of this length
    if (!is_pow2_size(n) || n < kMinN || n > kMaxN) return cudaErrorInvalidValue;
    int base = 0;
    for (int m = kMinN; m < n; m *= 2) base += tw_size_of(m);
    *out = g_tw_ptr[dev] + base;
    return cudaSuccess;
}

// Dynamic shared memory that launches without raising the attribute: the 48 KB default
// covers static and dynamic shared memory together, and the kernels here declare up to a
// few hundred bytes of static shared memory, so 1 KB is kept for it.
constexpr size_t kSmemNoAttr = 47 * 1024;

cudaError_t ensure_smem_at_least(const void* func, size_t bytes, std::atomic<int>* per_device) {
    if (bytes <= kSmemNoAttr) return cudaSuccess;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::atomic<int>& cur = per_device[dev & 63];
    if (cur.load(std::memory_order_acquire) >= (int)bytes) return cudaSuccess;
    e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) return e;
    int prev = cur.load(std::memory_order_relaxed);
    while (prev < (int)bytes && !cur.compare_exchange_weak(prev, (int)bytes)) {
    }
    return cudaSuccess;
}

cudaError_t ensure_smem_attr(const void* func, size_t bytes, std::atomic<unsigned long long>* done_mask) {
    if (bytes <= kSmemNoAttr) return cudaSuccess;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const unsigned long long bit = 1ull << (dev & 63);
    if (done_mask->load(std::memory_order_acquire) & bit) return cudaSuccess;
    e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) return e;
    done_mask->fetch_or(bit, std::memory_order_acq_rel);
    return cudaSuccess;
}

}  // namespace ffb
