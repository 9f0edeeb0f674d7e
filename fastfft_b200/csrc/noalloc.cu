// Allocation-free 2D padded cross-correlation.
//
// Some callers cannot allocate device memory at the point where they need a
// correlation: code that runs inside a host application whose memory pool owns every
// free byte of the GPU (a framework's caching allocator, or an image-processing program
// that sizes all device buffers at start-up), and steady-state processing loops that must
// not stall, since cudaMalloc and cudaFree synchronise the device.  For them this entry
// point keeps its two intermediate arrays in one fixed, file-scope device array instead
// of a per-plan buffer: nothing is allocated per call or per plan.  The price is that
// every GPU that loads the library holds the array (kNoAllocScratchBytes) until the
// process exits, and that all calls share it.
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/fastfft_capi.h"
#include "kernels_2d.cuh"
#include "launch.h"

namespace ffb {

// Scratch of the allocation-free correlation: row-pass output [kx][y] followed by the
// column-pass output [kx][y'].  24 MiB holds both for a 4096^2 transform with up to 384
// template rows and a 1024-row window (23.1 MB).
constexpr size_t kNoAllocScratchBytes = size_t(24) << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {
std::mutex g_noalloc_mutex;
unsigned char* g_noalloc_ptr[64] = {nullptr};

long long ru(long long v, long long m) { return (v + m - 1) / m * m; }
bool pow2(long long v) { return v >= 1 && (v & (v - 1)) == 0; }

fastfft_status noalloc_fail(fastfft_status st, const std::string& msg) {
    if (st == FASTFFT_ERR_CUDA) cudaGetLastError();
    set_unbound_error(msg.c_str());
    return st;
}

// Device address of the scratch array on the current device (looked up once per device,
// with that device current), plus the one-time twiddle-table set-up for the sizes used.
fastfft_status noalloc_setup(int nx, int ny, unsigned char** scratch) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return noalloc_fail(FASTFFT_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= 64) return noalloc_fail(FASTFFT_ERR_CUDA, "device index out of range");
    {
        std::lock_guard<std::mutex> lock(g_noalloc_mutex);
        if (!g_noalloc_ptr[dev]) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess || p == nullptr)
                return noalloc_fail(FASTFFT_ERR_CUDA,
                                    std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
            g_noalloc_ptr[dev] = static_cast<unsigned char*>(p);
        }
        *scratch = g_noalloc_ptr[dev];
    }
    const float2* tw = nullptr;
    if ((e = twiddles_for(nx, &tw)) != cudaSuccess || (e = twiddles_for(ny, &tw)) != cudaSuccess)
        return noalloc_fail(FASTFFT_ERR_CUDA, std::string("twiddle table: ") + cudaGetErrorString(e));
    return FASTFFT_OK;
}

}  // namespace
}  // namespace ffb

using namespace ffb;

extern "C" fastfft_status fastfft_fwd_image_inv_2d_noalloc(const float* input, int in_x, int in_y,
                                                           const void* image_spectrum, int n_x, int n_y,
                                                           float* output, int out_x, int out_y,
                                                           const fastfft_op* pre_op, const fastfft_op* intra_op,
                                                           const fastfft_op* post_op, void* cuda_stream) {
    if (!input || !image_spectrum || !output)
        return noalloc_fail(FASTFFT_ERR_INVALID_ARGUMENT, "null input, image or output pointer");
    if (!pow2(n_x) || !pow2(n_y) || n_x < kMinN || n_y < kMinN || n_x > kMaxN || n_y > kMaxN)
        return noalloc_fail(FASTFFT_ERR_INVALID_DIMS, "transform sizes must be powers of two in [16, 8192]");
    if (in_x < 1 || in_y < 1 || in_x > n_x || in_y > n_y)
        return noalloc_fail(FASTFFT_ERR_INVALID_DIMS, "template must fit in the transform (1 <= in <= n per axis)");
    if (out_x < 1 || out_y < 1 || out_x > n_x || out_y > n_y)
        return noalloc_fail(FASTFFT_ERR_INVALID_DIMS, "window must fit in the transform (1 <= out <= n per axis)");
    auto bad_op = [](const fastfft_op* op, bool intra) {
        if (!op) return false;
        if (intra) return !(op->kind == FASTFFT_OP_NOOP || op->kind == FASTFFT_OP_CONJ_MUL ||
                             op->kind == FASTFFT_OP_CONJ_MUL_THEN_SCALE);
        return !(op->kind == FASTFFT_OP_NOOP || op->kind == FASTFFT_OP_SCALE);
    };
    if (bad_op(pre_op, false) || bad_op(post_op, false) || bad_op(intra_op, true))
        return noalloc_fail(FASTFFT_ERR_INVALID_ARGUMENT, "unsupported functor kind");
    // scratch layout: [kx][y] row-pass output, then [kx][y'] column-pass output
    const long long kx = n_x / 2 + 1;
    const long long pitch_a = ru(in_y, 4), pitch_b = ru(out_y, 4);
    const long long bytes_a = ru(kx * pitch_a * 8, 256);
    const long long need = bytes_a + kx * pitch_b * 8;
    if (need > (long long)kNoAllocScratchBytes)
        return noalloc_fail(FASTFFT_ERR_UNSUPPORTED,
                            "sizes need " + std::to_string(need) + " bytes of scratch; the allocation-free path has " +
                                std::to_string(kNoAllocScratchBytes) +
                                " ((n_x/2+1) * (round_up(in_y,4) + round_up(out_y,4)) * 8 bytes must fit)");
    unsigned char* scratch = nullptr;
    fastfft_status st = noalloc_setup(n_x, n_y, &scratch);
    if (st != FASTFFT_OK) return st;
    float2* t1 = reinterpret_cast<float2*>(scratch);
    float2* t2 = reinterpret_cast<float2*>(scratch + bytes_a);
    cudaStream_t stream = cuda_stream ? static_cast<cudaStream_t>(cuda_stream) : cudaStreamPerThread;
    const float2* tw = nullptr;
    cudaError_t e;

    // 1. row R2C of the template rows (zero padding x >= in_x implicit) -> t1[kx][y]
    twiddles_for(n_x, &tw);
    RowFwdArgs a;
    std::memset(&a, 0, sizeof(a));
    a.in[0] = input;
    a.n_batch = 1;
    a.in_pitch = 2LL * ((in_x + (in_x % 2 == 0 ? 2 : 1)) / 2);
    a.n_rows = in_y;
    a.L = in_x;
    a.out = t1;
    a.out_pitch = pitch_a;
    a.kmax = (int)kx;
    a.scale = (pre_op && pre_op->kind == FASTFFT_OP_SCALE) ? pre_op->scale : 1.f;
    a.tw = tw;
    if ((e = launch_r2c_rows(n_x, FASTFFT_DTYPE_F32, a, stream)) != cudaSuccess)
        return noalloc_fail(FASTFFT_ERR_CUDA, std::string("r2c row pass: ") + cudaGetErrorString(e));

    // 2. fused column pass: forward (pruned), conj(T) * I, inverse keeping y < out_y -> t2
    twiddles_for(n_y, &tw);
    ColArgs c;
    std::memset(&c, 0, sizeof(c));
    c.in = t1;
    c.in_stride = pitch_a;
    c.L = in_y;
    c.img = image_spectrum;
    c.img_stride = n_y;
    c.out = t2;
    c.out_stride = pitch_b;
    c.W = out_y;
    c.n_cols = (int)kx;
    c.intra_kind = intra_op ? intra_op->kind : FASTFFT_OP_NOOP;
    c.intra_scale = intra_op ? intra_op->scale : 1.f;
    c.in_scale = 1.f;
    c.out_scale = 1.f;
    c.tw = tw;
    c.n_batch = 1;
    if ((e = launch_cols_xcorr(n_y, FASTFFT_DTYPE_C64, c, stream)) != cudaSuccess)
        return noalloc_fail(FASTFFT_ERR_CUDA, std::string("column pass: ") + cudaGetErrorString(e));

    // 3. row C2R keeping x < out_x -> output (pitch 2 * (out_x / 2 + 1))
    twiddles_for(n_x, &tw);
    RowInvArgs r;
    std::memset(&r, 0, sizeof(r));
    r.n_batch = 1;
    r.in = t2;
    r.in_pitch = pitch_b;
    r.n_rows = out_y;
    r.out[0] = output;
    r.out_pitch = 2LL * ((out_x + (out_x % 2 == 0 ? 2 : 1)) / 2);
    r.W = out_x;
    r.scale = (post_op && post_op->kind == FASTFFT_OP_SCALE) ? post_op->scale : 1.f;
    r.tw = tw;
    if ((e = launch_c2r_rows(n_x, FASTFFT_DTYPE_F32, r, stream)) != cudaSuccess)
        return noalloc_fail(FASTFFT_ERR_CUDA, std::string("c2r row pass: ") + cudaGetErrorString(e));
    return FASTFFT_OK;
}
