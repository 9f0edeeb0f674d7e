// C ABI: plan state, dimension validation, buffer sizing and pass dispatch.
//
// Host logic restated from the reference's FourierTransformer
// (include/FastFFT.h:84-732, src/fastfft/FastFFT.cu:58-3379) with status codes in
// place of std::abort().  The kernel sequence per call is chosen here:
//   2D FwdFFT          r2c_rows (N_x, L_y rows)  -> cols FWD (N_y)
//   2D InvFFT          cols INV (N_y, keep W_y)  -> c2r_rows (N_x, keep W_x)
//   2D FwdImageInvFFT  r2c_rows -> cols XCORR (fwd, conj-mul, inv, keep W_y) -> c2r_rows
//   3D FwdFFT          r2c_rows (x) -> cols FWD (z, transposed store) -> cols FWD (y)
//   3D InvFFT          cols INV (y, transposed) -> cols INV (z, transposed) -> c2r_rows (x)
//   3D FwdImageInvFFT  r2c_rows -> cols FWD (z) -> cols XCORR (y) -> cols INV (z) -> c2r_rows
// Intermediate layouts: forward [kx][y][z] then [kz][kx][y]; spectrum [kz][kx][ky];
// inverse [kx][y'][kz] then [kx][z'][y'] (primes: retained window coordinates).
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/fastfft_capi.h"
#include "fft3.cuh"
#include "kernels_xcorr.cuh"
#include "launch.h"
#include "spectrum_ops.h"
#include "plan.h"

using namespace ffb;

// Templates per block of the fused column pass (0: the whole launch's group).  Splitting a
// group of 16 over two blocks per column doubles the blocks of a launch (1538 instead of 769
// at 1536^2, 5.2 instead of 2.6 waves of two blocks per SM), which shortens the last, partly
// empty wave; the image column is then staged twice, from L2.  Measured on B200 at 16
// templates per launch: 7.8 instead of 8.5 us per template at 1536^2, 2.9 instead of 3.7 at
// 1024^2.
#ifndef FFB_XCORR_TPB
#define FFB_XCORR_TPB 8
#endif

// templates that one block of the fused column pass stages for a launch of n at column
// length my; measured best on B200 with 64 per launch: six at 1536 (= 3 * 512; 5.37 instead of
// 5.47 us per template for that pass; 4, 5 and 8 were slower), four at 1024 (1.99 instead of
// 2.06; 6 and 16 were slower), eight elsewhere (at 256: 0.23 against 0.29 with four)
// (fastfft_set_templates_per_block overrides it; the autotuner measures the candidates)
static inline int xcorr_tpb(const fastfft_plan_s* h, int n, long long my) {
    const int per_block = h->tpb_request > 0 ? h->tpb_request
                          : FFB_XCORR_TPB != 8 ? FFB_XCORR_TPB : my == 3 * 512 ? 6 : my == 1024 ? 4 : 8;
    return per_block > 0 && n > per_block ? per_block : n;
}

// Uneven batches: each template correlates at its own exact size class (1), or every
// template at the plan's size (0).
#ifndef FFB_SIZE_CLASSES
#define FFB_SIZE_CLASSES 1
#endif

// Lengths 3 * 2^k for the reduced-size correlation (1), or powers of two only (0).
#ifndef FFB_ENABLE_FFT3
#define FFB_ENABLE_FFT3 1
#endif
// Lengths 5 * 2^k among the reduced-size correlation's lengths (1), or not (0, the default):
// measured on B200 (64 templates per call) the 3 * 2^k length above a 5 * 2^k one is as fast or
// faster although 6/5 as long: 264,767 at 768 against 246,111 templates/s at 640 (128^2
// templates, 512^2 windows), 96,051 at 1536 against 89,653 at 1280 (300^2, 900^2), 23,681 at
// 3072 against 23,809 at 2560 (700^2, 1800^2); the uneven 1024-template batch gains 3.5 %.
// 5 * 2^k lengths run where a plan's own N is one.
#ifndef FFB_ENABLE_FFT5
#define FFB_ENABLE_FFT5 0
#endif
// Lengths 7 * 2^k among the reduced-size correlation's lengths (1), or not (0, the default):
// a 7 * 2^k transform costs far more per point than the power of two above it (measured on
// B200 in the uneven 1024-template batch, whose 384^2 templates with 512^2 windows would
// correlate at 896 instead of 1024: 186,916 instead of 365,798 templates/s), so the
// correlation uses 7 * 2^k lengths only when a plan's own N is one.
#ifndef FFB_ENABLE_FFT7
#define FFB_ENABLE_FFT7 0
#endif

namespace {

const char* kVersion = "fastfft_b200 0.1.0 (sm_100a)";

thread_local std::string g_null_handle_error;

fastfft_status fail(fastfft_plan_s* h, fastfft_status st, const std::string& msg) {
    if (h)
        h->last_error = msg;
    else
        g_null_handle_error = msg;
    return st;
}

fastfft_status cuda_fail(fastfft_plan_s* h, cudaError_t e, const char* where) {
    cudaGetLastError();  // leave no non-sticky error behind for the caller's next CUDA check
    return fail(h, FASTFFT_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

bool is_pow2(long long v) { return v >= 1 && (v & (v - 1)) == 0; }

bool real_dtype(int d) { return d == FASTFFT_DTYPE_F32 || d == FASTFFT_DTYPE_F16 || d == FASTFFT_DTYPE_BF16; }
bool cplx_dtype(int d) { return d == FASTFFT_DTYPE_C64 || d == FASTFFT_DTYPE_C32H || d == FASTFFT_DTYPE_C32BF; }

size_t real_size(int d) { return d == FASTFFT_DTYPE_F32 ? 4 : 2; }

long long round_up(long long v, long long m) { return (v + m - 1) / m * m; }

// ReturnPaddedMemorySize (include/FastFFT.h:363-404): real InputType rows hold w = x/2 + 1
// complex values after the R2C (FFTW pitch 2w); complex InputType rows hold w = x.  The
// count is in scalar components (two per complex value).
long long padded_elems(Dims& d, bool complex_input = false) {
    if (complex_input) {
        d.w = d.x;
        return 2LL * d.x * d.y * d.z;
    }
    const int jump = (d.x % 2 == 0) ? 2 : 1;
    d.w = (d.x + jump) / 2;
    return 2LL * d.w * d.y * d.z;
}

// Spectrum columns kx of a length-n x axis: n/2 + 1 for real input, n for complex input.
long long kx_count(const fastfft_plan_s* h, long long n) { return cplx_dtype(h->input_dtype) ? n : n / 2 + 1; }

// Classify one direction (FastFFT.cu:803-850).  Mixed growth/shrink is rejected.
bool classify(const Dims& in, const Dims& out, SizeChange* sc, std::string* why) {
    const bool any_up = out.x > in.x || out.y > in.y || out.z > in.z;
    const bool any_down = out.x < in.x || out.y < in.y || out.z < in.z;
    if (any_up && any_down) {
        *why = "all dimensions must either increase, decrease or stay the same";
        return false;
    }
    *sc = any_up ? SizeChange::Increase : any_down ? SizeChange::Decrease : SizeChange::NoChange;
    return true;
}

fastfft_status validate(fastfft_plan_s* h) {
    if (!h->fwd_set || !h->inv_set) return fail(h, FASTFFT_ERR_NOT_PLANNED, "forward and inverse plans must both be set");
    if (h->validated) return FASTFFT_OK;
    const Dims &fi = h->fwd_in, &fo = h->fwd_out, &ii = h->inv_in, &io = h->inv_out;
    if (fo.x != ii.x || fo.y != ii.y || fo.z != ii.z)
        return fail(h, FASTFFT_ERR_INVALID_DIMS, "forward output dims must match inverse input dims");
    std::string why;
    if (!classify(fi, fo, &h->fwd_change, &why)) return fail(h, FASTFFT_ERR_INVALID_DIMS, "forward plan: " + why);
    if (!classify(ii, io, &h->inv_change, &why)) return fail(h, FASTFFT_ERR_INVALID_DIMS, "inverse plan: " + why);
    // dimensionality (FastFFT.cu:866-890)
    int dim;
    if (fi.z == 1 && fo.z == 1) {
        if (ii.z != 1 || io.z != 1)
            return fail(h, FASTFFT_ERR_INVALID_DIMS, "fwd/inv dimensionality may not change (z dimension)");
        if (fi.y == 1 && fo.y == 1) return fail(h, FASTFFT_ERR_UNSUPPORTED, "1D transforms are not supported");
        dim = 2;
    } else {
        dim = 3;
        const int m = 512;
        const Dims* all[4] = {&fi, &fo, &ii, &io};
        for (const Dims* d : all)
            if (d->x > m || d->y > m || d->z > m)
                return fail(h, FASTFFT_ERR_INVALID_DIMS, "all dimensions must be <= 512 for 3d transforms");
    }
    if (dim != h->rank) return fail(h, FASTFFT_ERR_INVALID_DIMS, "plan dimensionality does not match the handle rank");
    // transform lengths: powers of two (FastFFT.cu:895-927); real-input 2D plans also take
    // 3 * 2^k with 128 <= 2^k <= 2048 (384 ... 6144), 5 * 2^k with 128 <= 2^k <= 1024
    // (640 ... 5120) and 7 * 2^k with 128 <= 2^k <= 512 (896 ... 3584); every plan, real or
    // complex input, 2D or 3D, any other length in [17, 4096] (chirp-z on a power-of-two FFT;
    // 3D plans stay within 512 per axis); the reference rejects all of these
    const bool wide = dim == 2 && !cplx_dtype(h->input_dtype);
    auto len_ok = [&](long long v) {
        return is_pow2(v) || (wide && v <= 6144 && ffb::is_rp_size((int)v)) || ffb::is_blue_size((int)v);
    };
    const char* lens = wide ? "powers of 2, 3 * 2^k (384 ... 6144), 5 * 2^k (640 ... 5120), 7 * 2^k (896 ... 3584) "
                              "or any other length in [17, 4096]"
                            : "powers of 2 or any other length in [17, 4096] (no 3 * 2^k, 5 * 2^k, 7 * 2^k)";
    if ((!len_ok(fi.x) || !len_ok(fi.y) || !len_ok(fi.z)) && h->fwd_change != SizeChange::Increase)
        return fail(h, FASTFFT_ERR_INVALID_DIMS,
                    std::string("input dimensions must be ") + lens + " unless the forward transform pads");
    if (!len_ok(fo.x) || !len_ok(fo.y) || !len_ok(fo.z))
        return fail(h, FASTFFT_ERR_INVALID_DIMS, std::string("forward output dimensions must be ") + lens);
    if ((!len_ok(io.x) || !len_ok(io.y) || !len_ok(io.z)) && h->inv_change != SizeChange::Decrease)
        return fail(h, FASTFFT_ERR_INVALID_DIMS,
                    std::string("output dimensions must be ") + lens + " unless the inverse transform crops");
    // transform sizes handled by the block FFTs
    const long long nx = std::max(fi.x, fo.x), ny = std::max(fi.y, fo.y), nz = std::max(fi.z, fo.z);
    auto in_range = [](long long n) { return n >= ffb::kMinN && n <= ffb::kMaxN; };
    if (!in_range(nx) || !in_range(ny) || (dim == 3 && !in_range(nz)))
        return fail(h, FASTFFT_ERR_UNSUPPORTED, "transform sizes must be in [16, 8192]");
    if (!in_range(ii.x) || !in_range(ii.y)) return fail(h, FASTFFT_ERR_UNSUPPORTED, "transform sizes must be in [16, 8192]");
    if (h->inv_change != SizeChange::Increase &&
        (h->org_x + io.x > ii.x || h->org_y + io.y > ii.y || h->org_z + io.z > ii.z))
        return fail(h, FASTFFT_ERR_INVALID_DIMS, "inverse output window exceeds the transform (origin + size > N)");
    h->validated = true;
    return FASTFFT_OK;
}

// Internal buffer layout (the reference's buffer_1 / buffer_2 pair):
//   region A: [kx][y] forward row-pass output, pitch pA >= L_y (multiple of 4)
//   region B: [kx][y] inverse column-pass output, pitch pB >= W_y (multiple of 4)
long long pow2_at_least(long long v) {
    long long p = 1;
    while (p < v) p <<= 1;
    return p;
}

// Smallest transform length >= v of the reduced-size correlation: a power of two, or
// 3 * 2^k (kMinP3 <= 2^k <= kMaxP3) when shorter (and 5 * 2^k, 7 * 2^k with FFB_ENABLE_FFT5,
// FFB_ENABLE_FFT7).
long long corr_size_at_least(long long v) {
    long long best = std::max<long long>(ffb::kMinN, pow2_at_least(v));
#if FFB_ENABLE_FFT3
    for (long long p = ffb::kMinP3; p <= ffb::kMaxP3; p *= 2)
        if (3 * p >= v && 3 * p < best) best = 3 * p;
#if FFB_ENABLE_FFT5
    for (long long p = ffb::kMinP3; p <= ffb::kMaxP5; p *= 2)
        if (5 * p >= v && 5 * p < best) best = 5 * p;
#endif
#if FFB_ENABLE_FFT7
    for (long long p = ffb::kMinP3; p <= ffb::kMaxP7; p *= 2)
        if (7 * p >= v && 7 * p < best) best = 7 * p;
#endif
#endif
    return best;
}

void size_buffers(fastfft_plan_s* h) {
    h->prepared_image = nullptr;
    const long long nx_f = std::max(h->fwd_in.x, h->fwd_out.x);
    const long long kx_f = kx_count(h, nx_f);
    const long long kx_i = kx_count(h, h->inv_in.x);
    if (h->rank == 3) {
        // A: forward [kx][y][z] (pitch round_up(Ly*Lz, 4)) / inverse [kx][y'][kz]
        // B: forward [kz][kx][y] / inverse [kx][z'][y'] (pitch round_up(Wz*Wy, 4))
        h->pitch_a = round_up(h->fwd_in.y * h->fwd_in.z, 4);
        h->pitch_b = round_up(h->inv_out.y * h->inv_out.z, 4);
        const long long nz_f = std::max(h->fwd_in.z, h->fwd_out.z);
        const long long a = std::max(kx_f * h->pitch_a, kx_i * h->inv_out.y * h->inv_in.z);
        const long long b = std::max(nz_f * h->fwd_out.w * h->fwd_in.y, kx_i * h->pitch_b);
        h->bytes_a = round_up(a * 8, 256);
        h->bytes_b = round_up(b * 8, 256);
        h->red_ok = false;
        h->bytes_c = 0;
        return;
    }
    h->pitch_a = round_up(h->fwd_in.y, 4);
    h->bytes_a = round_up(kx_f * h->pitch_a * 8, 256);
    h->pitch_b = round_up(h->inv_out.y, 4);
    h->bytes_b = round_up(kx_i * h->pitch_b * 8, 256);
    // reduced-size correlation
    h->red_ok = false;
    h->bytes_c = 0;
    const bool origin0 = h->org_x == 0 && h->org_y == 0 && h->org_z == 0;
    if (origin0 && !cplx_dtype(h->input_dtype) && h->fwd_change != SizeChange::Decrease && h->inv_change == SizeChange::Decrease) {
        const long long nx = h->fwd_out.x, ny = h->fwd_out.y;
        const long long mx = std::min(nx, corr_size_at_least(h->fwd_in.x + h->inv_out.x - 1));
        const long long my = std::min(ny, corr_size_at_least(h->fwd_in.y + h->inv_out.y - 1));
        // (an axis whose correlation would run at the plan's own chirp-z length keeps the
        // whole call at the plan's size: the batched kernels run powers of two and R * 2^k)
        if ((mx < nx || my < ny) && !ffb::is_blue_size((int)mx) && !ffb::is_blue_size((int)my)) {
            h->red_ok = true;
            h->red_mx = mx;
            h->red_my = my;
            const long long stage = std::max((nx / 2 + 1) * my, (mx / 2 + 1) * my) * 8;  // [kx][y] columns
            const long long real = my * (2 * (mx / 2 + 1)) * 4;                          // cropped image rows
            const long long spec = (mx / 2 + 1) * my * 8;                                // reduced spectrum
            h->off_c_real = round_up(stage, 256);
            h->off_c_spec = h->off_c_real + round_up(real, 256);
            // templates per launch: bounded by the shared memory of the fused column kernel
            h->red_batch = h->red_batch_request;
            while (h->red_batch > 1 &&
                   xcorr_cols_smem((int)my, FASTFFT_DTYPE_C64, (int)h->fwd_in.y, xcorr_tpb(h, h->red_batch, my)) >
                       226 * 1024)
                h->red_batch--;
            if (xcorr_cols_smem((int)my, FASTFFT_DTYPE_C64, (int)h->fwd_in.y, 1) > 226 * 1024) {
                h->red_ok = false;
                h->bytes_c = 0;
                return;
            }
            h->red_t1_stride = round_up((mx / 2 + 1) * h->pitch_a, 32);   // complex elements per template
            h->red_t2_stride = round_up((mx / 2 + 1) * h->pitch_b, 32);   // column output [kx][y]
            // one set of template slices per group in flight
            const long long slots = (long long)h->red_batch * (h->pipe_groups > 1 ? 2 : 1);
            h->off_c_t1 = h->off_c_spec + round_up(spec, 256);
            h->off_c_t2 = h->off_c_t1 + slots * h->red_t1_stride * 8;
            h->bytes_c = h->off_c_t2 + slots * h->red_t2_stride * 8;
        }
    }
}

// Side stream and events of the image preparation (created once, outside any stream
// capture since allocate() runs before a plan's first launch; left null on failure).
static void create_prep_stream(fastfft_plan_s* h) {
    if (h->prep_stream || !h->red_ok) return;
    int dev = 0, lo = 0, hi = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetStreamPriorityRange(&lo, &hi) != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    cudaStream_t s = nullptr;
    cudaEvent_t f = nullptr, j = nullptr;
    if (cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, hi) != cudaSuccess ||
        cudaEventCreateWithFlags(&f, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&j, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        if (j) cudaEventDestroy(j);
        if (f) cudaEventDestroy(f);
        if (s) cudaStreamDestroy(s);
        return;
    }
    h->prep_stream = s;
    h->prep_fork = f;
    h->prep_join = j;
    h->prep_device = dev;
}

// Second stream and events of the pipelined template groups (created once, like the
// preparation stream; left null on failure, and the groups then run on `stream` alone).
static void create_pipe_stream(fastfft_plan_s* h) {
    if (h->pipe_stream || !h->red_ok || h->pipe_groups < 2) return;
    cudaStream_t s = nullptr;
    cudaEvent_t f = nullptr, j = nullptr;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&f, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&j, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        if (j) cudaEventDestroy(j);
        if (f) cudaEventDestroy(f);
        if (s) cudaStreamDestroy(s);
        return;
    }
    h->pipe_stream = s;
    h->pipe_fork = f;
    h->pipe_join = j;
}

fastfft_status allocate(fastfft_plan_s* h) {
    size_buffers(h);
    create_prep_stream(h);
    create_pipe_stream(h);
    const size_t need = (size_t)(h->bytes_a + h->bytes_b + h->bytes_c) + 256;
    if (h->buffer && h->buffer_bytes >= need) return FASTFFT_OK;
    if (h->buffer) {
        cudaFree(h->buffer);
        h->buffer = nullptr;
        h->buffer_bytes = 0;
    }
    cudaError_t e = cudaGetDevice(&h->device);
    if (e != cudaSuccess) return cuda_fail(h, e, "cudaGetDevice");
    // A plain (synchronous) allocation: the buffer is then valid on every stream the
    // handle is later pointed at, not only on the stream that allocated it.
    e = cudaMalloc(&h->buffer, need);
    if (e != cudaSuccess) {
        h->buffer = nullptr;
        return fail(h, FASTFFT_ERR_ALLOC, std::string("cudaMalloc of the work buffer failed: ") + cudaGetErrorString(e));
    }
    h->buffer_bytes = need;
    h->dev_err = reinterpret_cast<int*>(static_cast<char*>(h->buffer) + need - 256);
    e = cudaMemset(h->dev_err, 0, sizeof(int));
    if (e != cudaSuccess) return cuda_fail(h, e, "cudaMemset of the status word");
    // the chirp-z tables of the plan's lengths, built here rather than at a first launch
    // that a stream capture may hold
    const long long lens[6] = {std::max(h->fwd_in.x, h->fwd_out.x), std::max(h->fwd_in.y, h->fwd_out.y),
                               std::max(h->fwd_in.z, h->fwd_out.z), h->inv_in.x, h->inv_in.y, h->inv_in.z};
    for (long long n : lens)
        if (ffb::is_blue_size((int)n) && (e = ffb::prepare_blue_tables((int)n)) != cudaSuccess)
            return cuda_fail(h, e, "chirp-z tables");
    return FASTFFT_OK;
}

float scale_of(const fastfft_op* op) { return (op && op->kind == FASTFFT_OP_SCALE) ? op->scale : 1.f; }

bool valid_op(const fastfft_op* op, bool intra) {
    if (!op) return true;
    if (intra) return op->kind == FASTFFT_OP_NOOP || op->kind == FASTFFT_OP_CONJ_MUL || op->kind == FASTFFT_OP_CONJ_MUL_THEN_SCALE;
    return op->kind == FASTFFT_OP_NOOP || op->kind == FASTFFT_OP_SCALE;
}

fastfft_status prepare_call(fastfft_plan_s* h) {
    fastfft_status st = validate(h);
    if (st != FASTFFT_OK) return st;
    if (!h->buffer) {
        st = allocate(h);
        if (st != FASTFFT_OK) return st;
    }
    return FASTFFT_OK;
}

float2* region_a(fastfft_plan_s* h) { return static_cast<float2*>(h->buffer); }
float2* region_b(fastfft_plan_s* h) { return reinterpret_cast<float2*>(static_cast<char*>(h->buffer) + h->bytes_a); }
char* region_c(fastfft_plan_s* h) { return static_cast<char*>(h->buffer) + h->bytes_a + h->bytes_b; }

// Per-pass timing marks (no-ops unless profiling is on).
void prof_begin_call(fastfft_plan_s* h) {
    if (!h->prof_events || h->prof_calls >= h->prof_capacity) return;
    h->prof_mark = 0;
    cudaEventRecord(h->prof_events[h->prof_calls * fastfft_plan_s::kProfMarks], h->stream);
    h->prof_mark = 1;
}
void prof_mark(fastfft_plan_s* h) {
    if (!h->prof_events || h->prof_calls >= h->prof_capacity) return;
    if (h->prof_mark <= 0 || h->prof_mark >= fastfft_plan_s::kProfMarks) return;
    cudaEventRecord(h->prof_events[h->prof_calls * fastfft_plan_s::kProfMarks + h->prof_mark], h->stream);
    h->prof_mark++;
}
void prof_end_call(fastfft_plan_s* h) {
    if (!h->prof_events || h->prof_calls >= h->prof_capacity) return;
    // unused marks of a shorter call repeat the last one (zero-length passes)
    while (h->prof_mark > 0 && h->prof_mark < fastfft_plan_s::kProfMarks) prof_mark(h);
    h->prof_calls++;
    h->prof_mark = 0;
}

// ---------------------------------------------------------------------------
// Stage helpers: one kernel launch each, counted and marked for profiling.
// ---------------------------------------------------------------------------
fastfft_status stage_r2c(fastfft_plan_s* h, int n, int in_dtype, const void* in, long long in_pitch, int n_rows,
                         int rows_y, int rows_z, int L, float2* out, long long out_pitch, int kmax, float scale) {
    const float2* tw = nullptr;
    cudaError_t e = twiddles_for(n, &tw);
    if (e != cudaSuccess) return cuda_fail(h, e, "twiddle table");
    RowFwdArgs a;
    std::memset(&a, 0, sizeof(a));
    a.in[0] = in;
    a.n_batch = 1;
    a.in_pitch = in_pitch;
    a.n_rows = n_rows;
    a.rows_y = rows_y;
    a.rows_z = rows_z;
    a.L = L;
    a.out = out;
    a.out_pitch = out_pitch;
    a.kmax = kmax;
    a.scale = scale;
    a.tw = tw;
    if (cplx_dtype(in_dtype)) {
        a.in_pitch = in_pitch / 2;  // pitches arrive in scalar components; complex rows hold half as many
        e = launch_c2c_rows_fwd(n, in_dtype, a, h->stream);
    } else {
        e = launch_r2c_rows(n, in_dtype, a, h->stream);
    }
    if (e != cudaSuccess) return cuda_fail(h, e, "row pass (forward)");
    h->launches++;
    prof_mark(h);
    return FASTFFT_OK;
}

fastfft_status stage_c2r(fastfft_plan_s* h, int n, const float2* in, long long in_pitch, int n_rows, void* out,
                         long long out_pitch, int W, int X0, float scale, unsigned long long* peaks = nullptr,
                         int peak_slot = 0, unsigned long long* mip = nullptr, int mip_base = 0) {
    const float2* tw = nullptr;
    cudaError_t e = twiddles_for(n, &tw);
    if (e != cudaSuccess) return cuda_fail(h, e, "twiddle table");
    RowInvArgs a;
    std::memset(&a, 0, sizeof(a));
    a.n_batch = 1;
    a.in = in;
    a.in_pitch = in_pitch;
    a.n_rows = n_rows;
    a.out[0] = out;
    a.out_pitch = out_pitch;
    a.W = W;
    a.X0 = X0;
    a.scale = scale;
    a.tw = tw;
    a.peaks = peaks;
    a.peaks_only = ((peaks != nullptr || mip != nullptr) && out == nullptr);
    a.peak_slot[0] = peak_slot;
    a.mip = mip;
    a.mip_base = mip_base;
    if (cplx_dtype(h->output_dtype)) {
        if (peaks || mip) return fail(h, FASTFFT_ERR_UNSUPPORTED, "peak search and projection need real output");
        a.out_pitch = out_pitch / 2;  // pitches arrive in scalar components
        e = launch_c2c_rows_inv(n, h->output_dtype, a, h->stream);
    } else {
        e = launch_c2r_rows(n, h->output_dtype, a, h->stream);
    }
    if (e != cudaSuccess) return cuda_fail(h, e, "row pass (inverse)");
    h->launches++;
    prof_mark(h);
    return FASTFFT_OK;
}

// Column arguments with the plain layout (column c at c * in_stride / c * out_stride).
ColArgs col_args(const void* in, long long in_stride, int L, void* out, long long out_stride, int W, int n_cols) {
    ColArgs c;
    std::memset(&c, 0, sizeof(c));
    c.in = in;
    c.in_stride = in_stride;
    c.L = L;
    c.out = out;
    c.out_stride = out_stride;
    c.W = W;
    c.n_cols = n_cols;
    c.in_scale = 1.f;
    c.out_scale = 1.f;
    c.intra_scale = 1.f;
    c.n_batch = 1;
    return c;
}

enum StageMode { ST_FWD, ST_INV, ST_XCORR };

// dtype: the spectrum's storage for ST_FWD (written), the input's for ST_INV, the image's for
// ST_XCORR
fastfft_status stage_cols(fastfft_plan_s* h, int n, StageMode mode, int dtype, ColArgs& c) {
    const float2* tw = nullptr;
    cudaError_t e = twiddles_for(n, &tw);
    if (e != cudaSuccess) return cuda_fail(h, e, "twiddle table");
    c.tw = tw;
    c.err = h->dev_err;
    if (mode == ST_FWD)
        e = launch_cols_fwd(n, dtype, c, h->stream);
    else if (mode == ST_INV)
        e = launch_cols_inv(n, dtype, c, h->stream);
    else
        e = launch_cols_xcorr(n, dtype, c, h->stream);
    if (e != cudaSuccess) return cuda_fail(h, e, mode == ST_XCORR ? "cross-correlation column pass" : "column pass");
    h->launches++;
    prof_mark(h);
    return FASTFFT_OK;
}

#define FFB_TRY(x)                               \
    do {                                         \
        fastfft_status st_ = (x);                \
        if (st_ != FASTFFT_OK) return st_;       \
    } while (0)

// ---------------------------------------------------------------------------
// Transform sequences
// ---------------------------------------------------------------------------
fastfft_status seq_fwd(fastfft_plan_s* h, const void* in, void* out, float pre_scale) {
    const Dims &fi = h->fwd_in, &fo = h->fwd_out;
    const int nx = (int)std::max(fi.x, fo.x), ny = (int)std::max(fi.y, fo.y), nz = (int)std::max(fi.z, fo.z);
    const int kmax = (int)fo.w;
    if (h->rank == 2) {
        FFB_TRY(stage_r2c(h, nx, h->input_dtype, in, 2LL * fi.w, (int)fi.y, (int)fi.y, 1, (int)fi.x, region_a(h),
                          h->pitch_a, kmax, pre_scale));
        ColArgs c = col_args(region_a(h), h->pitch_a, (int)fi.y, out, fo.y, (int)fo.y, kmax);
        c.out_scale = h->spec_scale;
        return stage_cols(h, ny, ST_FWD, h->spec_dtype, c);
    }
    const long long ly = fi.y, lz = fi.z;
    // x: rows (y, z) -> A[kx][y][z]
    FFB_TRY(stage_r2c(h, nx, h->input_dtype, in, 2LL * fi.w, (int)(ly * lz), (int)ly, (int)lz, (int)fi.x, region_a(h),
                      h->pitch_a, kmax, pre_scale));
    // z: columns (kx, y) -> B[kz][kx][y]
    ColArgs cz = col_args(region_a(h), h->pitch_a, (int)lz, region_b(h), 1, (int)fo.z, (int)(kmax * ly));
    cz.in_div = (int)ly;
    cz.in_stride2 = lz;
    cz.out_elem_stride = kmax * ly;
    FFB_TRY(stage_cols(h, nz, ST_FWD, FASTFFT_DTYPE_C64, cz));
    // y: columns (kz, kx) -> spectrum [kz][kx][ky]
    ColArgs cy = col_args(region_b(h), ly, (int)ly, out, fo.y, (int)fo.y, (int)(fo.z * kmax));
    cy.out_scale = h->spec_scale;
    return stage_cols(h, ny, ST_FWD, h->spec_dtype, cy);
}

// Inverse from a complex spectrum `in` (dtype in_dtype) of the inverse-input size.
fastfft_status seq_inv(fastfft_plan_s* h, const void* in, int in_dtype, void* out, float post_scale) {
    const Dims &ii = h->inv_in, &io = h->inv_out;
    const int nx = (int)ii.x, ny = (int)ii.y, nz = (int)ii.z;
    const int kw = (int)kx_count(h, nx);
    if (h->rank == 2) {
        ColArgs c = col_args(in, ny, ny, region_b(h), h->pitch_b, (int)io.y, kw);
        c.W0 = (int)h->org_y;
        FFB_TRY(stage_cols(h, ny, ST_INV, in_dtype, c));
        return stage_c2r(h, nx, region_b(h), h->pitch_b, (int)io.y, out, 2LL * io.w, (int)io.x, (int)h->org_x,
                         post_scale);
    }
    const long long wy = io.y, wz = io.z;
    // y: columns c = kx * Nz + kz -> A[kx][y'][kz]
    ColArgs cy = col_args(in, ny, ny, region_a(h), wy * nz, (int)wy, (int)(kw * nz));
    cy.in_div = nz;
    cy.in_stride2 = (long long)kw * ny;
    cy.out_div = nz;
    cy.out_stride2 = 1;
    cy.out_elem_stride = nz;
    cy.W0 = (int)h->org_y;
    FFB_TRY(stage_cols(h, ny, ST_INV, in_dtype, cy));
    // z: columns c = kx * Wy + y' -> B[kx][z'][y']
    ColArgs cz = col_args(region_a(h), nz, nz, region_b(h), h->pitch_b, (int)wz, (int)(kw * wy));
    cz.out_div = (int)wy;
    cz.out_stride2 = 1;
    cz.out_elem_stride = wy;
    cz.W0 = (int)h->org_z;
    FFB_TRY(stage_cols(h, nz, ST_INV, FASTFFT_DTYPE_C64, cz));
    // x: rows r = z' * Wy + y'
    return stage_c2r(h, nx, region_b(h), h->pitch_b, (int)(wz * wy), out, 2LL * io.w, (int)io.x, (int)h->org_x,
                     post_scale);
}

// 2D size-N fused correlation of one template of size (lx, ly) <= the plan's input size.
fastfft_status seq_xcorr_sized(fastfft_plan_s* h, const void* in, int lx, int ly, const void* img, void* out,
                               float pre_scale, const fastfft_op* intra_op, float post_scale,
                               unsigned long long* peaks = nullptr, int peak_slot = 0,
                               unsigned long long* mip = nullptr, int mip_base = 0) {
    const Dims &fo = h->fwd_out, &io = h->inv_out;
    const int nx = (int)fo.x, ny = (int)fo.y;
    const int kw = (int)kx_count(h, nx);
    const long long pitch = cplx_dtype(h->input_dtype) ? 2LL * lx : 2LL * ((lx + (lx % 2 == 0 ? 2 : 1)) / 2);
    FFB_TRY(stage_r2c(h, nx, h->input_dtype, in, pitch, ly, ly, 1, lx, region_a(h), h->pitch_a, kw, pre_scale));
    ColArgs c = col_args(region_a(h), h->pitch_a, ly, region_b(h), h->pitch_b, (int)io.y, kw);
    c.img = img;
    c.img_stride = ny;
    c.intra_kind = intra_op ? intra_op->kind : FASTFFT_OP_NOOP;
    c.intra_scale = intra_op ? intra_op->scale : 1.f;
    c.W0 = (int)h->org_y;
    FFB_TRY(stage_cols(h, ny, ST_XCORR, h->image_dtype, c));
    return stage_c2r(h, nx, region_b(h), h->pitch_b, (int)io.y, out, 2LL * io.w, (int)io.x, (int)h->org_x,
                     post_scale, peaks, peak_slot, mip, mip_base);
}

// Size-N fused correlation of one template (forward increase or no change).
fastfft_status seq_xcorr(fastfft_plan_s* h, const void* in, const void* img, void* out, float pre_scale,
                         const fastfft_op* intra_op, float post_scale) {
    const Dims &fi = h->fwd_in, &fo = h->fwd_out, &io = h->inv_out;
    const int nx = (int)fo.x, ny = (int)fo.y, nz = (int)fo.z;
    const int kw = (int)kx_count(h, nx);
    const int ikind = intra_op ? intra_op->kind : FASTFFT_OP_NOOP;
    const float iscale = intra_op ? intra_op->scale : 1.f;
    if (h->rank == 2) {
        FFB_TRY(stage_r2c(h, nx, h->input_dtype, in, 2LL * fi.w, (int)fi.y, (int)fi.y, 1, (int)fi.x, region_a(h),
                          h->pitch_a, kw, pre_scale));
        ColArgs c = col_args(region_a(h), h->pitch_a, (int)fi.y, region_b(h), h->pitch_b, (int)io.y, kw);
        c.img = img;
        c.img_stride = ny;
        c.intra_kind = ikind;
        c.intra_scale = iscale;
        c.W0 = (int)h->org_y;
        FFB_TRY(stage_cols(h, ny, ST_XCORR, h->image_dtype, c));
        return stage_c2r(h, nx, region_b(h), h->pitch_b, (int)io.y, out, 2LL * io.w, (int)io.x, (int)h->org_x,
                         post_scale);
    }
    const long long ly = fi.y, lz = fi.z, wy = io.y, wz = io.z;
    FFB_TRY(stage_r2c(h, nx, h->input_dtype, in, 2LL * fi.w, (int)(ly * lz), (int)ly, (int)lz, (int)fi.x, region_a(h),
                      h->pitch_a, kw, pre_scale));
    ColArgs cz = col_args(region_a(h), h->pitch_a, (int)lz, region_b(h), 1, nz, (int)(kw * ly));
    cz.in_div = (int)ly;
    cz.in_stride2 = lz;
    cz.out_elem_stride = (long long)kw * ly;
    FFB_TRY(stage_cols(h, nz, ST_FWD, FASTFFT_DTYPE_C64, cz));
    // y: columns c = kz * kw + kx (B layout); conj-multiply against image column c; inverse;
    // keep y' -> A[kx][y'][kz]
    ColArgs cy = col_args(region_b(h), ly, (int)ly, region_a(h), 1, (int)wy, nz * kw);
    cy.img = img;
    cy.img_stride = ny;
    cy.intra_kind = ikind;
    cy.intra_scale = iscale;
    cy.out_div = kw;
    cy.out_stride2 = wy * nz;
    cy.out_elem_stride = nz;
    cy.W0 = (int)h->org_y;
    FFB_TRY(stage_cols(h, ny, ST_XCORR, h->image_dtype, cy));
    ColArgs ci = col_args(region_a(h), nz, nz, region_b(h), h->pitch_b, (int)wz, (int)(kw * wy));
    ci.out_div = (int)wy;
    ci.out_stride2 = 1;
    ci.out_elem_stride = wy;
    ci.W0 = (int)h->org_z;
    FFB_TRY(stage_cols(h, nz, ST_INV, FASTFFT_DTYPE_C64, ci));
    return stage_c2r(h, nx, region_b(h), h->pitch_b, (int)(wz * wy), out, 2LL * io.w, (int)io.x, (int)h->org_x,
                     post_scale);
}

}  // namespace

namespace ffb {
// Message for fastfft_last_error(NULL) from entry points that take no handle.
void set_unbound_error(const char* msg) { g_null_handle_error = msg; }
}  // namespace ffb

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

fastfft_status fastfft_create(fastfft_handle* out, int compute_dtype, int input_dtype, int image_dtype, int rank) {
    if (!out) return fail(nullptr, FASTFFT_ERR_INVALID_ARGUMENT, "null handle pointer");
    *out = nullptr;
    if (compute_dtype != FASTFFT_DTYPE_F32) return fail(nullptr, FASTFFT_ERR_UNSUPPORTED, "compute type must be float");
    if (!real_dtype(input_dtype) && !cplx_dtype(input_dtype))
        return fail(nullptr, FASTFFT_ERR_UNSUPPORTED, "input type must be f32, f16, bf16, c64, c32h or c32bf");
    if (!cplx_dtype(image_dtype)) return fail(nullptr, FASTFFT_ERR_UNSUPPORTED, "image type must be complex (c64, c32h, c32bf)");
    if (rank != 2 && rank != 3) return fail(nullptr, FASTFFT_ERR_UNSUPPORTED, "only 2D and 3D FFTs are supported");
    fastfft_plan_s* h = new (std::nothrow) fastfft_plan_s();
    if (!h) return fail(nullptr, FASTFFT_ERR_ALLOC, "out of host memory");
    h->compute_dtype = compute_dtype;
    h->input_dtype = input_dtype;
    h->output_dtype = input_dtype;
    h->image_dtype = image_dtype;
    h->rank = rank;
    h->stream = cudaStreamPerThread;
    *out = h;
    return FASTFFT_OK;
}

fastfft_status fastfft_destroy(fastfft_handle h) {
    if (!h) return FASTFFT_OK;
    if (h->radial_scratch) {
        cudaStreamSynchronize(h->stream);
        cudaFree(h->radial_scratch);
    }
    if (h->prep_stream) {
        cudaStreamSynchronize(h->prep_stream);
        cudaEventDestroy(h->prep_fork);
        cudaEventDestroy(h->prep_join);
        cudaStreamDestroy(h->prep_stream);
    }
    if (h->pipe_stream) {
        cudaStreamSynchronize(h->pipe_stream);
        cudaEventDestroy(h->pipe_fork);
        cudaEventDestroy(h->pipe_join);
        cudaStreamDestroy(h->pipe_stream);
    }
    if (h->buffer) {
        cudaStreamSynchronize(h->stream);
        cudaFree(h->buffer);
    }
    if (h->prof_events) {
        for (int i = 0; i < h->prof_capacity * fastfft_plan_s::kProfMarks; i++) cudaEventDestroy(h->prof_events[i]);
        delete[] h->prof_events;
    }
    delete h;
    return FASTFFT_OK;
}

static fastfft_status set_plan(fastfft_handle h, bool fwd, size_t ix, size_t iy, size_t iz, size_t ox, size_t oy,
                               size_t oz, int is_padded) {
    if (!h) return fail(nullptr, FASTFFT_ERR_INVALID_ARGUMENT, "null handle");
    if (ix == 0 || iy == 0 || iz == 0 || ox == 0 || oy == 0 || oz == 0)
        return fail(h, FASTFFT_ERR_INVALID_DIMS, "logical dimensions must be > 0");
    const size_t lim = 1u << 15;
    if (ix >= lim || iy >= lim || iz >= lim || ox >= lim || oy >= lim || oz >= lim)
        return fail(h, FASTFFT_ERR_INVALID_DIMS, "logical dimensions must be < 32768");
    if (!is_padded) return fail(h, FASTFFT_ERR_UNSUPPORTED, "input arrays must be FFTW padded");
    Dims in{(long long)ix, (long long)iy, (long long)iz, 0}, outd{(long long)ox, (long long)oy, (long long)oz, 0};
    const bool cx = cplx_dtype(h->input_dtype);
    const long long n_in = padded_elems(in, cx), n_out = padded_elems(outd, cx);
    if (fwd) {
        h->fwd_in = in;
        h->fwd_out = outd;
        h->input_mem = n_in;
        h->fwd_out_mem = n_out;
        h->fwd_set = true;
    } else {
        h->inv_in = in;
        h->inv_out = outd;
        h->inv_out_mem = n_out;
        h->inv_set = true;
    }
    h->compute_mem = std::max(h->compute_mem, std::max(n_in, n_out));
    h->validated = false;
    if (h->fwd_set && h->inv_set) {
        fastfft_status st = validate(h);
        if (st != FASTFFT_OK) return st;
        size_buffers(h);
        // AllocateBufferMemory happens on the second plan call, as in the reference.
        // Without a visible CUDA device (host-only use of the plan logic) the
        // allocation is deferred to the first transform, which then reports it.
        int n_dev = 0;
        if (cudaGetDeviceCount(&n_dev) != cudaSuccess || n_dev == 0) {
            cudaGetLastError();
            return FASTFFT_OK;
        }
        return allocate(h);
    }
    return FASTFFT_OK;
}

fastfft_status fastfft_set_forward_plan(fastfft_handle h, size_t ix, size_t iy, size_t iz, size_t ox, size_t oy,
                                        size_t oz, int is_padded) {
    return set_plan(h, true, ix, iy, iz, ox, oy, oz, is_padded);
}

fastfft_status fastfft_set_inverse_plan(fastfft_handle h, size_t ix, size_t iy, size_t iz, size_t ox, size_t oy,
                                        size_t oz, int is_padded) {
    return set_plan(h, false, ix, iy, iz, ox, oy, oz, is_padded);
}

fastfft_status fastfft_set_stream(fastfft_handle h, void* cuda_stream) {
    if (!h) return fail(nullptr, FASTFFT_ERR_INVALID_ARGUMENT, "null handle");
    cudaStream_t s = cuda_stream ? static_cast<cudaStream_t>(cuda_stream) : cudaStreamPerThread;
    if (s != h->stream) h->prepared_image = nullptr;  // a preparation may still run on the old stream
    h->stream = s;
    return FASTFFT_OK;
}

fastfft_status fastfft_set_spectrum_output(fastfft_handle h, int dtype, float scale) {
    if (!h) return fail(nullptr, FASTFFT_ERR_INVALID_ARGUMENT, "null handle");
    if (dtype != FASTFFT_DTYPE_C64 && dtype != FASTFFT_DTYPE_C32H && dtype != FASTFFT_DTYPE_C32BF)
        return fail(h, FASTFFT_ERR_INVALID_ARGUMENT, "spectrum storage must be a complex dtype");
    if (!(scale == scale) || scale == 0.f || scale > 3.0e38f || scale < -3.0e38f)
        return fail(h, FASTFFT_ERR_INVALID_ARGUMENT, "spectrum scale must be finite and non-zero");
    h->spec_dtype = dtype;
    h->spec_scale = scale;
    return FASTFFT_OK;
}

static fastfft_status radial_checks(fastfft_handle h, const void* a, const void* b, int n, int n_bins) {
    if (!h) return fail(nullptr, FASTFFT_ERR_INVALID_ARGUMENT, "null handle");
    if (!a || !b) return fail(h, FASTFFT_ERR_INVALID_ARGUMENT, "null spectrum, filter or output pointer");
    if (n < 2 || n > 8192 || (n & 1)) return fail(h, FASTFFT_ERR_INVALID_DIMS, "n must be even and in [2, 8192]");
    if (n_bins < 1 || n_bins > 8192) return fail(h, FASTFFT_ERR_INVALID_ARGUMENT, "n_bins must be in [1, 8192]");
    return FASTFFT_OK;
}

fastfft_status fastfft_radial_power(fastfft_handle h, const void* spectrum, int n, float* power, int n_bins) {
    FFB_TRY(radial_checks(h, spectrum, power, n, n_bins));
    if (h->radial_scratch_bins < n_bins) {
        if (h->radial_scratch) {
            cudaStreamSynchronize(h->stream);
            cudaFree(h->radial_scratch);
            h->radial_scratch = nullptr;
            h->radial_scratch_bins = 0;
        }
        cudaError_t e = cudaMalloc(&h->radial_scratch, (size_t)2 * n_bins * sizeof(double));
        if (e != cudaSuccess) {
            h->radial_scratch = nullptr;
            return fail(h, FASTFFT_ERR_ALLOC, std::string("cudaMalloc of the radial work array: ") + cudaGetErrorString(e));
        }
        h->radial_scratch_bins = n_bins;
    }
    RadialArgs a;
    std::memset(&a, 0, sizeof(a));
    a.in = static_cast<const float2*>(spectrum);
    a.n = n;
    a.n_bins = n_bins;
    a.sums = h->radial_scratch;
    a.weights = h->radial_scratch + n_bins;
    const cudaError_t e = launch_radial_power(a, power, h->stream);
    if (e != cudaSuccess) return cuda_fail(h, e, "radial power");
    h->launches += 2;
    return FASTFFT_OK;
}

fastfft_status fastfft_apply_radial_filter(fastfft_handle h, const void* in, void* out, int n, const float* filter,
                                           int n_bins) {
    FFB_TRY(radial_checks(h, in, filter, n, n_bins));
    if (!out) return fail(h, FASTFFT_ERR_INVALID_ARGUMENT, "null output pointer");
    if (out == in && h->spec_dtype != FASTFFT_DTYPE_C64)
        return fail(h, FASTFFT_ERR_INVALID_ARGUMENT, "in-place filtering needs complex64 storage");
    RadialArgs a;
    std::memset(&a, 0, sizeof(a));
    a.in = static_cast<const float2*>(in);
    a.out = out;
    a.n = n;
    a.n_bins = n_bins;
    a.filter = filter;
    a.scale = h->spec_scale;
    const cudaError_t e = launch_radial_filter(h->spec_dtype, a, h->stream);
    if (e != cudaSuccess) return cuda_fail(h, e, "radial filter");
    h->launches++;
    return FASTFFT_OK;
}

fastfft_status fastfft_set_tensor_core_dft(fastfft_handle h, int enable) {
    if (!h) return fail(nullptr, FASTFFT_ERR_INVALID_ARGUMENT, "null handle");
    h->tc_dft = enable != 0;
    return FASTFFT_OK;
}

fastfft_status fastfft_tensor_core_dft_active(fastfft_handle h, int* active) {
    if (!h || !active) return fail(h, FASTFFT_ERR_INVALID_ARGUMENT, "null handle or output pointer");
    *active = 0;
    fastfft_status st = validate(h);
    if (st != FASTFFT_OK) return st;
    fastfft_plan_s sized = *h;  // the buffer plan of the current settings, without touching h
    size_buffers(&sized);
    *active = (h->tc_dft && sized.red_ok && !h->force_full_size && sized.red_my == 3 * 512 && h->fwd_in.y <= 512) ? 1 : 0;
    return FASTFFT_OK;
}

fastfft_status fastfft_set_image_reuse(fastfft_handle h, int enable) {
    if (!h) return fail(nullptr, FASTFFT_ERR_INVALID_ARGUMENT, "null handle");
    h->image_reuse = enable != 0;
    h->prepared_image = nullptr;
    return FASTFFT_OK;
}

fastfft_status fastfft_set_inverse_output_origin(fastfft_handle h, size_t ox, size_t oy, size_t oz) {
    if (!h) return fail(nullptr, FASTFFT_ERR_INVALID_ARGUMENT, "null handle");
    if (ox >= (1u << 15) || oy >= (1u << 15) || oz >= (1u << 15))
        return fail(h, FASTFFT_ERR_INVALID_DIMS, "origin out of range");
    h->org_x = (long long)ox;
    h->org_y = (long long)oy;
    h->org_z = (long long)oz;
    h->validated = false;
    if (h->fwd_set && h->inv_set) {
        fastfft_status st = validate(h);
        if (st != FASTFFT_OK) return st;
        const size_t before = h->buffer_bytes;
        size_buffers(h);
        if (h->buffer && (size_t)(h->bytes_a + h->bytes_b + h->bytes_c) + 256 > before) {
            cudaFree(h->buffer);
            h->buffer = nullptr;
            h->buffer_bytes = 0;
        }
    }
    return FASTFFT_OK;
}

fastfft_status fastfft_set_output_dtype(fastfft_handle h, int dtype) {
    if (!h) return fail(nullptr, FASTFFT_ERR_INVALID_ARGUMENT, "null handle");
    if (cplx_dtype(h->input_dtype) ? !cplx_dtype(dtype) : !real_dtype(dtype))
        return fail(h, FASTFFT_ERR_INVALID_ARGUMENT,
                    cplx_dtype(h->input_dtype) ? "output dtype of a complex-input plan must be complex (c64, c32h, c32bf)"
                                               : "output dtype must be real (f32, f16, bf16)");
    h->output_dtype = dtype;
    return FASTFFT_OK;
}

fastfft_status fastfft_fwd(fastfft_handle h, const void* input, void* output, const fastfft_op* pre_op,
                           const fastfft_op* intra_op) {
    if (!h) return fail(nullptr, FASTFFT_ERR_INVALID_ARGUMENT, "null handle");
    if (!input) return fail(h, FASTFFT_ERR_INVALID_ARGUMENT, "null input pointer");
    if (!valid_op(pre_op, false)) return fail(h, FASTFFT_ERR_INVALID_ARGUMENT, "pre-op must be NOOP or SCALE");
    if (intra_op && intra_op->kind != FASTFFT_OP_NOOP)
        return fail(h, FASTFFT_ERR_UNSUPPORTED, "FwdFFT takes no intra-op (use FwdImageInvFFT)");
    fastfft_status st = prepare_call(h);
    if (st != FASTFFT_OK) return st;
    void* out = output ? output : const_cast<void*>(input);
    prof_begin_call(h);
    st = seq_fwd(h, input, out, scale_of(pre_op));
    prof_end_call(h);
    return st;
}

fastfft_status fastfft_inv(fastfft_handle h, const void* input, void* output, const fastfft_op* intra_op,
                           const fastfft_op* post_op) {
    if (!h) return fail(nullptr, FASTFFT_ERR_INVALID_ARGUMENT, "null handle");
    if (!input) return fail(h, FASTFFT_ERR_INVALID_ARGUMENT, "null input pointer");
    if (!valid_op(post_op, false)) return fail(h, FASTFFT_ERR_INVALID_ARGUMENT, "post-op must be NOOP or SCALE");
    if (intra_op && intra_op->kind != FASTFFT_OP_NOOP)
        return fail(h, FASTFFT_ERR_UNSUPPORTED, "InvFFT takes no intra-op (use FwdImageInvFFT)");
    fastfft_status st = prepare_call(h);
    if (st != FASTFFT_OK) return st;
    if (h->inv_change == SizeChange::Increase)
        return fail(h, FASTFFT_ERR_UNSUPPORTED, "inverse size increase is not supported");
    void* out = output ? output : const_cast<void*>(input);
    prof_begin_call(h);
    st = seq_inv(h, input, FASTFFT_DTYPE_C64, out, scale_of(post_op));
    prof_end_call(h);
    return st;
}

static fastfft_status xcorr_checks(fastfft_handle h, const fastfft_op* pre_op, const fastfft_op* intra_op,
                                   const fastfft_op* post_op) {
    if (!valid_op(pre_op, false)) return fail(h, FASTFFT_ERR_INVALID_ARGUMENT, "pre-op must be NOOP or SCALE");
    if (!valid_op(post_op, false)) return fail(h, FASTFFT_ERR_INVALID_ARGUMENT, "post-op must be NOOP or SCALE");
    if (!valid_op(intra_op, true))
        return fail(h, FASTFFT_ERR_INVALID_ARGUMENT, "intra-op must be NOOP, CONJ_MUL or CONJ_MUL_THEN_SCALE");
    fastfft_status st = prepare_call(h);
    if (st != FASTFFT_OK) return st;
    if (h->fwd_change == SizeChange::Decrease)
        return fail(h, FASTFFT_ERR_UNSUPPORTED, "cross-correlation with a forward size decrease is not supported");
    if (h->inv_change == SizeChange::Increase)
        return fail(h, FASTFFT_ERR_UNSUPPORTED, "cross-correlation with an inverse size increase is not supported");
    return FASTFFT_OK;
}

static fastfft_status xcorr_many(fastfft_handle h, int n, const void* const* inputs, const int* dims,
                                 const void* const* image_spectra, void* const* outputs, const fastfft_op* pre_op,
                                 const fastfft_op* intra_op, const fastfft_op* post_op,
                                 unsigned long long* peaks = nullptr, unsigned long long* mip = nullptr,
                                 int mip_base = 0);

static fastfft_status xcorr_one(fastfft_handle h, const void* input, const void* image_spectrum, void* out,
                                const fastfft_op* pre_op, const fastfft_op* intra_op, const fastfft_op* post_op) {
    prof_begin_call(h);
    fastfft_status st = seq_xcorr(h, input, image_spectrum, out, scale_of(pre_op), intra_op, scale_of(post_op));
    prof_end_call(h);
    return st;
}

// Prepare the reduced spectrum of one image: C2R of the size-N spectrum keeping
// [0, My) x [0, Mx), R2C at size M, scaled by 1/(Mx*My) so that the size-M correlation
// carries the same Nx*Ny factor as the size-N one.
static fastfft_status red_prepare_image_on(fastfft_handle h, const void* image_spectrum, int mx, int my);

// Wait on `stream` (the plan's stream or, inside a pipelined call, the pipe stream) for a
// preparation still running on the side stream.
static fastfft_status join_prep(fastfft_handle h) {
    const bool pipe = h->pipe_stream && h->stream == h->pipe_stream;
    bool& pending = pipe ? h->prep_join_pending_pipe : h->prep_join_pending;
    if (!pending) return FASTFFT_OK;
    pending = false;
    const cudaError_t e = cudaStreamWaitEvent(h->stream, h->prep_join, 0);
    return e == cudaSuccess ? FASTFFT_OK : cuda_fail(h, e, "joining the image preparation");
}

static fastfft_status red_prepare_image(fastfft_handle h, const void* image_spectrum, int mx, int my) {
    if (h->image_reuse && h->prepared_image == image_spectrum && h->prepared_mx == mx && h->prepared_my == my)
        return FASTFFT_OK;
    FFB_TRY(join_prep(h));
    int dev = -1;
    const bool side = h->prep_stream && cudaGetDevice(&dev) == cudaSuccess && dev == h->prep_device;
    if (!side) return red_prepare_image_on(h, image_spectrum, mx, my);
    // fork after everything already on `stream` (earlier fused passes still read region C's
    // spectrum), prepare on the side stream, record the join for the next column pass
    cudaError_t e = cudaEventRecord(h->prep_fork, h->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(h->prep_stream, h->prep_fork, 0);
    // with pipelined groups the pipe stream may still read the previous spectrum too (only
    // once forked in this call: its earlier work is already ordered before `stream`)
    if (e == cudaSuccess && h->pipe_active) {
        e = cudaEventRecord(h->pipe_join, h->pipe_stream);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(h->prep_stream, h->pipe_join, 0);
    }
    if (e != cudaSuccess) return cuda_fail(h, e, "forking the image preparation");
    cudaStream_t main_stream = h->stream;
    h->stream = h->prep_stream;
    fastfft_status st = red_prepare_image_on(h, image_spectrum, mx, my);
    h->stream = main_stream;
    e = cudaEventRecord(h->prep_join, h->prep_stream);
    if (e != cudaSuccess) {
        // the side stream's work cannot be joined through the event: wait for it here
        cudaStreamSynchronize(h->prep_stream);
        return st != FASTFFT_OK ? st : cuda_fail(h, e, "joining the image preparation");
    }
    h->prep_join_pending = true;
    h->prep_join_pending_pipe = h->pipe_groups > 1 && h->pipe_stream;
    if (st != FASTFFT_OK) join_prep(h);
    return st;
}

static fastfft_status red_prepare_image_on(fastfft_handle h, const void* image_spectrum, int mx, int my) {
    h->prepared_image = nullptr;
    const int nx = (int)h->fwd_out.x, ny = (int)h->fwd_out.y;
    char* c = region_c(h);
    float2* stage = reinterpret_cast<float2*>(c);
    float* crop = reinterpret_cast<float*>(c + h->off_c_real);
    float2* spec = reinterpret_cast<float2*>(c + h->off_c_spec);
    const long long crop_pitch = 2LL * (mx / 2 + 1);
    const int saved_out = h->output_dtype;
    h->output_dtype = FASTFFT_DTYPE_F32;  // the cropped image is an internal FP32 array
    // 1. inverse along y keeping y < My: stage[kx][y]
    ColArgs c1 = col_args(image_spectrum, ny, ny, stage, my, my, nx / 2 + 1);
    fastfft_status st = stage_cols(h, ny, ST_INV, h->image_dtype, c1);
    // 2. C2R along x keeping x < Mx: crop[y][x]
    if (st == FASTFFT_OK) st = stage_c2r(h, nx, stage, my, my, crop, crop_pitch, mx, 0, 1.f);
    h->output_dtype = saved_out;
    if (st != FASTFFT_OK) return st;
    // 3. R2C along x at size Mx: stage[kx][y]
    FFB_TRY(stage_r2c(h, mx, FASTFFT_DTYPE_F32, crop, crop_pitch, my, my, 1, mx, stage, my, mx / 2 + 1, 1.f));
    // 4. forward along y at size My, scaled by 1/(Mx My): spec[kx][ky]
    ColArgs c4 = col_args(stage, my, my, spec, my, my, mx / 2 + 1);
    c4.out_scale = 1.f / ((float)mx * (float)my);
    fastfft_status st4 = stage_cols(h, my, ST_FWD, FASTFFT_DTYPE_C64, c4);
    if (st4 == FASTFFT_OK && h->image_reuse) {
        h->prepared_image = image_spectrum;
        h->prepared_mx = mx;
        h->prepared_my = my;
    }
    return st4;
}

// Up to kMaxBatch templates through the reduced-size correlation against the prepared
// spectrum: three launches whose grid.y runs over the templates.
static fastfft_status red_xcorr_batch(fastfft_handle h, int mx, int my, int n, const void* const* inputs,
                                      const int* dims, void* const* outs, const fastfft_op* pre_op,
                                      const fastfft_op* intra_op, const fastfft_op* post_op,
                                      unsigned long long* peaks = nullptr, const int* slots = nullptr,
                                      unsigned long long* mip = nullptr, int mip_base = 0, int slice0 = 0) {
    char* c0 = region_c(h);
    const float2* spec = reinterpret_cast<const float2*>(c0 + h->off_c_spec);
    // template slices [slice0, slice0 + n) of region C (slice0 > 0: the second group in flight)
    float2* t1 = reinterpret_cast<float2*>(c0 + h->off_c_t1) + (long long)slice0 * h->red_t1_stride;
    float2* t2 = reinterpret_cast<float2*>(c0 + h->off_c_t2) + (long long)slice0 * h->red_t2_stride;
    const float2* tw = nullptr;
    cudaError_t e;
    prof_begin_call(h);
    if ((e = twiddles_for(mx, &tw)) != cudaSuccess) return cuda_fail(h, e, "twiddle table");
    RowFwdArgs a;
    std::memset(&a, 0, sizeof(a));
    for (int g = 0; g < n; g++) a.in[g] = inputs[g];
    a.n_batch = n;
    a.in_pitch = 2LL * h->fwd_in.w; a.n_rows = (int)h->fwd_in.y; a.L = (int)h->fwd_in.x;
    a.out = t1; a.out_pitch = h->pitch_a; a.out_batch_stride = h->red_t1_stride;
    a.kmax = mx / 2 + 1; a.scale = scale_of(pre_op); a.tw = tw;
    if (dims) {
        for (int g = 0; g < n; g++) {
            a.L_g[g] = dims[2 * g];
            a.rows_g[g] = dims[2 * g + 1];
            a.pitch_g[g] = 2LL * ((dims[2 * g] + (dims[2 * g] % 2 == 0 ? 2 : 1)) / 2);
        }
    }
    if ((e = launch_r2c_rows(mx, h->input_dtype, a, h->stream)) != cudaSuccess) return cuda_fail(h, e, "r2c row pass");
    h->launches++;
    // the column pass reads the prepared spectrum (the R2C above overlapped its preparation;
    // the wait falls into the R2C's timing mark)
    FFB_TRY(join_prep(h));
    prof_mark(h);
    if ((e = twiddles_for(my, &tw)) != cudaSuccess) return cuda_fail(h, e, "twiddle table");
    XcorrColArgs c;
    std::memset(&c, 0, sizeof(c));
    c.t1 = t1; c.t1_pitch = h->pitch_a; c.t1_batch = h->red_t1_stride; c.L = (int)h->fwd_in.y;
    c.img = spec; c.img_stride = my;
    c.out = t2; c.out_pitch = h->pitch_b; c.out_batch = h->red_t2_stride; c.W = (int)h->inv_out.y;
    c.n_cols = mx / 2 + 1; c.n_batch = n;
    c.tpb = xcorr_tpb(h, n, my);
    if (dims)
        for (int g = 0; g < n; g++) c.L_g[g] = dims[2 * g + 1];
    c.intra_kind = intra_op ? intra_op->kind : FASTFFT_OP_NOOP;
    c.intra_scale = intra_op ? intra_op->scale : 1.f;
    c.tw = tw; c.err = h->dev_err;
    c.tc = h->tc_dft ? 1 : 0;
    if ((e = launch_xcorr_cols(my, FASTFFT_DTYPE_C64, c, h->stream)) != cudaSuccess)
        return cuda_fail(h, e, "cross-correlation column pass");
    h->launches++;
    prof_mark(h);
    if ((e = twiddles_for(mx, &tw)) != cudaSuccess) return cuda_fail(h, e, "twiddle table");
    RowInvArgs r;
    std::memset(&r, 0, sizeof(r));
    r.n_batch = n;
    r.in = t2; r.in_pitch = h->pitch_b; r.in_batch_stride = h->red_t2_stride; r.n_rows = (int)h->inv_out.y;
    for (int g = 0; g < n; g++) r.out[g] = outs[g];
    if (peaks || mip) {
        r.peaks = peaks;
        r.peaks_only = outs[0] == nullptr;
        for (int g = 0; g < n; g++) r.peak_slot[g] = slots[g];
        r.mip = mip;
        r.mip_base = mip_base;
    }
    r.out_pitch = 2LL * h->inv_out.w; r.W = (int)h->inv_out.x; r.scale = scale_of(post_op); r.tw = tw;
    if ((e = launch_c2r_rows(mx, h->output_dtype, r, h->stream)) != cudaSuccess)
        return cuda_fail(h, e, "c2r row pass");
    h->launches++;
    prof_mark(h);
    prof_end_call(h);
    return FASTFFT_OK;
}

// The reduced-size correlation is exact for the correlation functors only: with CONJ_MUL (or
// CONJ_MUL_THEN_SCALE) every retained output is a lag of the correlation, which the smaller
// transform computes exactly; with NOOP or SCALE the call is a round trip of the template,
// whose outputs scale with the transform size, so those calls run at the plan's size.
static bool correlation_op(const fastfft_op* intra_op) {
    return intra_op && (intra_op->kind == FASTFFT_OP_CONJ_MUL || intra_op->kind == FASTFFT_OP_CONJ_MUL_THEN_SCALE);
}

fastfft_status fastfft_fwd_image_inv(fastfft_handle h, const void* input, const void* image_spectrum, void* output,
                                     const fastfft_op* pre_op, const fastfft_op* intra_op,
                                     const fastfft_op* post_op) {
    if (!h) return fail(nullptr, FASTFFT_ERR_INVALID_ARGUMENT, "null handle");
    if (!input || !image_spectrum) return fail(h, FASTFFT_ERR_INVALID_ARGUMENT, "null input or image pointer");
    fastfft_status st = xcorr_checks(h, pre_op, intra_op, post_op);
    if (st != FASTFFT_OK) return st;
    void* out = output ? output : const_cast<void*>(input);
    // With image reuse declared, a single template also goes through the reduced-size path:
    // the image is prepared on the first call that names it and reused after that.
    if (h->image_reuse && h->red_ok && !h->force_full_size && correlation_op(intra_op))
        return xcorr_many(h, 1, &input, nullptr, &image_spectrum, &out, pre_op, intra_op, post_op);
    return xcorr_one(h, input, image_spectrum, out, pre_op, intra_op, post_op);
}

// Shared body of the batched calls; dims (x, y per template) may be NULL (plan size).
static fastfft_status xcorr_many(fastfft_handle h, int n, const void* const* inputs, const int* dims,
                                 const void* const* image_spectra, void* const* outputs, const fastfft_op* pre_op,
                                 const fastfft_op* intra_op, const fastfft_op* post_op, unsigned long long* peaks,
                                 unsigned long long* mip, int mip_base) {
    // with a peak array or a projection the windows are written only where outputs[i] is set
    const bool reduce = peaks != nullptr || mip != nullptr;
    if (n < 0 || (n > 0 && (!inputs || !image_spectra)))
        return fail(h, FASTFFT_ERR_INVALID_ARGUMENT, "null input or image array");
    for (int i = 0; i < n; i++)
        if (!inputs[i] || !image_spectra[i])
            return fail(h, FASTFFT_ERR_INVALID_ARGUMENT, "null input or image pointer in the batch");
    fastfft_status st = xcorr_checks(h, pre_op, intra_op, post_op);
    if (st != FASTFFT_OK) return st;
    if (dims) {
        if (h->rank != 2) return fail(h, FASTFFT_ERR_UNSUPPORTED, "per-template sizes are 2D only");
        for (int i = 0; i < n; i++)
            if (dims[2 * i] < 1 || dims[2 * i + 1] < 1 || dims[2 * i] > h->fwd_in.x || dims[2 * i + 1] > h->fwd_in.y)
                return fail(h, FASTFFT_ERR_INVALID_DIMS,
                            "template " + std::to_string(i) + " is larger than the plan's forward input size");
    }
    if (peaks) {
        cudaError_t e = cudaMemsetAsync(peaks, 0, sizeof(unsigned long long) * (size_t)n, h->stream);
        if (e != cudaSuccess) return cuda_fail(h, e, "clearing the peak array");
    }
    if (!h->red_ok || h->force_full_size || !correlation_op(intra_op)) {
        if ((peaks || mip) && ffb::is_blue_size((int)h->inv_in.x))
            return fail(h, FASTFFT_ERR_UNSUPPORTED,
                        "the fused peak search and projection need a power-of-two or R * 2^k inverse row length");
        for (int i = 0; i < n; i++) {
            void* out = reduce ? (outputs ? outputs[i] : nullptr)
                               : ((outputs && outputs[i]) ? outputs[i] : const_cast<void*>(inputs[i]));
            if (dims || reduce) {
                prof_begin_call(h);
                st = seq_xcorr_sized(h, inputs[i], dims ? dims[2 * i] : (int)h->fwd_in.x,
                                     dims ? dims[2 * i + 1] : (int)h->fwd_in.y, image_spectra[i], out,
                                     scale_of(pre_op), intra_op, scale_of(post_op), peaks, i, mip, mip_base);
                prof_end_call(h);
            } else {
                st = xcorr_one(h, inputs[i], image_spectra[i], out, pre_op, intra_op, post_op);
            }
            if (st != FASTFFT_OK) return st;
        }
        return FASTFFT_OK;
    }
    // Reduced-size path: templates are grouped by image and, within an image, by size class
    // (the exact correlation size of each template, which for templates smaller than the
    // plan's can be smaller than the plan's), in order of first use; the image is prepared
    // once per class for the whole call; up to red_batch templates per launch.
    std::vector<char> done(n, 0);
    std::vector<int> cls_x(n), cls_y(n);
    for (int k = 0; k < n; k++) {
        cls_x[k] = (int)h->red_mx;
        cls_y[k] = (int)h->red_my;
#if FFB_SIZE_CLASSES
        if (dims) {
            cls_x[k] = (int)std::min<long long>(cls_x[k], corr_size_at_least(dims[2 * k] + h->inv_out.x - 1));
            cls_y[k] = (int)std::min<long long>(cls_y[k], corr_size_at_least(dims[2 * k + 1] + h->inv_out.y - 1));
        }
#endif
    }
    const void* grp_in[kMaxBatch];
    void* grp_out[kMaxBatch];
    int grp_dims[2 * kMaxBatch];
    int grp_slot[kMaxBatch];
    // Pipelined groups: every second group runs on the pipe stream with the second set of
    // template slices; the pipe stream is forked from `stream` before its first group and
    // joined back before returning (also on errors).
    const bool pipe = h->pipe_groups > 1 && h->pipe_stream != nullptr;
    bool pipe_forked = false;
    int group_no = 0;
    auto run_group = [&](int mx, int my, int m) -> fastfft_status {
        const bool second = pipe && (group_no++ & 1);
        if (!second)
            return red_xcorr_batch(h, mx, my, m, grp_in, dims ? grp_dims : nullptr, grp_out, pre_op, intra_op,
                                   post_op, peaks, grp_slot, mip, mip_base, 0);
        if (!pipe_forked) {
            cudaError_t e = cudaEventRecord(h->pipe_fork, h->stream);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(h->pipe_stream, h->pipe_fork, 0);
            if (e != cudaSuccess) return cuda_fail(h, e, "forking the pipelined groups");
            pipe_forked = true;
            h->pipe_active = true;
        }
        cudaStream_t main_stream = h->stream;
        h->stream = h->pipe_stream;
        fastfft_status s2 = red_xcorr_batch(h, mx, my, m, grp_in, dims ? grp_dims : nullptr, grp_out, pre_op,
                                            intra_op, post_op, peaks, grp_slot, mip, mip_base, h->red_batch);
        h->stream = main_stream;
        return s2;
    };
    auto join_pipe = [&](fastfft_status prior) -> fastfft_status {
        if (!pipe_forked) return prior;
        h->pipe_active = false;
        cudaError_t e = cudaEventRecord(h->pipe_join, h->pipe_stream);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(h->stream, h->pipe_join, 0);
        if (e != cudaSuccess) {
            cudaStreamSynchronize(h->pipe_stream);
            return prior != FASTFFT_OK ? prior : cuda_fail(h, e, "joining the pipelined groups");
        }
        return prior;
    };
    for (int i = 0; i < n; i++) {
        if (done[i]) continue;
        const void* img = image_spectra[i];
        const int mx = cls_x[i], my = cls_y[i];
        st = red_prepare_image(h, img, mx, my);
        if (st != FASTFFT_OK) return join_pipe(st);
        int m = 0;
        for (int k = i; k < n; k++) {
            if (done[k] || image_spectra[k] != img || cls_x[k] != mx || cls_y[k] != my) continue;
            grp_in[m] = inputs[k];
            grp_out[m] = reduce ? (outputs ? outputs[k] : nullptr)
                                : ((outputs && outputs[k]) ? outputs[k] : const_cast<void*>(inputs[k]));
            grp_slot[m] = k;
            if (dims) {
                grp_dims[2 * m] = dims[2 * k];
                grp_dims[2 * m + 1] = dims[2 * k + 1];
            }
            done[k] = 1;
            if (++m == h->red_batch) {
                st = run_group(mx, my, m);
                if (st != FASTFFT_OK) return join_pipe(st);
                m = 0;
            }
        }
        if (m > 0) {
            st = run_group(mx, my, m);
            if (st != FASTFFT_OK) return join_pipe(st);
        }
    }
    return join_pipe(FASTFFT_OK);
}

fastfft_status fastfft_fwd_image_inv_many(fastfft_handle h, int n, const void* const* inputs,
                                          const void* const* image_spectra, void* const* outputs,
                                          const fastfft_op* pre_op, const fastfft_op* intra_op,
                                          const fastfft_op* post_op) {
    if (!h) return fail(nullptr, FASTFFT_ERR_INVALID_ARGUMENT, "null handle");
    return xcorr_many(h, n, inputs, nullptr, image_spectra, outputs, pre_op, intra_op, post_op);
}

fastfft_status fastfft_fwd_image_inv_many_sized(fastfft_handle h, int n, const void* const* inputs,
                                                const int* template_dims, const void* const* image_spectra,
                                                void* const* outputs, const fastfft_op* pre_op,
                                                const fastfft_op* intra_op, const fastfft_op* post_op) {
    if (!h) return fail(nullptr, FASTFFT_ERR_INVALID_ARGUMENT, "null handle");
    if (n > 0 && !template_dims) return fail(h, FASTFFT_ERR_INVALID_ARGUMENT, "null template size array");
    return xcorr_many(h, n, inputs, template_dims, image_spectra, outputs, pre_op, intra_op, post_op);
}

fastfft_status fastfft_fwd_image_inv_many_peaks(fastfft_handle h, int n, const void* const* inputs,
                                                const int* template_dims, const void* const* image_spectra,
                                                void* const* outputs, unsigned long long* peaks,
                                                const fastfft_op* pre_op, const fastfft_op* intra_op,
                                                const fastfft_op* post_op) {
    if (!h) return fail(nullptr, FASTFFT_ERR_INVALID_ARGUMENT, "null handle");
    if (n > 0 && !peaks) return fail(h, FASTFFT_ERR_INVALID_ARGUMENT, "null peak array");
    if (h->rank != 2) return fail(h, FASTFFT_ERR_UNSUPPORTED, "the fused peak search is 2D only");
    if (outputs)
        for (int i = 0; i < n; i++)
            if (!outputs[i]) return fail(h, FASTFFT_ERR_INVALID_ARGUMENT, "null output pointer in the batch");
    return xcorr_many(h, n, inputs, template_dims, image_spectra, outputs, pre_op, intra_op, post_op, peaks);
}

fastfft_status fastfft_fwd_image_inv_many_mip(fastfft_handle h, int n, const void* const* inputs,
                                              const int* template_dims, const void* const* image_spectra,
                                              void* const* outputs, unsigned long long* mip, int index_base,
                                              const fastfft_op* pre_op, const fastfft_op* intra_op,
                                              const fastfft_op* post_op) {
    if (!h) return fail(nullptr, FASTFFT_ERR_INVALID_ARGUMENT, "null handle");
    if (n > 0 && !mip) return fail(h, FASTFFT_ERR_INVALID_ARGUMENT, "null projection array");
    if (h->rank != 2) return fail(h, FASTFFT_ERR_UNSUPPORTED, "the fused maximum projection is 2D only");
    if (index_base < 0 || (long long)index_base + n > 0x7FFFFFFFLL)
        return fail(h, FASTFFT_ERR_INVALID_ARGUMENT, "template indices must be in [0, 2^31)");
    if (outputs)
        for (int i = 0; i < n; i++)
            if (!outputs[i]) return fail(h, FASTFFT_ERR_INVALID_ARGUMENT, "null output pointer in the batch");
    return xcorr_many(h, n, inputs, template_dims, image_spectra, outputs, pre_op, intra_op, post_op, nullptr, mip,
                      index_base);
}

fastfft_status fastfft_set_templates_per_launch(fastfft_handle h, int n) {
    if (!h) return fail(nullptr, FASTFFT_ERR_INVALID_ARGUMENT, "null handle");
    if (n < 1 || n > kMaxBatch)
        return fail(h, FASTFFT_ERR_INVALID_ARGUMENT, "templates per launch must be in [1, " + std::to_string(kMaxBatch) + "]");
    h->red_batch_request = n;
    h->validated = false;
    if (h->fwd_set && h->inv_set) {
        fastfft_status st = validate(h);
        if (st != FASTFFT_OK) return st;
        const size_t before = h->buffer_bytes;
        size_buffers(h);
        if (h->buffer && (size_t)(h->bytes_a + h->bytes_b + h->bytes_c) + 256 > before) {
            cudaFree(h->buffer);
            h->buffer = nullptr;
            h->buffer_bytes = 0;
        }
    }
    return FASTFFT_OK;
}

fastfft_status fastfft_set_templates_per_block(fastfft_handle h, int n) {
    if (!h) return fail(nullptr, FASTFFT_ERR_INVALID_ARGUMENT, "null handle");
    if (n < 0 || n > kMaxBatch)
        return fail(h, FASTFFT_ERR_INVALID_ARGUMENT, "templates per block must be in [0, " + std::to_string(kMaxBatch) + "]");
    if (h->buffer) cudaStreamSynchronize(h->stream);   // earlier calls may still use the slices
    h->tpb_request = n;
    h->validated = false;
    if (h->fwd_set && h->inv_set) {
        fastfft_status st = validate(h);
        if (st != FASTFFT_OK) return st;
        // the templates per launch follow (they shrink where shared memory needs it, and grow
        // back to the request); a buffer too small for them is reallocated by the next call
        const size_t before = h->buffer_bytes;
        size_buffers(h);
        if (h->buffer && (size_t)(h->bytes_a + h->bytes_b + h->bytes_c) + 256 > before) {
            cudaFree(h->buffer);
            h->buffer = nullptr;
            h->buffer_bytes = 0;
        }
    }
    return FASTFFT_OK;
}

fastfft_status fastfft_templates_per_block(fastfft_handle h, int* n) {
    if (!h || !n) return fail(h, FASTFFT_ERR_INVALID_ARGUMENT, "null argument");
    *n = (h->red_ok && !h->force_full_size) ? xcorr_tpb(h, h->red_batch, h->red_my) : 1;
    return FASTFFT_OK;
}

fastfft_status fastfft_set_pipelined_groups(fastfft_handle h, int n) {
    if (!h) return fail(nullptr, FASTFFT_ERR_INVALID_ARGUMENT, "null handle");
    if (n != 1 && n != 2) return fail(h, FASTFFT_ERR_INVALID_ARGUMENT, "pipelined groups must be 1 or 2");
    if (n == h->pipe_groups) return FASTFFT_OK;
    if (h->buffer) cudaStreamSynchronize(h->stream);   // earlier calls may still use the slices
    h->pipe_groups = n;
    h->prepared_image = nullptr;
    h->validated = false;
    if (h->fwd_set && h->inv_set) {
        fastfft_status st = validate(h);
        if (st != FASTFFT_OK) return st;
        const size_t before = h->buffer_bytes;
        size_buffers(h);
        if (h->buffer && (size_t)(h->bytes_a + h->bytes_b + h->bytes_c) + 256 > before) {
            cudaFree(h->buffer);
            h->buffer = nullptr;
            h->buffer_bytes = 0;
        }
        int n_dev = 0;
        if (cudaGetDeviceCount(&n_dev) == cudaSuccess && n_dev > 0)
            create_pipe_stream(h);
        else
            cudaGetLastError();
    }
    return FASTFFT_OK;
}

fastfft_status fastfft_pipelined_groups(fastfft_handle h, int* n) {
    if (!h || !n) return fail(h, FASTFFT_ERR_INVALID_ARGUMENT, "null argument");
    *n = (h->pipe_groups > 1 && h->pipe_stream && h->red_ok && !h->force_full_size) ? 2 : 1;
    return FASTFFT_OK;
}

fastfft_status fastfft_templates_per_launch(fastfft_handle h, int* n) {
    if (!h || !n) return fail(h, FASTFFT_ERR_INVALID_ARGUMENT, "null argument");
    *n = h->red_ok && !h->force_full_size ? h->red_batch : 1;
    return FASTFFT_OK;
}

fastfft_status fastfft_set_full_size_correlation(fastfft_handle h, int force) {
    if (!h) return fail(nullptr, FASTFFT_ERR_INVALID_ARGUMENT, "null handle");
    h->force_full_size = force != 0;
    return FASTFFT_OK;
}

fastfft_status fastfft_correlation_size(fastfft_handle h, int dims[2]) {
    if (!h || !dims) return fail(h, FASTFFT_ERR_INVALID_ARGUMENT, "null argument");
    fastfft_status st = validate(h);
    if (st != FASTFFT_OK) return st;
    size_buffers(h);
    const bool red = h->red_ok && !h->force_full_size;
    dims[0] = (int)(red ? h->red_mx : h->fwd_out.x);
    dims[1] = (int)(red ? h->red_my : h->fwd_out.y);
    return FASTFFT_OK;
}

fastfft_status fastfft_launch_count(fastfft_handle h, long long* n) {
    if (!h || !n) return fail(h, FASTFFT_ERR_INVALID_ARGUMENT, "null argument");
    *n = h->launches;
    return FASTFFT_OK;
}

fastfft_status fastfft_profile_start(fastfft_handle h, int max_calls) {
    if (!h) return fail(nullptr, FASTFFT_ERR_INVALID_ARGUMENT, "null handle");
    if (max_calls <= 0) return fail(h, FASTFFT_ERR_INVALID_ARGUMENT, "max_calls must be > 0");
    if (h->prof_events) return fail(h, FASTFFT_ERR_INVALID_ARGUMENT, "profiling is already on");
    const int n = max_calls * fastfft_plan_s::kProfMarks;
    cudaEvent_t* ev = new (std::nothrow) cudaEvent_t[n];
    if (!ev) return fail(h, FASTFFT_ERR_ALLOC, "out of host memory");
    for (int i = 0; i < n; i++) {
        cudaError_t e = cudaEventCreate(&ev[i]);
        if (e != cudaSuccess) {
            for (int k = 0; k < i; k++) cudaEventDestroy(ev[k]);
            delete[] ev;
            return cuda_fail(h, e, "cudaEventCreate");
        }
    }
    h->prof_events = ev;
    h->prof_capacity = max_calls;
    h->prof_calls = 0;
    h->prof_mark = 0;
    return FASTFFT_OK;
}

fastfft_status fastfft_profile_stop(fastfft_handle h, double* pass_ms, int n_pass, long long* n_calls) {
    if (!h) return fail(nullptr, FASTFFT_ERR_INVALID_ARGUMENT, "null handle");
    if (!h->prof_events) return fail(h, FASTFFT_ERR_INVALID_ARGUMENT, "profiling is not on");
    constexpr int M = fastfft_plan_s::kProfMarks;
    fastfft_status st = FASTFFT_OK;
    double acc[M - 1] = {0, 0, 0};
    for (int c = 0; c < h->prof_calls && st == FASTFFT_OK; c++) {
        for (int p = 0; p < M - 1; p++) {
            cudaError_t e = cudaEventSynchronize(h->prof_events[c * M + p + 1]);
            float ms = 0.f;
            if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, h->prof_events[c * M + p], h->prof_events[c * M + p + 1]);
            if (e != cudaSuccess) {
                st = cuda_fail(h, e, "profile events");
                break;
            }
            acc[p] += ms;
        }
    }
    if (pass_ms)
        for (int p = 0; p < n_pass && p < M - 1; p++) pass_ms[p] = acc[p];
    if (n_calls) *n_calls = h->prof_calls;
    for (int i = 0; i < h->prof_capacity * M; i++) cudaEventDestroy(h->prof_events[i]);
    delete[] h->prof_events;
    h->prof_events = nullptr;
    h->prof_capacity = 0;
    h->prof_calls = 0;
    return st;
}

static fastfft_status get_ll(fastfft_handle h, long long* n, long long v) {
    if (!h || !n) return fail(h, FASTFFT_ERR_INVALID_ARGUMENT, "null argument");
    *n = v;
    return FASTFFT_OK;
}

fastfft_status fastfft_input_memory_size(fastfft_handle h, long long* n) { return get_ll(h, n, h ? h->input_mem : 0); }
fastfft_status fastfft_fwd_output_memory_size(fastfft_handle h, long long* n) {
    return get_ll(h, n, h ? h->fwd_out_mem : 0);
}
fastfft_status fastfft_inv_output_memory_size(fastfft_handle h, long long* n) {
    return get_ll(h, n, h ? h->inv_out_mem : 0);
}
fastfft_status fastfft_buffer_bytes(fastfft_handle h, long long* n) {
    return get_ll(h, n, h ? (long long)h->buffer_bytes : 0);
}

static fastfft_status get_dims(fastfft_handle h, int dims[4], const Dims& d) {
    if (!h || !dims) return fail(h, FASTFFT_ERR_INVALID_ARGUMENT, "null argument");
    dims[0] = (int)d.x;
    dims[1] = (int)d.y;
    dims[2] = (int)d.z;
    dims[3] = (int)d.w;
    return FASTFFT_OK;
}

fastfft_status fastfft_fwd_input_dims(fastfft_handle h, int dims[4]) { return get_dims(h, dims, h ? h->fwd_in : Dims{}); }
fastfft_status fastfft_fwd_output_dims(fastfft_handle h, int dims[4]) { return get_dims(h, dims, h ? h->fwd_out : Dims{}); }
fastfft_status fastfft_inv_input_dims(fastfft_handle h, int dims[4]) { return get_dims(h, dims, h ? h->inv_in : Dims{}); }
fastfft_status fastfft_inv_output_dims(fastfft_handle h, int dims[4]) { return get_dims(h, dims, h ? h->inv_out : Dims{}); }

fastfft_status fastfft_wait(fastfft_handle h) {
    if (!h) return fail(nullptr, FASTFFT_ERR_INVALID_ARGUMENT, "null handle");
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cuda_fail(h, e, "cudaStreamSynchronize");
    if (h->prep_join_pending) {
        // an image preparation whose column pass never ran (a failed call): wait for it too
        h->prep_join_pending = false;
        e = cudaStreamSynchronize(h->prep_stream);
        if (e != cudaSuccess) return cuda_fail(h, e, "cudaStreamSynchronize (image preparation)");
    }
    if (h->dev_err) {
        int flag = 0;
        e = cudaMemcpy(&flag, h->dev_err, sizeof(int), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return cuda_fail(h, e, "reading the status word");
        if (flag) {
            cudaMemset(h->dev_err, 0, sizeof(int));
            return fail(h, FASTFFT_ERR_TIMEOUT, "a kernel gave up waiting for its bulk copies; its outputs are incomplete");
        }
    }
    return FASTFFT_OK;
}

const char* fastfft_last_error(fastfft_handle h) { return h ? h->last_error.c_str() : g_null_handle_error.c_str(); }

const char* fastfft_status_string(int status) {
    switch (status) {
        case FASTFFT_OK: return "ok";
        case FASTFFT_ERR_INVALID_ARGUMENT: return "invalid argument";
        case FASTFFT_ERR_INVALID_DIMS: return "invalid dimensions";
        case FASTFFT_ERR_UNSUPPORTED: return "unsupported";
        case FASTFFT_ERR_NOT_PLANNED: return "not planned";
        case FASTFFT_ERR_CUDA: return "cuda error";
        case FASTFFT_ERR_ALLOC: return "allocation failed";
        case FASTFFT_ERR_TIMEOUT: return "device wait timed out";
        default: return "unknown status";
    }
}

const char* fastfft_version(void) { return kVersion; }

void fastfft_decode_peak(unsigned long long key, float* value, unsigned int* index) {
    const unsigned int ordered = (unsigned int)(key >> 32);
    const unsigned int bits = (ordered & 0x80000000u) ? (ordered & 0x7FFFFFFFu) : ~ordered;
    float v;
    std::memcpy(&v, &bits, sizeof(v));
    if (value) *value = v;
    if (index) *index = 0xFFFFFFFFu - (unsigned int)(key & 0xFFFFFFFFu);
}

}  // extern "C"
