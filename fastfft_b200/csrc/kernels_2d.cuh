// 2D passes of the size-changing FFT path (sm_100a).
//
//   r2c_rows   : row R2C along x of up to L_y rows, zero padding x >= L implicit,
//                two real rows per complex FFT, output transposed to [kx][y]
//                (replaces block_fft_kernel_R2C_{NONE,INCREASE,DECREASE}_XY,
//                 src/fastfft/FastFFT.cu:1055-1077, :1107-1166, :1232-1261)
//   cols       : column C2C along y over the [kx][y] layout; three modes
//                  COL_FWD   forward, zero padding y >= L, keep first W outputs
//                            (C2C_NONE / C2C_INCREASE / C2C_DECREASE, :1348-1475)
//                  COL_INV   inverse, keep first W outputs (C2C inverse passes)
//                  COL_XCORR forward (pruned) -> conj(T)*I intra-op against the
//                            resident image spectrum -> inverse, keep first W
//                            (the fused C2C_FWD_INCREASE_OP_INV_NONE, :20-56, extended
//                             with the trimmed inverse that the reference aborts on,
//                             :673-679)
//   c2r_rows   : row C2R along x reading [kx][y], two rows per complex FFT, keep
//                the first W_x outputs (C2R_NONE_XY / C2R_DECREASE_XY, :1641-1692)
#pragma once

#include "fft_core.cuh"
#include "tma.cuh"

namespace ffb {

// ---------------------------------------------------------------------------
// dtype helpers
// ---------------------------------------------------------------------------
template <class T> __device__ __forceinline__ float ld_real(const T* p);
template <> __device__ __forceinline__ float ld_real<float>(const float* p) { return __ldg(p); }
template <> __device__ __forceinline__ float ld_real<__half>(const __half* p) { return __half2float(__ldg(p)); }
template <> __device__ __forceinline__ float ld_real<__nv_bfloat16>(const __nv_bfloat16* p) {
    return __bfloat162float(__ldg(p));
}

template <class T> __device__ __forceinline__ void st_real(T* p, float v);
template <> __device__ __forceinline__ void st_real<float>(float* p, float v) { *p = v; }
template <> __device__ __forceinline__ void st_real<__half>(__half* p, float v) { *p = __float2half_rn(v); }
template <> __device__ __forceinline__ void st_real<__nv_bfloat16>(__nv_bfloat16* p, float v) {
    *p = __float2bfloat16_rn(v);
}

// Complex loads.  The streaming variant (evict-first) is used for the resident
// image spectrum, which is read exactly once per template and should not push
// the template's intermediates out of L2.
template <class T> __device__ __forceinline__ float2 ld_cplx(const T* p);
template <> __device__ __forceinline__ float2 ld_cplx<float2>(const float2* p) { return *p; }
template <> __device__ __forceinline__ float2 ld_cplx<__half2>(const __half2* p) { return __half22float2(*p); }
template <> __device__ __forceinline__ float2 ld_cplx<__nv_bfloat162>(const __nv_bfloat162* p) {
    return __bfloat1622float2(*p);
}

// Complex stores (the forward spectrum may be written in FP16 / BF16, rounded to nearest)
template <class T> __device__ __forceinline__ void st_cplx(T* p, float2 v);
template <> __device__ __forceinline__ void st_cplx<float2>(float2* p, float2 v) { *p = v; }
template <> __device__ __forceinline__ void st_cplx<__half2>(__half2* p, float2 v) { *p = __float22half2_rn(v); }
template <> __device__ __forceinline__ void st_cplx<__nv_bfloat162>(__nv_bfloat162* p, float2 v) {
    *p = __float22bfloat162_rn(v);
}

template <class T> __device__ __forceinline__ float2 ld_cplx_stream(const T* p);
template <> __device__ __forceinline__ float2 ld_cplx_stream<float2>(const float2* p) { return __ldcs(p); }
template <> __device__ __forceinline__ float2 ld_cplx_stream<__half2>(const __half2* p) {
    unsigned int u = __ldcs(reinterpret_cast<const unsigned int*>(p));
    __half2 h = *reinterpret_cast<__half2*>(&u);
    return __half22float2(h);
}
template <> __device__ __forceinline__ float2 ld_cplx_stream<__nv_bfloat162>(const __nv_bfloat162* p) {
    unsigned int u = __ldcs(reinterpret_cast<const unsigned int*>(p));
    __nv_bfloat162 h = *reinterpret_cast<__nv_bfloat162*>(&u);
    return __bfloat1622float2(h);
}

// Shared-memory loads of the staged image column, kept at their point of use (a plain
// load could be hoisted above the forward transform, holding 16 more complex values live
// across it and pushing the kernel past its register budget).
template <class T> __device__ __forceinline__ float2 lds_cplx(const T* p);
template <> __device__ __forceinline__ float2 lds_cplx<float2>(const float2* p) {
    float2 r;
    asm volatile("ld.shared.v2.f32 {%0, %1}, [%2];" : "=f"(r.x), "=f"(r.y) : "r"(smem_addr(p)));
    return r;
}
template <> __device__ __forceinline__ float2 lds_cplx<__half2>(const __half2* p) {
    unsigned int u;
    asm volatile("ld.shared.b32 %0, [%1];" : "=r"(u) : "r"(smem_addr(p)));
    return __half22float2(*reinterpret_cast<__half2*>(&u));
}
template <> __device__ __forceinline__ float2 lds_cplx<__nv_bfloat162>(const __nv_bfloat162* p) {
    unsigned int u;
    asm volatile("ld.shared.b32 %0, [%1];" : "=r"(u) : "r"(smem_addr(p)));
    return __bfloat1622float2(*reinterpret_cast<__nv_bfloat162*>(&u));
}

// number of leading q slots (x[j + T q]) that can be non-zero when only n < L is loaded
template <int T>
__device__ __forceinline__ int leading_slots(int L, int j) {
    if (L <= j) return 0;
    int q = (L - j + T - 1) / T;
    return q > 16 ? 16 : q;
}

// ---------------------------------------------------------------------------
// Row R2C (forward), two rows per complex FFT
// ---------------------------------------------------------------------------
// Templates per launch: blockIdx.y selects the template of a batch (the row passes take them
// in reverse order, so that each pass starts on the data its predecessor wrote last).
// Templates per launch of the batched passes (grid.y).  Up to 64: more templates per launch
// mean more blocks per launch and a shorter partly empty last wave in all three passes
// (measured on B200 at 1536^2: 13.8, 12.1 and 11.5 us per template at 16, 32 and 64).
constexpr int kMaxBatch = 64;

struct RowFwdArgs {
    const void* in[kMaxBatch];  // real rows of template g: row r at in[g] + r * in_pitch (elements)
    long long in_pitch;
    long long out_batch_stride; // complex elements between the outputs of consecutive templates
    int n_rows;            // rows that exist (rows >= n_rows are not produced)
    int L;                 // valid x per row; x in [L, N) is zero padding
    float2* out;           // out[k * out_pitch + r] for k < kmax
    long long out_pitch;   // >= n_rows, even
    int kmax;              // kx outputs written (N/2+1, or fewer for a decrease)
    float scale;           // pre-op SCALE (1 = NOOP)
    const float2* tw;      // twiddle table of size N (N = 3P: of the sub-FFT size P)
    const float2* tw3;     // N = 3P: radix-3 pass twiddles (set by the launcher)
    int n_batch;           // templates in this launch (grid.y)
    // 3D: flat row r = y * rows_z + z reads input row z * rows_y + y, so that the output
    // [kx][y][z] has z contiguous.  rows_z <= 1: row r reads input row r.
    int rows_y;
    int rows_z;
    // Per-template sizes of a batch of uneven templates (0: use n_rows / L / in_pitch).
    int rows_g[kMaxBatch];
    int L_g[kMaxBatch];
    long long pitch_g[kMaxBatch];
};

__device__ __forceinline__ long long input_row(int r, int rows_y, int rows_z) {
    if (rows_z <= 1) return r;
    return (long long)(r % rows_z) * rows_y + r / rows_z;
}

template <int N, class InT, int FPB>
__global__ void __launch_bounds__(FftShape<N>::T * FPB, (FftShape<N>::T * FPB <= 256) ? 4 : 2)
r2c_rows_kernel(RowFwdArgs a) {
    using S = FftShape<N>;
    constexpr int T = S::T;
    extern __shared__ float2 smem[];
    using G = FftGroup<N, FPB, false>;
    const int f = threadIdx.x / T;
    const int j = threadIdx.x - f * T;
    G g(smem, f);
    float2* s = g.base;
    // batch entries in reverse order: the batched column pass that follows starts with entry 0,
    // whose rows are then the last written and still in L2
    const int gb = gridDim.y - 1 - blockIdx.y;
    const int n_rows = a.rows_g[gb] > 0 ? a.rows_g[gb] : a.n_rows;
    const int L = a.L_g[gb] > 0 ? a.L_g[gb] : a.L;
    const long long in_pitch = a.pitch_g[gb] > 0 ? a.pitch_g[gb] : a.in_pitch;
    const int ra = 2 * (blockIdx.x * FPB + f);
    const bool has_a = ra < n_rows, has_b = ra + 1 < n_rows;
    const InT* in_g = static_cast<const InT*>(a.in[gb]);
    const InT* pa = in_g + input_row(ra, a.rows_y, a.rows_z) * in_pitch;
    const InT* pb = in_g + input_row(ra + 1, a.rows_y, a.rows_z) * in_pitch;
    float2* const out_g = a.out + (long long)gb * a.out_batch_stride;
    float2 v[16];
#pragma unroll
    for (int q = 0; q < 16; q++) {
        const int n = j + T * q;
        float xa = 0.f, xb = 0.f;
        if (n < L) {
            if (has_a) xa = ld_real<InT>(pa + n);
            if (has_b) xb = ld_real<InT>(pb + n);
        }
        v[q] = make_float2(xa * a.scale, xb * a.scale);
    }
    BlockFft<N, false>::run(v, g, j, a.tw, leading_slots<T>(L, j));

    // Split Z = A + iB into the two real-row spectra: A[k] = (Z[k] + conj Z[N-k]) / 2,
    // B[k] = -i (Z[k] - conj Z[N-k]) / 2.
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 16; q++) s[phys(j + T * q)] = v[q];
    __syncthreads();
    // item it of this thread: spectrum index k = k0 + T it of FFT ff0
    constexpr int kItemsPerThread = (FPB * (N / 2 + 1) + T * FPB - 1) / (T * FPB);
    const int ff0 = threadIdx.x % FPB;
    const int k0 = threadIdx.x / FPB;
    const float2* sf = smem + ff0 * G::STRIDE;
    const int rr0 = 2 * (blockIdx.x * FPB + ff0);
    const bool two = rr0 + 1 < n_rows, one = rr0 < n_rows;
    float2* o = out_g + (long long)k0 * a.out_pitch + rr0;
    const long long step = (long long)T * a.out_pitch;
#pragma unroll
    for (int it = 0; it < kItemsPerThread; it++, o += step) {
        const int k = k0 + T * it;
        if (k >= a.kmax) continue;
        const float2 z1 = sf[phys(k)];
        const float2 z2 = sf[phys((N - k) & (N - 1))];
        const float2 A = make_float2(0.5f * (z1.x + z2.x), 0.5f * (z1.y - z2.y));
        const float2 B = make_float2(0.5f * (z1.y + z2.y), 0.5f * (z2.x - z1.x));
        if (two) {
            *reinterpret_cast<float4*>(o) = make_float4(A.x, A.y, B.x, B.y);
        } else if (one) {
            *o = A;
        }
    }
}

// ---------------------------------------------------------------------------
// Column C2C
// ---------------------------------------------------------------------------
enum ColMode { COL_FWD = 0, COL_INV = 1, COL_XCORR = 2 };

struct ColArgs {
    const void* in;          // column c of batch entry g at in + g * in_batch_stride + c * in_stride
    long long in_stride;
    long long in_batch_stride;
    long long img_batch_stride;  // 0: every batch entry searches the same image
    long long out_batch_stride;
    int L;                   // valid input rows per column (zero beyond)
    const void* img;         // XCORR: image spectrum column c at img + c * img_stride
    long long img_stride;
    void* out;               // column c at out + c * out_stride
    long long out_stride;
    int W;                   // outputs kept per column
    int n_cols;
    int intra_kind;          // 0 NOOP, 2 CONJ_MUL, 3 CONJ_MUL_THEN_SCALE
    float intra_scale;
    float in_scale;
    float out_scale;
    const float2* tw;
    const float2* tw3;       // N = 3P: radix-3 pass twiddles (set by the launcher)
    int n_batch;             // batch entries in this launch (grid.y)
    // General addressing (3D passes); zero values select the plain 2D layout above.
    //   input  column c: (c / in_div) * in_stride + (c % in_div) * in_stride2
    //   output column c, element n in [W0, W0 + W):
    //          (c / out_div) * out_stride + (c % out_div) * out_stride2 + (n - W0) * out_elem_stride
    int in_div;
    long long in_stride2;
    int out_div;
    long long out_stride2;
    long long out_elem_stride;
    int W0;
    // XCORR with one column per block: the image column is staged in shared memory by a bulk
    // copy issued at the start of the block, so its load overlaps the forward transform
    // (set by the launcher when the column is 16-byte aligned; err receives a timeout).
    int stage_img;
    int* err;
    // Transposed output (out_elem_stride > 1) whose FPB columns of a block are consecutive in
    // memory for every element: the block writes through shared memory so that consecutive
    // threads store consecutive columns (FPB x 8 bytes contiguous per element instead of two
    // columns per warp).  Set by the launcher when the addressing allows it.
    int out_coalesce;
};

// Shared-memory plan of cols_kernel (bytes): the FFT groups' exchange buffers, then (when the
// image column is staged) the column and its barrier.
template <int N, class ImgC, int FPB>
struct ColSmem {
    static constexpr int kXchBytes = FftGroup<N, FPB, true>::BYTES;
    static constexpr int kImgOff = (kXchBytes + 127) & ~127;
    static constexpr int kImgBytes = N * (int)sizeof(ImgC);
    static constexpr int kBarOff = (kImgOff + kImgBytes + 15) & ~15;
    static constexpr int kStagedBytes = kBarOff + 16;
};

template <int N, int MODE, class InC, class ImgC, class OutC, int FPB>
__global__ void __launch_bounds__(FftShape<N>::T * FPB, (FftShape<N>::T * FPB <= 256) ? 2 : 1)
cols_kernel(ColArgs a) {
    using S = FftShape<N>;
    constexpr int T = S::T;
    extern __shared__ __align__(128) float2 smem[];
    using G = FftGroup<N, FPB, true>;
    using CS = ColSmem<N, ImgC, FPB>;
    const int f = threadIdx.x / T;
    const int j = threadIdx.x - f * T;
    G g(smem, f);
    const int col = blockIdx.x * FPB + f;
    const bool valid = col < a.n_cols;
    const long long bz = blockIdx.y;
    // image staging (XCORR, one column per block, block-uniform): thread 0 starts the bulk copy
    // now; the block waits for it (bounded) just before the conj-multiply
    unsigned char* const sm_raw = reinterpret_cast<unsigned char*>(smem);
    const ImgC* img_s = reinterpret_cast<const ImgC*>(sm_raw + CS::kImgOff);
    uint64_t* img_bar = reinterpret_cast<uint64_t*>(sm_raw + CS::kBarOff);
    __shared__ int img_ok;
    bool staged = false;
    if constexpr (MODE == COL_XCORR && FPB == 1) {
        staged = a.stage_img && a.intra_kind != 0 && valid;
        if (staged && threadIdx.x == 0) {
            mbar_init(img_bar, 1);
            fence_barrier_init();
            mbar_arrive_expect_tx(img_bar, (uint32_t)CS::kImgBytes);
            bulk_g2s(sm_raw + CS::kImgOff,
                     static_cast<const ImgC*>(a.img) + bz * a.img_batch_stride + (long long)col * a.img_stride,
                     (uint32_t)CS::kImgBytes, img_bar);
        }
    }
    const int in_div = a.in_div > 0 ? a.in_div : 1;
    const InC* pin = static_cast<const InC*>(a.in) + bz * a.in_batch_stride + (long long)(col / in_div) * a.in_stride +
                     (long long)(col % in_div) * a.in_stride2;
    float2 v[16];
#pragma unroll
    for (int q = 0; q < 16; q++) {
        const int n = j + T * q;
        float2 x = make_float2(0.f, 0.f);
        if (valid && n < a.L) x = ld_cplx<InC>(pin + n);
        v[q] = (a.in_scale != 1.f) ? cscale(x, a.in_scale) : x;
    }
    const int qnz = valid ? leading_slots<T>(a.L, j) : 0;
    // output pruning: a window at the origin keeps X[j + T q] for q < qout only
    const int qout = a.W0 == 0 ? leading_slots<T>(a.W, j) : 16;
    if constexpr (MODE == COL_INV) {
        BlockFft<N, true>::run(v, g, j, a.tw, qnz, qout);
    } else {
        // a forward size decrease keeps the first W outputs too; the correlation's forward
        // feeds every output to the product
        BlockFft<N, false>::run(v, g, j, a.tw, qnz, MODE == COL_FWD ? qout : 16);
    }
    if constexpr (MODE == COL_XCORR) {
        if (staged) {
            // block-uniform: thread 0 waits with the bounds and tells the block; a block whose
            // copy did not land records the timeout and leaves after one more bounded wait
            if (threadIdx.x == 0) {
                const bool ok = mbar_wait(img_bar, 0);
                img_ok = ok ? 1 : 0;
                if (!ok) {
                    if (a.err) atomicExch(a.err, kErrTimeout);
                    mbar_wait(img_bar, 0);
                }
            }
            __syncthreads();
            if (!img_ok) return;
            mbar_wait(img_bar, 0);
            const float sc = a.intra_kind == 3 ? a.intra_scale : 1.f;
#pragma unroll
            for (int q = 0; q < 16; q++) {
                const float2 p = conj_mul(v[q], lds_cplx<ImgC>(img_s + j + T * q));
                v[q] = (sc != 1.f) ? cscale(p, sc) : p;
            }
        } else if (a.intra_kind != 0) {
            const ImgC* pimg = static_cast<const ImgC*>(a.img) + bz * a.img_batch_stride + (long long)col * a.img_stride;
            const float sc = a.intra_kind == 3 ? a.intra_scale : 1.f;
#pragma unroll
            for (int q = 0; q < 16; q++) {
                float2 im = make_float2(0.f, 0.f);
                if (valid) im = ld_cplx_stream<ImgC>(pimg + j + T * q);
                float2 p = conj_mul(v[q], im);
                v[q] = (sc != 1.f) ? cscale(p, sc) : p;
            }
        }
        BlockFft<N, true>::run(v, g, j, a.tw, 16, qout);
    }
    const int out_div = a.out_div > 0 ? a.out_div : 1;
    const long long es = a.out_elem_stride > 0 ? a.out_elem_stride : 1;
    if constexpr (FPB > 1) {
        if (a.out_coalesce) {
            // every group parks its column in its own buffer (natural order), then item i of
            // the block stores element W0 + i / FPB of column c0 + i % FPB
            __syncthreads();
#pragma unroll
            for (int q = 0; q < 16; q++) g.base[phys(j + T * q)] = v[q];
            __syncthreads();
            const int c0 = blockIdx.x * FPB;
            const int cols_here = min(FPB, a.n_cols - c0);
            OutC* pout0 = static_cast<OutC*>(a.out) + bz * a.out_batch_stride +
                          (long long)(c0 / out_div) * a.out_stride + (long long)(c0 % out_div) * a.out_stride2;
            for (int i = threadIdx.x; i < a.W * FPB; i += T * FPB) {
                const int n = i / FPB, ff = i - n * FPB;
                if (ff < cols_here) {
                    const float2 x = smem[ff * G::STRIDE + phys(n + a.W0)];
                    st_cplx<OutC>(pout0 + ff + n * es, (a.out_scale != 1.f) ? cscale(x, a.out_scale) : x);
                }
            }
            return;
        }
    }
    if (valid) {
        OutC* pout = static_cast<OutC*>(a.out) + bz * a.out_batch_stride + (long long)(col / out_div) * a.out_stride +
                     (long long)(col % out_div) * a.out_stride2;
#pragma unroll
        for (int q = 0; q < 16; q++) {
            const int n = j + T * q - a.W0;
            if (n >= 0 && n < a.W) {
                const float2 x = (a.out_scale != 1.f) ? cscale(v[q], a.out_scale) : v[q];
                st_cplx<OutC>(pout + n * es, x);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Row C2R (inverse), two rows per complex FFT
// ---------------------------------------------------------------------------
struct RowInvArgs {
    const float2* in;      // batch entry g: in[g * in_batch_stride + k * in_pitch + r], k in [0, N/2], r < n_rows
    long long in_pitch;    // even
    long long in_batch_stride;
    int n_rows;
    void* out[kMaxBatch];  // real rows of batch entry g: row r at out[g] + r * out_pitch (elements)
    long long out_pitch;
    int W;                 // x outputs kept per row: x in [X0, X0 + W)
    float scale;           // post-op SCALE (1 = NOOP)
    const float2* tw;
    const float2* tw3;     // N = 3P: radix-3 pass twiddles (set by the launcher)
    int n_batch;           // batch entries in this launch (grid.y)
    int X0;
    // Fused peak search: if peaks is set, batch entry g's maximum over the retained
    // window and its first flat index (row * W + x) are folded into peaks[g] as a
    // peak_key(); with peaks_only the window itself is not written.
    unsigned long long* peaks;
    int peaks_only;            // the windows are not written (peak search or projection only)
    int peak_slot[kMaxBatch];  // batch entry g folds into peaks[peak_slot[g]]
    // Fused maximum projection across templates: if mip is set, every retained pixel
    // (row r, x) of batch entry g folds peak_key(value, mip_base + peak_slot[g]) into
    // mip[r * W + x] (the best value over the templates and its first template).
    unsigned long long* mip;
    int mip_base;
};

// Total order on (value, index) for a 64-bit atomicMax: larger value wins, and among
// equal values the smaller index (the first occurrence, as argmax returns it).
__device__ __forceinline__ unsigned long long peak_key(float v, unsigned int index) {
    const unsigned int b = __float_as_uint(v);
    const unsigned int ordered = (b & 0x80000000u) ? ~b : (b | 0x80000000u);
    return ((unsigned long long)ordered << 32) | (0xFFFFFFFFu - index);
}

template <int N, class OutT, int FPB>
__global__ void __launch_bounds__(FftShape<N>::T * FPB, (FftShape<N>::T * FPB <= 256) ? 4 : 2)
c2r_rows_kernel(RowInvArgs a) {
    using S = FftShape<N>;
    constexpr int T = S::T;
    constexpr int H = N / 2;
    extern __shared__ float2 smem[];
    using G = FftGroup<N, FPB, false>;
    const int f = threadIdx.x / T;
    const int j = threadIdx.x - f * T;
    G g(smem, f);
    float2* s = g.base;
    // batch entries in reverse order: the batched column pass wrote the last entries last, so
    // theirs are the columns still in L2
    const int gb = gridDim.y - 1 - blockIdx.y;
    // Gather rows (2 per FFT) and build Z[k] = A[k] + i B[k] over the full circle
    // from the half spectrum (A, B Hermitian).  The imaginary parts of the k = 0
    // and k = N/2 bins are dropped, as a C2R of a Hermitian spectrum does.
    // (H + 1) / T <= 9 items per thread: all of a thread's loads are issued before any of
    // them is used, so they are in flight together.
    // Item it of this thread is spectrum index k = k0 + T it of FFT ff0 (the block's item
    // stride T FPB is a multiple of FPB): one pointer, advanced by T rows per item.
    constexpr int kItemsPerThread = (FPB * (H + 1) + T * FPB - 1) / (T * FPB);
    const int ff0 = threadIdx.x % FPB;
    const int k0 = threadIdx.x / FPB;
    float4 ld[kItemsPerThread];
    {
        const int rr0 = 2 * (blockIdx.x * FPB + ff0);
        const bool two = rr0 + 1 < a.n_rows, one = rr0 < a.n_rows;
        const float2* p = a.in + (long long)gb * a.in_batch_stride + (long long)k0 * a.in_pitch + rr0;
        const long long step = (long long)T * a.in_pitch;
#pragma unroll
        for (int it = 0; it < kItemsPerThread; it++, p += step) {
            ld[it] = make_float4(0.f, 0.f, 0.f, 0.f);
            if (k0 + T * it <= H) {
                if (two) {
                    ld[it] = *reinterpret_cast<const float4*>(p);
                } else if (one) {
                    const float2 t = *p;
                    ld[it] = make_float4(t.x, t.y, 0.f, 0.f);
                }
            }
        }
    }
#pragma unroll
    for (int it = 0; it < kItemsPerThread; it++) {
        const int k = k0 + T * it;
        if (k <= H) {
            const float2 A = make_float2(ld[it].x, ld[it].y), B = make_float2(ld[it].z, ld[it].w);
            float2* sf = smem + ff0 * G::STRIDE;
            if (k == 0 || k == H) {
                sf[phys(k)] = make_float2(A.x, B.x);
            } else {
                sf[phys(k)] = make_float2(A.x - B.y, A.y + B.x);
                sf[phys(N - k)] = make_float2(A.x + B.y, B.x - A.y);
            }
        }
    }
    __syncthreads();
    float2 v[16];
#pragma unroll
    for (int q = 0; q < 16; q++) v[q] = s[phys(j + T * q)];
    // output pruning: a window at the origin keeps X[j + T q] for q < qout only
    BlockFft<N, true>::run(v, g, j, a.tw, 16, a.X0 == 0 ? leading_slots<T>(a.W, j) : 16);
    const int ra = 2 * (blockIdx.x * FPB + f);
    OutT* oa = static_cast<OutT*>(a.out[gb]) + (long long)ra * a.out_pitch;
    OutT* ob = oa + a.out_pitch;
    const bool has_a = ra < a.n_rows, has_b = ra + 1 < a.n_rows;
    if (!a.peaks_only) {
#pragma unroll
        for (int q = 0; q < 16; q++) {
            const int n = j + T * q - a.X0;
            if (n >= 0 && n < a.W) {
                if (has_a) st_real<OutT>(oa + n, v[q].x * a.scale);
                if (has_b) st_real<OutT>(ob + n, v[q].y * a.scale);
            }
        }
    }
    if (a.mip) {
        const unsigned int tmpl = (unsigned)(a.mip_base + a.peak_slot[gb]);
        unsigned long long* ma = a.mip + (long long)ra * a.W;
#pragma unroll
        for (int q = 0; q < 16; q++) {
            const int n = j + T * q - a.X0;
            if (n >= 0 && n < a.W) {
                if (has_a) atomicMax(ma + n, peak_key(v[q].x * a.scale, tmpl));
                if (has_b) atomicMax(ma + a.W + n, peak_key(v[q].y * a.scale, tmpl));
            }
        }
    }
    if (a.peaks) {
        unsigned long long best = 0;
#pragma unroll
        for (int q = 0; q < 16; q++) {
            const int n = j + T * q - a.X0;
            if (n >= 0 && n < a.W) {
                if (has_a) {
                    const unsigned long long k = peak_key(v[q].x * a.scale, (unsigned)(ra * a.W + n));
                    best = k > best ? k : best;
                }
                if (has_b) {
                    const unsigned long long k = peak_key(v[q].y * a.scale, (unsigned)((ra + 1) * a.W + n));
                    best = k > best ? k : best;
                }
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long other = __shfl_xor_sync(0xffffffffu, best, o);
            best = other > best ? other : best;
        }
        if ((threadIdx.x & 31) == 0 && best != 0) atomicMax(a.peaks + a.peak_slot[gb], best);
    }
}

}  // namespace ffb
