/*
 * fastfft_capi.h -- C ABI of the B200-native size-changing FFT library
 * (libfastfft_b200.so).  Plain pointers, sizes and integer codes only.
 *
 * Every entry point below replaces one piece of the reference's
 * FastFFT::FourierTransformer<ComputeBaseType, InputType, OtherImageType, Rank>
 * (reference: include/FastFFT.h:84-219, src/fastfft/FastFFT.cu:58-3379) and is what a
 * ctypes / cgo / JNI binding of that path would call.  The reference aborts on
 * user error (include/detail/checks_and_debug.h:86-87); here every call returns a
 * fastfft_status and the message of the last failure is kept per handle.
 *
 * Conventions (identical to the reference):
 *   - dims are logical (x, y, z); z = 1 for 2D.
 *   - real arrays use the FFTW pitch 2*(x/2+1) elements per row.
 *   - spectra are complex64 in the transposed layout [kz][kx][ky], ky contiguous,
 *     kx in [0, Nx/2]; for 2D that is [kx][ky].
 *   - forward sign -1, no normalisation (a round trip scales by Nx*Ny*Nz).
 *   - size decrease keeps the first outputs along each axis (window at the origin).
 *   - all work is asynchronous on the handle's stream (default cudaStreamPerThread).
 *   - an output pointer of NULL means "in place" (written over the input buffer,
 *     which must then hold the larger of the two sizes).
 */
#ifndef FASTFFT_B200_CAPI_H
#define FASTFFT_B200_CAPI_H

#include <stddef.h>

#if defined(__GNUC__)
#define FASTFFT_API __attribute__((visibility("default")))
#else
#define FASTFFT_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fastfft_plan_s* fastfft_handle;

typedef enum {
    FASTFFT_OK = 0,
    FASTFFT_ERR_INVALID_ARGUMENT = 1, /* null handle/pointer, bad dtype or op            */
    FASTFFT_ERR_INVALID_DIMS = 2,     /* dimension rules of ValidateDimensions violated  */
    FASTFFT_ERR_UNSUPPORTED = 3,      /* valid request that this library does not do     */
    FASTFFT_ERR_NOT_PLANNED = 4,      /* transform called before both plans were set    */
    FASTFFT_ERR_CUDA = 5,             /* a CUDA runtime call failed                      */
    FASTFFT_ERR_ALLOC = 6,            /* device allocation failed                        */
    FASTFFT_ERR_TIMEOUT = 7           /* a bounded device wait gave up                   */
} fastfft_status;

typedef enum {
    FASTFFT_DTYPE_F32 = 0,  /* float            (real)    */
    FASTFFT_DTYPE_F16 = 1,  /* __half           (real)    */
    FASTFFT_DTYPE_BF16 = 2, /* __nv_bfloat16    (real)    */
    FASTFFT_DTYPE_C64 = 3,  /* float2           (complex) */
    FASTFFT_DTYPE_C32H = 4, /* __half2          (complex) */
    FASTFFT_DTYPE_C32BF = 5 /* __nv_bfloat162   (complex) */
} fastfft_dtype;

/* Functor kinds, mirroring KernelFunction::my_functor (include/detail/functors.h:15-80). */
typedef enum {
    FASTFFT_OP_NOOP = 0,
    FASTFFT_OP_SCALE = 1,              /* x * scale (pre-op / post-op)                      */
    FASTFFT_OP_CONJ_MUL = 2,           /* conj(template) * image   (intra-op)              */
    FASTFFT_OP_CONJ_MUL_THEN_SCALE = 3 /* conj(template) * image * scale (intra-op)        */
} fastfft_op_kind;

typedef struct {
    int kind;    /* fastfft_op_kind */
    float scale; /* used by SCALE and CONJ_MUL_THEN_SCALE */
} fastfft_op;

/* FourierTransformer() constructor (FastFFT.cu:58-74).  compute_dtype must be F32;
 * input_dtype F32/F16/BF16 (real data, R2C / C2R transforms) or C64/C32H/C32BF (complex
 * data, C2C transforms: the reference's complex InputType, whose paths it leaves as stubs,
 * FastFFT.cu:369-391; spectra keep the [kx][ky] layout with kx over all N_x, rows have
 * pitch x, powers of two only); image_dtype C64/C32H/C32BF (OtherImageType); rank 2 or 3. */
FASTFFT_API fastfft_status fastfft_create(fastfft_handle* out, int compute_dtype, int input_dtype, int image_dtype,
                              int rank);
/* ~FourierTransformer() (FastFFT.cu:76-80, Deallocate :105-113). */
FASTFFT_API fastfft_status fastfft_destroy(fastfft_handle h);

/* SetForwardFFTPlan (FastFFT.cu:132-161).  is_padded must be 1 (the reference asserts it). */
FASTFFT_API fastfft_status fastfft_set_forward_plan(fastfft_handle h, size_t ix, size_t iy, size_t iz, size_t ox, size_t oy,
                                        size_t oz, int is_padded);
/* SetInverseFFTPlan (FastFFT.cu:180-200); the second of the two allocates the buffer
 * (AllocateBufferMemory, FastFFT.cu:210-227).  Transform lengths as ValidateDimensions
 * (FastFFT.cu:803-930): powers of two in [16, 8192]; real-input 2D plans also accept
 * 3 * 2^k (384 ... 6144), 5 * 2^k (640 ... 5120) and 7 * 2^k (896 ... 3584) per axis, and
 * every plan (real or complex input, 2D or 3D within 512 per axis) any other length in
 * [17, 4096] (extensions; the last run as chirp-z transforms on a power-of-two FFT of length
 * >= 2N - 1, without the fused peak search or projection). */
FASTFFT_API fastfft_status fastfft_set_inverse_plan(fastfft_handle h, size_t ix, size_t iy, size_t iz, size_t ox, size_t oy,
                                        size_t oz, int is_padded);

/* Work stream; NULL selects cudaStreamPerThread (the reference's only stream, usage.md:13). */
FASTFFT_API fastfft_status fastfft_set_stream(fastfft_handle h, void* cuda_stream);
/* First retained output (x, y, z) of an inverse size decrease; default (0, 0, 0), the
 * reference's origin-anchored window.  (N - W) / 2 per axis keeps the central W.  The
 * batched correlation's reduced-size path needs the origin at 0 and falls back to the
 * size-N kernels otherwise.  No reference counterpart. */
FASTFFT_API fastfft_status fastfft_set_inverse_output_origin(fastfft_handle h, size_t ox, size_t oy, size_t oz);
/* Output dtype of InvFFT / FwdImageInvFFT (default: input_dtype, as in the reference): real
 * for real-input plans, complex for complex-input plans. */
FASTFFT_API fastfft_status fastfft_set_output_dtype(fastfft_handle h, int dtype);
/* Storage of the spectrum FwdFFT writes: FASTFFT_DTYPE_C64 (default), C32H or C32BF, each
 * value multiplied by `scale` (1 = as computed) and rounded to nearest once in the last pass:
 * the normalised, quantised image spectrum that FwdImageInvFFT reads with a matching
 * image_dtype, written without a separate conversion pass (e.g. scale 1/N against FP16
 * overflow).  The output buffer then holds ReturnFwdOutputMemorySize() / 2 complex values of
 * that type.  No reference counterpart (the reference's spectra are FP32). */
FASTFFT_API fastfft_status fastfft_set_spectrum_output(fastfft_handle h, int dtype, float scale);
/* Rotationally averaged power of a square 2D half spectrum `spectrum` (complex64, the [kx][ky]
 * layout FwdFFT writes for an n x n transform): power[r] = mean |S|^2 over the elements of the
 * full spectrum at radius r = floor(sqrt(kx^2 + ky^2)) (signed ky, frequency-index units),
 * r = 0 .. n_bins - 1, the last bin also holding every larger radius; n_bins floats on the
 * device.  Uses a small work array of the plan (allocated on first use).  No reference
 * counterpart. */
FASTFFT_API fastfft_status fastfft_radial_power(fastfft_handle h, const void* spectrum, int n, float* power,
                                                int n_bins);
/* out = in x filter[r] for every element of a square 2D half spectrum (complex64 in, radius r
 * as in fastfft_radial_power, n_bins filter factors on the device): a band-pass, or whitening
 * with filter = 1 / sqrt(power).  `out` is written in the plan's spectrum storage and scale
 * (fastfft_set_spectrum_output); in place (out == in) only with complex64 storage.  No
 * reference counterpart. */
FASTFFT_API fastfft_status fastfft_apply_radial_filter(fastfft_handle h, const void* in, void* out, int n,
                                                       const float* filter, int n_bins);

/* FwdFFT(input, output, pre_op, intra_op) (FastFFT.h:165-170, FastFFT.cu:263-277).
 * Ops may be NULL (NOOP).  Output: complex64 spectrum [kz][kx][ky]. */
FASTFFT_API fastfft_status fastfft_fwd(fastfft_handle h, const void* input, void* output, const fastfft_op* pre_op,
                           const fastfft_op* intra_op);
/* InvFFT(input, output, intra_op, post_op) (FastFFT.h:172-177, FastFFT.cu:279-293). */
FASTFFT_API fastfft_status fastfft_inv(fastfft_handle h, const void* input, void* output, const fastfft_op* intra_op,
                           const fastfft_op* post_op);
/* FwdImageInvFFT(input, image_to_search, output, pre_op, intra_op, post_op)
 * (FastFFT.h:179-187, FastFFT.cu:295-313, Generic_Fwd_Image_Inv :609-798).
 * image_spectrum has the forward output's layout and the handle's image_dtype. */
FASTFFT_API fastfft_status fastfft_fwd_image_inv(fastfft_handle h, const void* input, const void* image_spectrum, void* output,
                                     const fastfft_op* pre_op, const fastfft_op* intra_op,
                                     const fastfft_op* post_op);

/* Many templates in one call: FwdImageInvFFT of inputs[i] against image_spectra[i] into
 * outputs[i] (NULL entries or a NULL array mean in place), i < n, all on the handle's
 * stream (pass the same image pointer n times to search one image).  The reference
 * correlates one template per FwdImageInvFFT call (FastFFT.cu:295-313); this is that
 * call repeated without a host round trip per template. */
FASTFFT_API fastfft_status fastfft_fwd_image_inv_many(fastfft_handle h, int n, const void* const* inputs,
                                                      const void* const* image_spectra, void* const* outputs,
                                                      const fastfft_op* pre_op, const fastfft_op* intra_op,
                                                      const fastfft_op* post_op);

/* fastfft_fwd_image_inv_many for templates of uneven sizes: template i is
 * template_dims[2i] x template_dims[2i+1] (x, y), no larger than the plan's forward input
 * size, with rows of pitch 2*(x/2+1); all share the plan's transform and window.  The
 * reference plans one size per FourierTransformer; no counterpart. */
FASTFFT_API fastfft_status fastfft_fwd_image_inv_many_sized(fastfft_handle h, int n, const void* const* inputs,
                                                            const int* template_dims,
                                                            const void* const* image_spectra, void* const* outputs,
                                                            const fastfft_op* pre_op, const fastfft_op* intra_op,
                                                            const fastfft_op* post_op);
/* Batched correlation with a fused peak search: peaks[i] (device memory, n values)
 * receives the maximum of template i's window and its first flat index
 * y * out_x + x, packed as ((ordered float bits) << 32) | (0xFFFFFFFF - index), where
 * ordered bits = bits | 0x80000000 for v >= 0 and ~bits for v < 0 (decode with
 * fastfft_decode_peak).  outputs NULL: the windows are not written at all (the window
 * write is the largest store of the correlation); otherwise they are written too.
 * template_dims may be NULL (plan size).  No reference counterpart (the reference's
 * callers search the returned window on their own). */
FASTFFT_API fastfft_status fastfft_fwd_image_inv_many_peaks(fastfft_handle h, int n, const void* const* inputs,
                                                            const int* template_dims,
                                                            const void* const* image_spectra, void* const* outputs,
                                                            unsigned long long* peaks, const fastfft_op* pre_op,
                                                            const fastfft_op* intra_op, const fastfft_op* post_op);
/* Batched correlation with a fused maximum projection across templates (the per-pixel
 * best score and best template of a template search): for every retained pixel (y, x) of
 * every template i of the call, mip[y * out_x + x] (device memory, out_x * out_y values)
 * is raised to the key of (score, index_base + i), packed as for the peak search with the
 * template number in place of the pixel index; the larger score wins and, on equal
 * scores, the smaller template number.  The array is not cleared: zero it once, then
 * stream any number of calls into it, numbering their templates with index_base.
 * outputs NULL: the windows are not written.  template_dims may be NULL (plan size).  No
 * reference counterpart. */
FASTFFT_API fastfft_status fastfft_fwd_image_inv_many_mip(fastfft_handle h, int n, const void* const* inputs,
                                                          const int* template_dims,
                                                          const void* const* image_spectra, void* const* outputs,
                                                          unsigned long long* mip, int index_base,
                                                          const fastfft_op* pre_op, const fastfft_op* intra_op,
                                                          const fastfft_op* post_op);
/* Host-side decode of one peaks[] or mip[] entry. */
FASTFFT_API void fastfft_decode_peak(unsigned long long key, float* value, unsigned int* index);

/* Templates per launch of the batched reduced-size path (1..64, default 16; lowered if the
 * fused column kernel's shared memory would not fit), and the value in effect. */
FASTFFT_API fastfft_status fastfft_set_templates_per_launch(fastfft_handle h, int n);
FASTFFT_API fastfft_status fastfft_templates_per_launch(fastfft_handle h, int* n);

/* Templates that one block of the batched fused column pass stages and transforms (0, the
 * default: a per-length choice measured on B200 -- 6 at length 1536, 4 at 1024, 8 elsewhere),
 * and the value in effect for the plan's correlation size.  No reference counterpart. */
FASTFFT_API fastfft_status fastfft_set_templates_per_block(fastfft_handle h, int n);
FASTFFT_API fastfft_status fastfft_templates_per_block(fastfft_handle h, int* n);

/* Groups of the batched reduced-size path in flight (1, the default, or 2).  With 2,
 * consecutive groups of templates alternate between the plan's stream and a second stream
 * of the plan, each with its own intermediate slices, so one group's row passes overlap the
 * other's fused column pass and a group's intermediates can stay in L2; the call still
 * completes in the plan's stream order.  No reference counterpart (the reference has no
 * batched call). */
FASTFFT_API fastfft_status fastfft_set_pipelined_groups(fastfft_handle h, int n);
FASTFFT_API fastfft_status fastfft_pipelined_groups(fastfft_handle h, int* n);

/* The batched call correlates at the smallest size M >= L + W - 1 per axis among powers of
 * two and 3 * 2^k when that is below the plan's N (template in [0, L),
 * window in [0, W)): every retained lag then reads image pixels in [0, L + W - 1) only, so
 * the size-M circular correlation against the spectrum of the image cropped to [0, M) gives
 * the same values as the size-N one.  This holds for the correlation intra-ops (CONJ_MUL,
 * CONJ_MUL_THEN_SCALE); calls with NOOP or SCALE (a round trip of the template, whose values
 * scale with the transform size) run at N.  Each distinct image in a call is prepared once.
 * force != 0 selects the size-N kernels instead.  No reference counterpart (the
 * reference aborts on a forward increase with an inverse decrease, FastFFT.cu:673-679). */
FASTFFT_API fastfft_status fastfft_set_full_size_correlation(fastfft_handle h, int force);

/* enable != 0 declares that an image spectrum does not change while it is in use: the
 * reduced spectrum prepared for an image address is then kept and reused by later calls
 * naming the same address (batched or single FwdImageInvFFT, which then also correlates at
 * the reduced size), instead of being prepared again in every call.  The caller must not
 * modify the spectrum behind that address while reuse is on (or must call this again,
 * which forgets the prepared image).  Changing the plan, the stream or the plan's settings
 * also forgets it.  Default off.  No reference counterpart. */
FASTFFT_API fastfft_status fastfft_set_image_reuse(fastfft_handle h, int enable);
/* enable != 0 runs the batched correlation's fused column pass at length 1536 along y on the
 * tensor cores (tcgen05.mma with FP32 accumulators in tensor memory): each column's forward
 * FFT, image product and inverse FFT as a four-step 48 x 32 DFT whose four stages are
 * BF16 split-precision matrix products (hi/lo parts, three products per stage; about 1e-5
 * relative L2 against FP64 instead of about 6e-7 for the FP32 form).  Applies to templates of
 * up to 512 rows with CONJ_MUL or CONJ_MUL_THEN_SCALE; every other pass and size keeps the
 * FP32 CUDA-core FFTs.  Default off.  No reference counterpart (the reference computes in
 * FP32). */
FASTFFT_API fastfft_status fastfft_set_tensor_core_dft(fastfft_handle h, int enable);
/* *active = 1 when the batched correlation of this plan runs the tensor-core pass (the option
 * is on, the plan correlates at length 1536 along y and its templates have at most 512
 * rows), else 0. */
FASTFFT_API fastfft_status fastfft_tensor_core_dft_active(fastfft_handle h, int* active);
/* Transform size {x, y} that fastfft_fwd_image_inv_many uses for this plan. */
FASTFFT_API fastfft_status fastfft_correlation_size(fastfft_handle h, int dims[2]);

/* 2D padded cross-correlation that allocates no device memory.  No counterpart in the
 * reference.  For callers that cannot allocate where they correlate: code inside a host
 * application whose memory pool owns the GPU's free memory, and steady-state loops that
 * must not stall on cudaMalloc/cudaFree (both synchronise the device).  The result is
 * the one FwdImageInvFFT gives for a plan (in_x, in_y, 1) -> (n_x, n_y, 1) ->
 * (out_x, out_y, 1) with a forward pad (or no change) and an inverse crop at the origin
 * (or no change): FP32 template rows of pitch 2*(in_x/2+1), a complex64 (float2) image
 * spectrum [kx][ky], an FP32 window of pitch 2*(out_x/2+1).
 * Limit: its two intermediate arrays live in one fixed device array of 24 MiB that every
 * GPU the library's device code has been loaded on holds until exit; sizes with
 * (n_x/2+1) * (round_up(in_y,4) + round_up(out_y,4)) * 8 bytes above it are rejected
 * with FASTFFT_ERR_UNSUPPORTED (4096^2 with a 384-row template and a 1024-row window
 * fits).  CUDA loads device code and data lazily, so the first call on a device is what
 * places that array, the twiddle tables and the kernels on it; it also looks up the
 * array's address and builds the twiddle tables (it synchronises).  Make one such call per
 * device at start-up, before a memory pool claims the device's free memory and before any
 * stream capture; later calls allocate nothing.  All calls share
 * the array and it keeps the last call's contents (every value a call reads is written
 * by that call first): calls that overlap on the GPU race.  cuda_stream NULL selects
 * cudaStreamPerThread.  Errors: fastfft_last_error(NULL). */
FASTFFT_API fastfft_status fastfft_fwd_image_inv_2d_noalloc(const float* input, int in_x, int in_y,
                                                            const void* image_spectrum, int n_x, int n_y,
                                                            float* output, int out_x, int out_y,
                                                            const fastfft_op* pre_op, const fastfft_op* intra_op,
                                                            const fastfft_op* post_op, void* cuda_stream);

/* ReturnInputMemorySize / ReturnFwdOutputMemorySize / ReturnInvOutputMemorySize
 * (FastFFT.h:194-204): element counts of InputType, FFTW-padded. */
FASTFFT_API fastfft_status fastfft_input_memory_size(fastfft_handle h, long long* n);
FASTFFT_API fastfft_status fastfft_fwd_output_memory_size(fastfft_handle h, long long* n);
FASTFFT_API fastfft_status fastfft_inv_output_memory_size(fastfft_handle h, long long* n);
/* Return{Fwd,Inv}{Input,Output}Dimensions (FastFFT.h:206-220): {x, y, z, w}, w = complex
 * elements along x after the R2C (set by ReturnPaddedMemorySize, FastFFT.h:363-404). */
FASTFFT_API fastfft_status fastfft_fwd_input_dims(fastfft_handle h, int dims[4]);
FASTFFT_API fastfft_status fastfft_fwd_output_dims(fastfft_handle h, int dims[4]);
FASTFFT_API fastfft_status fastfft_inv_input_dims(fastfft_handle h, int dims[4]);
FASTFFT_API fastfft_status fastfft_inv_output_dims(fastfft_handle h, int dims[4]);
/* Bytes of the internal work buffer (the reference's buffer_1/buffer_2 pair). */
FASTFFT_API fastfft_status fastfft_buffer_bytes(fastfft_handle h, long long* n);

/* Number of kernels this handle has launched (for launch accounting in benchmarks). */
FASTFFT_API fastfft_status fastfft_launch_count(fastfft_handle h, long long* n);
/* Per-pass device timing with CUDA events on the work stream, for up to max_calls
 * transform calls.  stop() waits for the events and returns the summed milliseconds of
 * pass 0/1/2 (row pass, column pass, row pass) over the recorded calls.  The reference
 * times with CUDA events in its test harness only (src/fastfft/Image.cuh:64-84). */
FASTFFT_API fastfft_status fastfft_profile_start(fastfft_handle h, int max_calls);
FASTFFT_API fastfft_status fastfft_profile_stop(fastfft_handle h, double* pass_ms, int n_pass, long long* n_calls);

/* Wait() (FastFFT.h:124-126): synchronise the handle's stream. */
FASTFFT_API fastfft_status fastfft_wait(fastfft_handle h);

/* Message of the last failed call on h ("" if none); static text for a NULL handle. */
FASTFFT_API const char* fastfft_last_error(fastfft_handle h);
FASTFFT_API const char* fastfft_status_string(int status);
/* Library version string. */
FASTFFT_API const char* fastfft_version(void);

#ifdef __cplusplus
}
#endif

#endif /* FASTFFT_B200_CAPI_H */
