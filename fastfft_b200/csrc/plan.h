// Plan state behind a fastfft_handle (the reference keeps the same state as members of
// FourierTransformer, include/FastFFT.h:319-362 and :680-732).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <string>

namespace ffb {

struct Dims {
    long long x = 0, y = 0, z = 0;
    long long w = 0;  // complex elements along x after an R2C (ReturnPaddedMemorySize)
};

enum class SizeChange { Increase = 0, Decrease = 1, NoChange = 2 };

}  // namespace ffb

struct fastfft_plan_s {
    int compute_dtype = 0;
    int input_dtype = 0;
    int output_dtype = 0;
    int image_dtype = 3;
    int rank = 2;
    int device = 0;

    ffb::Dims fwd_in, fwd_out, inv_in, inv_out;
    bool fwd_set = false, inv_set = false, validated = false;
    ffb::SizeChange fwd_change = ffb::SizeChange::NoChange;
    ffb::SizeChange inv_change = ffb::SizeChange::NoChange;
    // first retained output per axis of an inverse size decrease (the reference keeps
    // the window at the origin; fastfft_set_inverse_output_origin moves it)
    long long org_x = 0, org_y = 0, org_z = 0;

    // ReturnInputMemorySize / ReturnFwdOutputMemorySize / ReturnInvOutputMemorySize and
    // compute_memory_wanted_ (element counts, include/FastFFT.h:194-204, :363-404)
    long long input_mem = 0, fwd_out_mem = 0, inv_out_mem = 0, compute_mem = 0;

    // work buffer: region A (forward row-pass output) then region B (inverse
    // column-pass output); pitches in complex elements
    void* buffer = nullptr;
    size_t buffer_bytes = 0;
    long long pitch_a = 0, bytes_a = 0, pitch_b = 0, bytes_b = 0;

    // Reduced-size correlation (2D, forward pad + inverse crop): with the template in
    // [0, L) and the window in [0, W) per axis, every valid lag reads only image pixels
    // [0, L + W - 1), so the size-N circular correlation equals a size-M one with
    // M = pow2 >= L + W - 1, computed against the spectrum of the image cropped to
    // [0, M) (prepared once per image, region C).
    bool red_ok = false;
    long long red_mx = 0, red_my = 0;
    long long bytes_c = 0;     // prep work (max of the two column-major stages) + real crop + reduced spectrum
    long long off_c_real = 0, off_c_spec = 0;
    bool force_full_size = false;  // fastfft_set_full_size_correlation
    // fastfft_set_image_reuse: the image spectrum at a given address is declared unchanged,
    // so the reduced spectrum prepared for prepared_image (still in region C) is reused
    // when the next call names the same address; cleared whenever region C may have been
    // rewritten or the work moved to another stream.
    bool image_reuse = false;
    bool tc_dft = false;            // fastfft_set_tensor_core_dft
    double* radial_scratch = nullptr;  // fastfft_radial_power's sums (2 x radial_scratch_bins)
    int radial_scratch_bins = 0;
    int spec_dtype = 3;             // fastfft_set_spectrum_output: FwdFFT's spectrum storage
    float spec_scale = 1.f;         //   and scale
    const void* prepared_image = nullptr;
    long long prepared_mx = 0, prepared_my = 0;   // the size it was prepared at
    int red_batch = 16;             // templates per launch in the reduced-size path
    int red_batch_request = 16;     // fastfft_set_templates_per_launch (bounded by shared memory)
    int tpb_request = 0;            // fastfft_set_templates_per_block (0: built-in choice per length)
    long long red_t1_stride = 0, red_t2_stride = 0;  // complex elements per template slice
    long long off_c_t1 = 0, off_c_t2 = 0;
    int* dev_err = nullptr;  // device status word of bounded waits (inside the work buffer)

    cudaStream_t stream = cudaStreamPerThread;
    std::string last_error;

    // The image preparation of the reduced-size path runs on a second stream of this plan
    // (higher priority), forked from `stream` after all earlier work and joined back before
    // the first fused column pass that reads the prepared spectrum, so that it overlaps the
    // templates' row R2C (which does not read the image).  Null when it could not be created:
    // the preparation then runs on `stream`.
    cudaStream_t prep_stream = nullptr;
    cudaEvent_t prep_fork = nullptr, prep_join = nullptr;
    int prep_device = -1;
    bool prep_join_pending = false;  // prep_join recorded and not yet waited on by `stream`

    // Pipelined template groups (fastfft_set_pipelined_groups): with 2, consecutive groups of
    // the reduced-size correlation alternate between `stream` and pipe_stream, each with its
    // own slices of region C, so that one group's row passes overlap the other's column pass
    // and each group's intermediates are small enough to stay in L2.  pipe_stream is forked
    // from `stream` at the start of a call and joined back at its end.
    int pipe_groups = 1;
    cudaStream_t pipe_stream = nullptr;
    cudaEvent_t pipe_fork = nullptr, pipe_join = nullptr;
    bool prep_join_pending_pipe = false;  // prep_join not yet waited on by pipe_stream
    bool pipe_active = false;             // pipe_stream forked in the current call, not yet joined

    // kernels launched through this handle (fastfft_launch_count)
    long long launches = 0;

    // optional per-pass timing: events recorded before the first pass and after each
    // pass of every transform call while profiling is on (fastfft_profile_start/stop)
    static constexpr int kProfMarks = 4;
    cudaEvent_t* prof_events = nullptr;
    int prof_capacity = 0;  // calls
    int prof_calls = 0;
    int prof_mark = 0;      // next mark within the current call
};
