// The reference's cuFFT pad-then-transform recipe, as a comparator for bench.py (not part
// of the library): per template, clip it into the top-left corner of a zeroed N x N real
// buffer (FourierTransformer::ClipIntoTopLeft, src/fastfft/FastFFT.cu:1766-1778), an
// in-place cufftExecR2C, and an in-place cufftExecC2R whose load callback forms
// conj(template) x image x scale (the recipe of src/tests/padded_convolution_FastFFT_vs_cuFFT.cu:317-378,
// callback src/fastfft/Image.cu:315-343).  The full N x N output is written, as there.
// The callback is a device function pointer set with cufftXtSetCallback, as in the reference,
// which needs the static cuFFT library (the program is built with -rdc and libcufft_static).
//
// A standalone program (its own process and its own statically linked cuFFT):
//   cufft_recipe_bench <dir> <n> <L> <batch> <reps> <rows>
// reads <dir>/template.f32 (L x L, row pitch L) and <dir>/image_kykx.c64 (N x (N/2+1)
// complex64), correlates `batch` copies of the template per execution, times `reps`
// executions with CUDA events after a warm-up and writes the first template's correlation
// rows 0..rows-1 (N + 2 floats each) to <dir>/corr.f32; prints one JSON line.
#include <cuda_runtime.h>
#include <cufftXt.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <new>
#include <string>
#include <vector>

namespace {

struct CmpConjMulParams {
    const cufftComplex* image;
    unsigned long long image_elems;
    float scale;
};

// Load callback of the C2R: conj(template spectrum) x image spectrum x scale, the product of
// the reference's CB_complexConjMulLoad_32f (src/fastfft/Image.cu:315-325 with
// ComplexConjMulAndScale, include/detail/device_functions.h:10-15).
__device__ cufftComplex conj_mul_load(void* data_in, size_t offset, void* caller_info, void* shared_ptr) {
    const CmpConjMulParams* p = static_cast<const CmpConjMulParams*>(caller_info);
    const cufftComplex t = static_cast<const cufftComplex*>(data_in)[offset];
    const cufftComplex im = p->image[offset % p->image_elems];
    cufftComplex r;
    r.x = p->scale * (t.x * im.x + t.y * im.y);
    r.y = p->scale * (t.x * im.y - t.y * im.x);
    return r;
}
__device__ cufftCallbackLoadC d_conj_mul_load = conj_mul_load;

struct Recipe {
    int n = 0, batch = 0;
    cufftHandle fwd = 0, inv = 0;
    CmpConjMulParams* d_params = nullptr;
};

// Zero the padded N x (N + 2) rows and copy the L x L template (row pitch `pitch`) into the
// top-left corner; one thread per output element of a row, one block row per (row, batch).
__global__ void clip_into_top_left(const float* __restrict__ in, int L, long long pitch, long long in_batch,
                                   float* __restrict__ out, int n) {
    const int y = blockIdx.y;
    const int b = blockIdx.z;
    const long long opitch = n + 2;
    float* o = out + (long long)b * n * opitch + (long long)y * opitch;
    const float* src = in + (long long)b * in_batch + (long long)y * pitch;
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < n + 2; x += gridDim.x * blockDim.x)
        o[x] = (y < L && x < L) ? src[x] : 0.f;
}



int create(Recipe* r, int n, int batch) {
    r->n = n;
    r->batch = batch;
    int dims[2] = {n, n};
    int inembed[2] = {n, n + 2}, cembed[2] = {n, n / 2 + 1};
    if (cudaMalloc(&r->d_params, sizeof(CmpConjMulParams)) != cudaSuccess) return 2;
    size_t ws = 0;
    if (cufftCreate(&r->fwd) != CUFFT_SUCCESS || cufftCreate(&r->inv) != CUFFT_SUCCESS) return 3;
    cufftResult cr = cufftMakePlanMany(r->fwd, 2, dims, inembed, 1, n * (n + 2), cembed, 1, n * (n / 2 + 1),
                                       CUFFT_R2C, batch, &ws);
    if (cr != CUFFT_SUCCESS) return 400 + (int)cr;
    cr = cufftMakePlanMany(r->inv, 2, dims, cembed, 1, n * (n / 2 + 1), inembed, 1, n * (n + 2), CUFFT_C2R, batch,
                           &ws);
    if (cr != CUFFT_SUCCESS) return 500 + (int)cr;
    cufftCallbackLoadC h_cb = nullptr;
    if (cudaMemcpyFromSymbol(&h_cb, d_conj_mul_load, sizeof(h_cb)) != cudaSuccess) return 6;
    void* info = r->d_params;
    cr = cufftXtSetCallback(r->inv, reinterpret_cast<void**>(&h_cb), CUFFT_CB_LD_COMPLEX, &info);
    if (cr != CUFFT_SUCCESS) return 100 + (int)cr;
    return 0;
}

int run(Recipe* r, const float* templates, int L, float* work, cudaStream_t st) {
    clip_into_top_left<<<dim3(2, r->n, r->batch), 1024, 0, st>>>(templates, L, L, 0, work, r->n);
    if (cudaGetLastError() != cudaSuccess) return 1;
    if (cufftSetStream(r->fwd, st) != CUFFT_SUCCESS || cufftSetStream(r->inv, st) != CUFFT_SUCCESS) return 2;
    if (cufftExecR2C(r->fwd, work, reinterpret_cast<cufftComplex*>(work)) != CUFFT_SUCCESS) return 3;
    if (cufftExecC2R(r->inv, reinterpret_cast<cufftComplex*>(work), work) != CUFFT_SUCCESS) return 4;
    return 0;
}

std::vector<char> read_all(const char* path) {
    std::vector<char> v;
    FILE* f = std::fopen(path, "rb");
    if (!f) return v;
    std::fseek(f, 0, SEEK_END);
    v.resize((size_t)std::ftell(f));
    std::fseek(f, 0, SEEK_SET);
    if (std::fread(v.data(), 1, v.size(), f) != v.size()) v.clear();
    std::fclose(f);
    return v;
}

int fail(const char* what, int code) {
    std::printf("{\"error\": \"%s\", \"code\": %d}\n", what, code);
    return 1;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 7) return fail("usage: cufft_recipe_bench <dir> <n> <L> <batch> <reps> <rows>", 2);
    const std::string dir = argv[1];
    const int n = std::atoi(argv[2]), L = std::atoi(argv[3]), batch = std::atoi(argv[4]), reps = std::atoi(argv[5]);
    const int rows = std::atoi(argv[6]);
    if (n < 16 || L < 1 || L > n || batch < 1 || reps < 1 || rows < 1 || rows > n) return fail("bad arguments", 2);
    const std::vector<char> tpl = read_all((dir + "/template.f32").c_str());
    const std::vector<char> img = read_all((dir + "/image_kykx.c64").c_str());
    const size_t img_bytes = (size_t)n * (n / 2 + 1) * 8;
    if (tpl.size() != (size_t)L * L * 4 || img.size() != img_bytes) return fail("inputs", 3);
    float* d_t = nullptr;
    void* d_img = nullptr;
    float* d_work = nullptr;
    const size_t work_elems = (size_t)batch * n * (n + 2);
    if (cudaMalloc(&d_t, tpl.size()) != cudaSuccess || cudaMalloc(&d_img, img_bytes) != cudaSuccess ||
        cudaMalloc(&d_work, work_elems * 4) != cudaSuccess)
        return fail("cudaMalloc", 4);
    cudaMemcpy(d_t, tpl.data(), tpl.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(d_img, img.data(), img_bytes, cudaMemcpyHostToDevice);
    Recipe r;
    int rc = create(&r, n, batch);
    if (rc != 0) return fail("plan or callback", rc);
    // the reference scales by FT_normalization_factor^2; here 1, the unnormalised product
    CmpConjMulParams p{static_cast<const cufftComplex*>(d_img), (unsigned long long)n * (n / 2 + 1), 1.f};
    cudaMemcpy(r.d_params, &p, sizeof(p), cudaMemcpyHostToDevice);
    cudaStream_t st;
    cudaStreamCreate(&st);
    for (int i = 0; i < 3; i++)
        if ((rc = run(&r, d_t, L, d_work, st)) != 0) return fail("run", rc);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, st);
    for (int i = 0; i < reps; i++) run(&r, d_t, L, d_work, st);
    cudaEventRecord(e1, st);
    if (cudaEventSynchronize(e1) != cudaSuccess) return fail("timed run", 6);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    // first template's correlation rows [0, rows) (pitch n + 2), for the accuracy check
    std::vector<float> out((size_t)rows * (n + 2));
    cudaMemcpy(out.data(), d_work, out.size() * 4, cudaMemcpyDeviceToHost);
    FILE* f = std::fopen((dir + "/corr.f32").c_str(), "wb");
    if (!f || std::fwrite(out.data(), 4, out.size(), f) != out.size()) return fail("write", 7);
    std::fclose(f);
    std::printf("{\"ms_per_execution\": %.6f, \"templates_per_execution\": %d, \"reps\": %d}\n", ms / reps, batch,
                reps);
    cufftDestroy(r.fwd);
    cufftDestroy(r.inv);
    return 0;
}
