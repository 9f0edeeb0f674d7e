// Runs transforms through the C++ drop-in header exactly as a reference caller would
// (FourierTransformer<float, float, float2, 2>, functor objects, default stream, Wait()),
// on inputs the test writes to a directory, and writes the results back there:
//   cfg1: 64x64 -> 512x512 FwdFFT (pre-op SCALE 0.5) into a spectrum buffer, then the
//         512x512 InvFFT of that spectrum;
//   cfg2: FwdFFT of a 4096x4096 image (its spectrum is the image to search), then
//         FwdImageInvFFT of a 384x384 template zero-padded to 4096x4096, cropped to the
//         1024x1024 window (NOOP, CONJ_MUL, NOOP), as in the reference's
//         padded_convolution_FastFFT_vs_cuFFT.cu.
// Usage: shim_transforms <dir>
#include <cstdio>
#include <string>
#include <vector>

#include "FastFFT.h"

namespace KF = FastFFT::KernelFunction;

static std::vector<float> read_file(const std::string& path, size_t n) {
    std::vector<float> v(n, 0.f);
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f || std::fread(v.data(), sizeof(float), n, f) != n) {
        std::fprintf(stderr, "cannot read %zu floats from %s\n", n, path.c_str());
        std::exit(2);
    }
    std::fclose(f);
    return v;
}

static void write_file(const std::string& path, const std::vector<float>& v) {
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f || std::fwrite(v.data(), sizeof(float), v.size(), f) != v.size()) {
        std::fprintf(stderr, "cannot write %s\n", path.c_str());
        std::exit(2);
    }
    std::fclose(f);
}

static void cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        std::fprintf(stderr, "%s: %s\n", what, cudaGetErrorString(e));
        std::exit(3);
    }
}

static float* to_device(const std::vector<float>& h, size_t n) {
    float* d = nullptr;
    cuda_check(cudaMalloc(&d, n * sizeof(float)), "cudaMalloc");
    cuda_check(cudaMemset(d, 0, n * sizeof(float)), "cudaMemset");
    cuda_check(cudaMemcpy(d, h.data(), h.size() * sizeof(float), cudaMemcpyHostToDevice), "upload");
    return d;
}

static std::vector<float> to_host(const float* d, size_t n) {
    std::vector<float> h(n);
    cuda_check(cudaMemcpy(h.data(), d, n * sizeof(float), cudaMemcpyDeviceToHost), "download");
    return h;
}

int main(int argc, char** argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s <dir>\n", argv[0]);
        return 2;
    }
    const std::string dir = argv[1];

    // cfg1: forward size increase and a no-change inverse
    {
        FastFFT::FourierTransformer<float, float, float2, 2> ft;
        ft.SetForwardFFTPlan(64, 64, 1, 512, 512, 1, true);
        ft.SetInverseFFTPlan(512, 512, 1, 512, 512, 1, true);
        const size_t n_in = ft.ReturnInputMemorySize(), n_spec = ft.ReturnFwdOutputMemorySize();
        const size_t n_out = ft.ReturnInvOutputMemorySize();
        float* d_in = to_device(read_file(dir + "/cfg1_in.f32", n_in), n_in);
        float* d_spec = to_device({}, n_spec);
        float* d_out = to_device({}, n_out);
        KF::my_functor<float, 2, KF::SCALE> half(0.5f);
        ft.FwdFFT(d_in, d_spec, half);
        ft.InvFFT(d_spec, d_out);
        ft.Wait();
        write_file(dir + "/cfg1_spec.f32", to_host(d_spec, n_spec));
        write_file(dir + "/cfg1_out.f32", to_host(d_out, n_out));
        cudaFree(d_in);
        cudaFree(d_spec);
        cudaFree(d_out);
    }

    // cfg2: the image spectrum from the transformer's own FwdFFT, then the fused correlation
    {
        FastFFT::FourierTransformer<float, float, float2, 2> prep;
        prep.SetForwardFFTPlan(4096, 4096, 1, 4096, 4096, 1, true);
        prep.SetInverseFFTPlan(4096, 4096, 1, 4096, 4096, 1, true);
        const size_t n_img = prep.ReturnInputMemorySize(), n_img_spec = prep.ReturnFwdOutputMemorySize();
        float* d_img = to_device(read_file(dir + "/cfg2_image.f32", n_img), n_img);
        float* d_img_spec = to_device({}, n_img_spec);
        prep.FwdFFT(d_img, d_img_spec);
        prep.Wait();

        FastFFT::FourierTransformer<float, float, float2, 2> ft;
        ft.SetForwardFFTPlan(384, 384, 1, 4096, 4096, 1, true);
        ft.SetInverseFFTPlan(4096, 4096, 1, 1024, 1024, 1, true);
        const size_t n_in = ft.ReturnInputMemorySize(), n_out = ft.ReturnInvOutputMemorySize();
        float* d_t = to_device(read_file(dir + "/cfg2_template.f32", n_in), n_in);
        float* d_win = to_device({}, n_out);
        KF::my_functor<float, 0, KF::NOOP> noop;
        KF::my_functor<float, 4, KF::CONJ_MUL> conj_mul;
        ft.FwdImageInvFFT(d_t, reinterpret_cast<float2*>(d_img_spec), d_win, noop, conj_mul, noop);
        ft.Wait();
        write_file(dir + "/cfg2_window.f32", to_host(d_win, n_out));
        cudaFree(d_img);
        cudaFree(d_img_spec);
        cudaFree(d_t);
        cudaFree(d_win);
    }
    std::printf("ok\n");
    return 0;
}
