// Host-only check of the C++ drop-in header: plans and size queries (no GPU needed).
#define FASTFFT_B200_THROW
#include <cstdio>
#include <stdexcept>

#include "FastFFT.h"

// the functor kinds keep the reference's enumerator values (include/detail/concepts.h:22-25)
namespace KF = FastFFT::KernelFunction;
static_assert(KF::NOOP == 0 && KF::SCALE == 1 && KF::CONJ_MUL == 2 && KF::CONJ_MUL_THEN_SCALE == 3,
              "IKF_t values differ from the reference's");
static_assert(int(KF::SCALE) == int(FASTFFT_OP_SCALE) && int(KF::CONJ_MUL) == int(FASTFFT_OP_CONJ_MUL) &&
                  int(KF::CONJ_MUL_THEN_SCALE) == int(FASTFFT_OP_CONJ_MUL_THEN_SCALE),
              "IKF_t values differ from the C ABI's op kinds");

int main(int argc, char**) {
    FastFFT::FourierTransformer<float, float, float2, 2> ft;
    ft.SetForwardFFTPlan(384, 384, 1, 4096, 4096, 1, true);
    ft.SetInverseFFTPlan(4096, 4096, 1, 1024, 1024, 1, true);
    short4 o = ft.ReturnFwdOutputDimensions();
    std::printf("%d %d %d %d %d %d %d %d\n", ft.ReturnInputMemorySize(), ft.ReturnFwdOutputMemorySize(),
                ft.ReturnInvOutputMemorySize(), (int)o.x, (int)o.y, (int)o.z, (int)o.w,
                (int)ft.ReturnInvOutputDimensions().w);
    if (argc > 99) {  // compiled but never run here: type-checks the batched extensions
        FastFFT::KernelFunction::my_functor<float, 4, FastFFT::KernelFunction::CONJ_MUL> conj_mul;
        ft.FwdImageInvFFTMany(0, nullptr, nullptr, nullptr, nullptr, conj_mul, nullptr);
        ft.FwdImageInvFFTManyMip(0, nullptr, nullptr, nullptr, nullptr, nullptr, 0, nullptr, conj_mul, nullptr);
        ft.SetImageReuse(true);
        ft.SetTensorCoreDFT(true);
        ft.SetSpectrumOutput(FASTFFT_DTYPE_C32BF, 1.f / 4096);
    }
    FastFFT::FourierTransformer<float, __half, __half2, 3> ft3;
    ft3.SetForwardFFTPlan(64, 64, 64, 256, 256, 256);
    try {
        ft3.SetInverseFFTPlan(256, 256, 256, 1024, 1024, 1024);  // > 512 in 3D
        std::printf("no error\n");
        return 1;
    } catch (const std::runtime_error& e) {
        std::printf("rejected: %s\n", e.what());
    }
    return 0;
}
