// cuFFT load callback of the cuFFT comparator (compiled to LTO-IR and handed to
// cufftXtSetJITCallback): the C2R's input element is conj(template spectrum) x image
// spectrum x scale, the same product as the reference's CB_complexConjMulLoad_32f
// (src/fastfft/Image.cu:315-325 with ComplexConjMulAndScale, include/detail/device_functions.h:10-15).
// Not part of the library: it only serves bench.py's comparator.
#include <cufftXt.h>

struct CmpConjMulParams {
    const cufftComplex* image;     // [ky][kx] half spectrum, N x (N/2 + 1)
    unsigned long long image_elems;
    float scale;
};

extern "C" __device__ cufftComplex cmp_conj_mul_load(void* data_in, unsigned long long offset, void* caller_info,
                                                     void* shared_ptr) {
    const CmpConjMulParams* p = static_cast<const CmpConjMulParams*>(caller_info);
    const cufftComplex t = static_cast<const cufftComplex*>(data_in)[offset];
    const cufftComplex im = p->image[offset % p->image_elems];
    cufftComplex r;
    r.x = p->scale * (t.x * im.x + t.y * im.y);
    r.y = p->scale * (t.x * im.y - t.y * im.x);
    return r;
}
