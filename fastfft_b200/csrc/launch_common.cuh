// Shared helpers for the launcher translation units.
#pragma once

#include <atomic>

#include "fft3.cuh"
#include "kernels_2d.cuh"
#include "launch.h"

// Runtime N -> compile-time N.  FN<N>(args...) must return cudaError_t.
#define FFB_SIZE_SWITCH(n, FN, ...)                 \
    switch (n) {                                    \
        case 16: return FN<16>(__VA_ARGS__);        \
        case 32: return FN<32>(__VA_ARGS__);        \
        case 64: return FN<64>(__VA_ARGS__);        \
        case 128: return FN<128>(__VA_ARGS__);      \
        case 256: return FN<256>(__VA_ARGS__);      \
        case 512: return FN<512>(__VA_ARGS__);      \
        case 1024: return FN<1024>(__VA_ARGS__);    \
        case 2048: return FN<2048>(__VA_ARGS__);    \
        case 4096: return FN<4096>(__VA_ARGS__);    \
        case 8192: return FN<8192>(__VA_ARGS__);    \
        default: return cudaErrorInvalidValue;      \
    }

namespace ffb {

// FFTs per block: row passes use 512-thread blocks (two rows per FFT, so the
// transposed [kx][y] accesses cover whole 32-byte sectors at N = 4096); column
// passes use 256-thread blocks so two blocks fit per SM at up to 128 registers.
template <int N>
constexpr int row_fpb() {
    return FftShape<N>::T >= 512 ? 1 : 512 / FftShape<N>::T;
}
// Row C2R below N = 4096: 256-thread blocks, four per SM (64 registers); measured on B200 in
// the batched correlation: 0.90 instead of 0.99 us per template at 1024^2, 0.20 instead of 0.22
// at 256^2.  At 4096 (the image preparation and the size-N path) the 512-thread blocks stay.
template <int N>
constexpr int c2r_fpb() {
    return N >= 4096 ? row_fpb<N>() : (FftShape<N>::T >= 256 ? 1 : 256 / FftShape<N>::T);
}
// Row R2C likewise: 256-thread blocks below 4096 (0.81 instead of 0.85 us per template at
// 1024^2, 0.24 instead of 0.26 at 256^2).
template <int N>
constexpr int r2c_fpb() {
    return N >= 4096 ? row_fpb<N>() : (FftShape<N>::T >= 256 ? 1 : 256 / FftShape<N>::T);
}
template <int N>
constexpr int col_fpb() {
    return FftShape<N>::T >= 256 ? 1 : 256 / FftShape<N>::T;
}

}  // namespace ffb
