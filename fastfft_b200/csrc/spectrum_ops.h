// Arguments of the radial spectrum operations (spectrum_ops.cu).
#pragma once

#include <cuda_runtime.h>

namespace ffb {

struct RadialArgs {
    const float2* in;      // spectrum [kx][ky] of an n x n transform, pitch n, kx <= n / 2
    void* out;             // filtered spectrum, same layout, storage out_dtype
    int n;                 // transform edge
    int n_bins;
    const float* filter;   // n_bins factors
    float scale;
    double* sums;          // n_bins: weighted sums of |S|^2 (power pass)
    double* weights;       // n_bins: weights
};

}  // namespace ffb
