"""fastfft_b200: B200-native (sm_100a) size-changing FFTs and padded cross-correlation.

A drop-in for the FourierTransformer path of FastFFT: zero-padded forward real FFTs,
cropped inverse FFTs and the fused forward -> conj-multiply -> inverse correlation,
computed by hand-written CUDA kernels in libfastfft_b200.so (C ABI:
include/fastfft_capi.h).
"""
from ._capi import FastFFTError, LIB_PATH
from .transformer import FourierTransformer, KernelFunction, decode_peaks

__all__ = ["FourierTransformer", "KernelFunction", "FastFFTError", "LIB_PATH", "decode_peaks"]
