"""Radial operations for the image-spectrum preparation: rotationally averaged power
(fastfft_radial_power) and radial filtering (fastfft_apply_radial_filter) of a square 2D half
spectrum, against the FP64 oracle; whitening (filter = 1 / sqrt(power)) leaves a flat power.
"""
import numpy as np
import pytest

import fastfft_b200 as F
from oracle import fastfft_oracle as O
from tests._util import dev, empty, host

pytestmark = pytest.mark.gpu

N = 512


def spectrum(torch, seed, n=N):
    img = O.gaussian_blob_image(n, n_blobs=5, seed=seed)
    spec = O.image_spectrum_fp32(img)
    return spec, dev(torch, spec.view(np.float32))


def plan(n=N):
    ft = F.FourierTransformer()
    ft.SetForwardFFTPlan(n, n, 1, n, n, 1)
    ft.SetInverseFFTPlan(n, n, 1, n, n, 1)
    return ft


@pytest.mark.parametrize("n_bins", [N // 2 * 3 // 2 + 2, 100])
def test_radial_power_matches_oracle(torch_cuda, n_bins):
    torch = torch_cuda
    spec, d_spec = spectrum(torch, 71)
    power = torch.zeros(n_bins, dtype=torch.float32, device="cuda")
    ft = plan()
    ft.RadialPower(d_spec, N, power)
    torch.cuda.synchronize()
    ref = O.radial_power(spec.astype(np.complex128), N, n_bins)
    got = host(power).astype(np.float64)
    assert np.max(np.abs(got - ref) / np.maximum(ref, 1e-30)) <= 1e-5


@pytest.mark.parametrize("dtype,tol", [("complex64", 1e-6), ("complex32", 1e-3), ("complex_bf16", 8e-3)])
def test_radial_filter_matches_oracle(torch_cuda, dtype, tol):
    torch = torch_cuda
    spec, d_spec = spectrum(torch, 72)
    rng = np.random.default_rng(73)
    filt = rng.uniform(0.1, 2.0, N // 2 * 3 // 2 + 2).astype(np.float32)
    d_filt = dev(torch, filt)
    ft = plan()
    scale = 1.0 / N
    ft.SetSpectrumOutput(dtype, scale)
    out = empty(torch, d_spec.numel(), torch.float32)
    ft.ApplyRadialFilter(d_spec, out, N, d_filt)
    torch.cuda.synchronize()
    n_c = (N // 2 + 1) * N
    if dtype == "complex64":
        got = host(out)[: 2 * n_c].view(np.complex64)
    else:
        tdt = torch.float16 if dtype == "complex32" else torch.bfloat16
        got = out.view(tdt)[: 2 * n_c].float().cpu().numpy().view(np.complex64)
    ref = O.radial_filter(spec.astype(np.complex128), N, filt, scale).ravel()
    assert O.rel_l2(got, ref) <= tol


def test_in_place_filter_and_whitening(torch_cuda):
    torch = torch_cuda
    spec, d_spec = spectrum(torch, 74)
    n_bins = N // 2 * 3 // 2 + 2
    ft = plan()
    power = torch.zeros(n_bins, dtype=torch.float32, device="cuda")
    ft.RadialPower(d_spec, N, power)
    filt = torch.where(power > 0, power.rsqrt(), torch.zeros_like(power))
    ft.ApplyRadialFilter(d_spec, d_spec, N, filt)                      # in place, complex64
    flat = torch.zeros_like(power)
    ft.RadialPower(d_spec, N, flat)
    torch.cuda.synchronize()
    f = host(flat)
    assert np.allclose(f[host(power) > 0], 1.0, rtol=1e-4)
    ft.SetSpectrumOutput("complex32", 1.0)
    with pytest.raises(F.FastFFTError):
        ft.ApplyRadialFilter(d_spec, d_spec, N, filt)                  # in place needs complex64
