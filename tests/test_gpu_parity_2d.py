"""GPU parity of the 2D path against the FP64 host oracle, through the C ABI.

Bars: relative L2 <= 1e-5 (FP32 path vs FP64), bit-exact results for the
reference's known-answer tests (impulse, constant, impulse convolution, functor
scaling), bit-exact peak index for the cross-correlation window.
"""
import numpy as np
import pytest

import fastfft_b200 as F
from fastfft_b200 import KernelFunction as KF
from oracle import fastfft_oracle as O
from tests._util import RTOL_L2_FP32, RTOL_MAX_FP32, dev, empty, host, random_real, spectrum_view

pytestmark = pytest.mark.gpu


def make(fin, fout, iout, input_dtype="float32", image_dtype="complex64"):
    ft = F.FourierTransformer(input_dtype=input_dtype, image_dtype=image_dtype, rank=2)
    ft.SetForwardFFTPlan(*fin, *fout)
    ft.SetInverseFFTPlan(*fout, *iout)
    return ft


def run_fwd(torch, ft, x_host, fin, fout, in_place=False, pre_op=None):
    n_in, n_out = ft.ReturnInputMemorySize(), ft.ReturnFwdOutputMemorySize()
    xin = dev(torch, O.real_to_padded(x_host, fin), max(n_in, n_out) if in_place else n_in)
    if in_place:
        ft.FwdFFT(xin, None, pre_op)
        out = xin
    else:
        out = empty(torch, n_out, torch.float32)
        ft.FwdFFT(xin, out, pre_op)
    return spectrum_view(out, fout)


FWD_CASES = [
    ((16, 16, 1), (16, 16, 1)),
    ((32, 32, 1), (32, 32, 1)),
    ((64, 64, 1), (64, 64, 1)),
    ((128, 128, 1), (128, 128, 1)),
    ((256, 256, 1), (256, 256, 1)),
    ((512, 512, 1), (512, 512, 1)),
    ((1024, 1024, 1), (1024, 1024, 1)),
    ((2048, 2048, 1), (2048, 2048, 1)),
    ((4096, 4096, 1), (4096, 4096, 1)),
    ((8192, 32, 1), (8192, 32, 1)),         # 8192-point rows
    ((32, 8192, 1), (32, 8192, 1)),         # 8192-point columns
    ((64, 64, 1), (512, 512, 1)),           # 64^2 zero-padded into a 512^2 transform
    ((384, 384, 1), (4096, 4096, 1)),       # template padding of the 4096^2 correlation
    ((100, 37, 1), (256, 128, 1)),          # non-power-of-two inputs, rectangular
    ((48, 80, 1), (128, 256, 1)),
    ((1, 1, 1), (64, 64, 1)),
    ((512, 512, 1), (128, 128, 1)),         # forward decrease: first outputs kept
    ((256, 64, 1), (64, 16, 1)),
]


@pytest.mark.parametrize("fin,fout", FWD_CASES)
def test_forward_matches_oracle(torch_cuda, fin, fout):
    torch = torch_cuda
    x = random_real((fin[1], fin[0]), seed=fin[0] * 131 + fout[0])
    ft = make(fin, fout, fout)
    got = run_fwd(torch, ft, x, fin, fout)
    ref = O.fwd(O.real_to_padded(x, fin), fin, fout)
    assert O.rel_l2(got, ref) <= RTOL_L2_FP32
    assert O.rel_max(got, ref) <= RTOL_MAX_FP32


@pytest.mark.parametrize("fin,fout", [((64, 64, 1), (512, 512, 1)), ((256, 256, 1), (256, 256, 1))])
def test_forward_in_place_equals_out_of_place(torch_cuda, fin, fout):
    torch = torch_cuda
    x = random_real((fin[1], fin[0]), seed=3)
    ft = make(fin, fout, fout)
    a = run_fwd(torch, ft, x, fin, fout, in_place=False)
    b = run_fwd(torch, ft, x, fin, fout, in_place=True)
    assert np.array_equal(a, b)


INV_CASES = [
    ((16, 16, 1), (16, 16, 1)),
    ((64, 64, 1), (64, 64, 1)),
    ((512, 512, 1), (512, 512, 1)),
    ((2048, 2048, 1), (2048, 2048, 1)),
    ((4096, 4096, 1), (4096, 4096, 1)),
    ((4096, 4096, 1), (1024, 1024, 1)),     # crop to the correlation window
    ((256, 128, 1), (100, 37, 1)),          # non-power-of-two output window
    ((8192, 32, 1), (8192, 32, 1)),
    ((32, 8192, 1), (32, 8192, 1)),
]


@pytest.mark.parametrize("iin,iout", INV_CASES)
def test_inverse_matches_oracle(torch_cuda, iin, iout):
    torch = torch_cuda
    rng = np.random.default_rng(iin[0] + 7 * iout[0])
    w, _ = O.padded_x(iin[0])
    spec = (rng.standard_normal((1, w, iin[1])) + 1j * rng.standard_normal((1, w, iin[1]))).astype(np.complex64)
    ft = make(iin, iin, iout)
    sin = dev(torch, spec.view(np.float32))
    out = empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32)
    ft.InvFFT(sin, out)
    got = O.real_from_padded(host(out), iout)
    ref = O.real_from_padded(O.inv(spec, iin, iout, out_dtype=np.float64), iout)
    assert O.rel_l2(got, ref) <= RTOL_L2_FP32
    assert O.rel_max(got, ref) <= RTOL_MAX_FP32


def test_round_trip_64_in_512(torch_cuda):
    """64x64 N(0,1) zero-padded into a 512^2 R2C, then the 512^2 C2R."""
    torch = torch_cuda
    fin, fout = (64, 64, 1), (512, 512, 1)
    x = random_real((64, 64), seed=O.SEED_BASE + 0)
    ft = make(fin, fout, fout)
    n_max = max(ft.ReturnInputMemorySize(), ft.ReturnFwdOutputMemorySize(), ft.ReturnInvOutputMemorySize())
    buf = dev(torch, O.real_to_padded(x, fin), n_max)
    ft.FwdFFT(buf)
    spec_gpu = spectrum_view(buf, fout).copy()
    ft.InvFFT(buf)
    back = O.real_from_padded(host(buf), fout)
    spec_ref = O.fwd(O.real_to_padded(x, fin), fin, fout)
    assert O.rel_l2(spec_gpu, spec_ref) <= RTOL_L2_FP32
    ref = np.zeros((1, 512, 512))
    ref[0, :64, :64] = x * 512 * 512
    assert O.rel_l2(back, ref) <= RTOL_L2_FP32


# ---------------------------------------------------------------------------
# Known-answer tests of the reference, bit-exact on the GPU
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("n_in,n_out", [(32, 32), (64, 512), (128, 4096), (4096, 4096), (16, 8192)])
def test_kat_unit_impulse(torch_cuda, n_in, n_out):
    torch = torch_cuda
    fin, fout = (n_in, n_in, 1), (n_out, n_out, 1)
    x = np.zeros((n_in, n_in), np.float32)
    x[0, 0] = 1.0
    ft = make(fin, fout, fout)
    spec = run_fwd(torch, ft, x, fin, fout)
    assert np.all(spec == np.complex64(1.0))                    # every coefficient exactly 1
    n_max = max(ft.ReturnInputMemorySize(), ft.ReturnInvOutputMemorySize())
    buf = dev(torch, spec.view(np.float32), n_max)
    ft.InvFFT(buf)
    r = O.real_from_padded(host(buf), fout)
    assert r[0, 0, 0] == n_out * n_out
    assert np.count_nonzero(r) == 1                              # sum == Nx*Ny exactly


@pytest.mark.parametrize("n", [64, 512, 4096])
def test_kat_constant_image(torch_cuda, n):
    torch = torch_cuda
    fin = (n, n, 1)
    ft = make(fin, fin, fin)
    spec = run_fwd(torch, ft, np.ones((n, n), np.float32), fin, fin)
    assert spec[0, 0, 0] == np.complex64(n * n)
    flat = spec.ravel()
    assert np.count_nonzero(flat[1:]) == 0


@pytest.mark.parametrize("n_in,n_out,w", [(64, 64, 64), (64, 512, 512), (384, 4096, 4096), (384, 4096, 1024)])
def test_kat_impulse_convolution(torch_cuda, n_in, n_out, w):
    """Template impulse 2.0, image impulse 3.0: out[0] = N^2 * 6, every other pixel 0."""
    torch = torch_cuda
    fin, fout, iout = (n_in, n_in, 1), (n_out, n_out, 1), (w, w, 1)
    t = np.zeros((n_in, n_in), np.float32)
    t[0, 0] = 2.0
    img = np.full((1, n_out // 2 + 1, n_out), 3.0, np.complex64)  # spectrum of an impulse 3.0
    ft = make(fin, fout, iout)
    tin = dev(torch, O.real_to_padded(t, fin))
    out = empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32)
    ft.FwdImageInvFFT(tin, dev(torch, img.view(np.float32)), out, KF.noop(), KF.conj_mul(), KF.noop())
    r = O.real_from_padded(host(out), iout)
    assert r[0, 0, 0] == n_out * n_out * 6.0
    assert np.count_nonzero(r) == 1


@pytest.mark.parametrize("n", [64, 512])
def test_kat_functor_scaling(torch_cuda, n):
    """SCALE pre-op and CONJ_MUL_THEN_SCALE intra-op by 1/(N^2*6) give exactly 1.0 at the origin."""
    torch = torch_cuda
    fin = (n, n, 1)
    sf = float(n * n * 6)
    t = np.zeros((n, n), np.float32)
    t[0, 0] = 2.0
    img = dev(torch, np.full((1, n // 2 + 1, n), 3.0, np.complex64).view(np.float32))
    ft = make(fin, fin, fin)
    tin = dev(torch, O.real_to_padded(t, fin))
    for pre, intra, want in [(KF.noop(), KF.conj_mul(), sf), (KF.scale(1 / sf), KF.conj_mul(), 1.0),
                             (KF.noop(), KF.conj_mul_then_scale(1 / sf), 1.0)]:
        out = empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32)
        ft.FwdImageInvFFT(tin, img, out, pre, intra, KF.noop())
        r = O.real_from_padded(host(out), fin)
        assert r[0, 0, 0] == np.float32(want)
        assert np.count_nonzero(r) == 1


# ---------------------------------------------------------------------------
# Cross-correlation on random data
# ---------------------------------------------------------------------------
XCORR_CASES = [
    ((48, 48, 1), (128, 128, 1), (40, 40, 1)),
    ((64, 64, 1), (256, 256, 1), (256, 256, 1)),      # reference-supported combo: increase / none
    ((100, 60, 1), (512, 256, 1), (130, 70, 1)),
    ((128, 128, 1), (1024, 1024, 1), (512, 512, 1)),
    ((256, 256, 1), (256, 256, 1), (100, 100, 1)),     # forward none / inverse decrease
    ((33, 17, 1), (8192, 32, 1), (8192, 16, 1)),
]


@pytest.mark.parametrize("fin,fout,iout", XCORR_CASES)
def test_xcorr_matches_oracle(torch_cuda, fin, fout, iout):
    torch = torch_cuda
    rng = np.random.default_rng(fin[0] + fout[0] + iout[0])
    t = rng.standard_normal((fin[1], fin[0])).astype(np.float32)
    img = rng.standard_normal((fout[1], fout[0]))
    spec = O.fwd(O.real_to_padded(img, fout, dtype=np.float64), fout, fout).astype(np.complex64)
    ft = make(fin, fout, iout)
    out = empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32)
    ft.FwdImageInvFFT(dev(torch, O.real_to_padded(t, fin)), dev(torch, spec.view(np.float32)), out)
    got = O.real_from_padded(host(out), iout)
    plan = O.Plan(fin, fout, fout, iout)
    ref = O.real_from_padded(O.fwd_image_inv(O.real_to_padded(t, fin), spec, plan, out_dtype=np.float64), iout)
    assert O.rel_l2(got, ref) <= RTOL_L2_FP32
    assert O.rel_max(got, ref) <= RTOL_MAX_FP32


def test_xcorr_4096_template_384_window_1024(torch_cuda):
    """The headline workload: 4096^2 noise + 20 blobs, 384^2 N(0,1) template, 1024^2 window."""
    torch = torch_cuda
    n, L, W = 4096, 384, 1024
    img = O.gaussian_blob_image(n)
    spec = O.image_spectrum_fp32(img)
    t = O.normal_template(L, O.SEED_BASE + 1).astype(np.float32)
    fin, fout, iout = (L, L, 1), (n, n, 1), (W, W, 1)
    ft = make(fin, fout, iout)
    out = empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32)
    ft.FwdImageInvFFT(dev(torch, O.real_to_padded(t, fin)), dev(torch, spec.view(np.float32)), out)
    got = O.real_from_padded(host(out), iout)[0]
    plan = O.Plan(fin, fout, fout, iout)
    ref = O.real_from_padded(O.fwd_image_inv(O.real_to_padded(t, fin), spec, plan, out_dtype=np.float64), iout)[0]
    assert O.rel_l2(got, ref) <= RTOL_L2_FP32
    gi, _, _ = O.peak(got)
    ri, rtop, margin = O.peak(ref)
    assert margin > 1e-4 * abs(rtop)      # the peak is well separated at FP32 accuracy
    assert gi == ri


def test_golden_vectors_on_gpu(torch_cuda):
    import os
    torch = torch_cuda
    here = os.path.dirname(os.path.abspath(__file__))
    g = np.load(os.path.join(here, "golden", "fwd_32_to_128.npz"))
    fin, fout = tuple(g["fwd_in"]), tuple(g["fwd_out"])
    ft = make(fin, fout, fout)
    xin = dev(torch, g["input"].astype(np.float32))
    out = empty(torch, ft.ReturnFwdOutputMemorySize(), torch.float32)
    ft.FwdFFT(xin, out)
    assert O.rel_l2(spectrum_view(out, fout), g["spectrum"]) <= RTOL_L2_FP32
    g = np.load(os.path.join(here, "golden", "xcorr_48_to_128_w40.npz"))
    fin, fout, iout = tuple(g["fwd_in"]), tuple(g["fwd_out"]), tuple(g["inv_out"])
    ft = make(fin, fout, iout)
    out = empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32)
    img = np.ascontiguousarray(g["image_spectrum"]).astype(np.complex64)
    ft.FwdImageInvFFT(dev(torch, g["input"].astype(np.float32)), dev(torch, img.view(np.float32)), out)
    got = O.real_from_padded(host(out), iout)
    assert O.rel_l2(got, O.real_from_padded(g["output"], iout)) <= 2e-5   # image rounded to complex64


# ---------------------------------------------------------------------------
# Reduced-precision storage (FP16 / BF16 template and image spectrum)
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("in_dt,img_dt,tol", [("float16", "complex32", 2e-5), ("bfloat16", "complex_bf16", 2e-5)])
def test_xcorr_low_precision_storage(torch_cuda, in_dt, img_dt, tol):
    torch = torch_cuda
    n, L, W = 1024, 128, 256
    rng = np.random.default_rng(99)
    tdt = torch.float16 if in_dt == "float16" else torch.bfloat16
    t32 = rng.standard_normal((L, L)).astype(np.float32)
    t_q = torch.from_numpy(t32).to(tdt)
    t_deq = t_q.float().numpy()
    img = rng.standard_normal((n, n))
    spec = O.fwd(O.real_to_padded(img, (n, n, 1), dtype=np.float64), (n, n, 1), (n, n, 1)) / n
    spec_c = torch.from_numpy(spec.astype(np.complex64).view(np.float32).reshape(-1)).to(tdt)
    spec_deq = spec_c.float().numpy().view(np.complex64).reshape(spec.shape)
    fin, fout, iout = (L, L, 1), (n, n, 1), (W, W, 1)
    ft = make(fin, fout, iout, input_dtype=in_dt, image_dtype=img_dt)
    ft.SetOutputDtype("float32")
    tin = torch.zeros(ft.ReturnInputMemorySize(), dtype=tdt)
    tin.view(L, -1)[:, :L] = t_q
    out = empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32)
    ft.FwdImageInvFFT(tin.cuda(), spec_c.cuda(), out)
    got = O.real_from_padded(host(out), iout)
    plan = O.Plan(fin, fout, fout, iout)
    ref = O.real_from_padded(O.fwd_image_inv(O.real_to_padded(t_deq, fin), spec_deq, plan, out_dtype=np.float64), iout)
    assert O.rel_l2(got, ref) <= tol


def test_non_default_stream(torch_cuda):
    torch = torch_cuda
    fin, fout = (64, 64, 1), (256, 256, 1)
    x = random_real((64, 64), seed=5)
    ft = make(fin, fout, fout)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        xin = dev(torch, O.real_to_padded(x, fin))
        out = empty(torch, ft.ReturnFwdOutputMemorySize(), torch.float32)
        ft.FwdFFT(xin, out)
    s.synchronize()
    ref = O.fwd(O.real_to_padded(x, fin), fin, fout)
    assert O.rel_l2(spectrum_view(out, fout), ref) <= RTOL_L2_FP32


def test_inverse_increase_is_rejected(torch_cuda):
    ft = F.FourierTransformer()
    ft.SetForwardFFTPlan(64, 64, 1, 64, 64, 1)
    ft.SetInverseFFTPlan(64, 64, 1, 128, 128, 1)
    with pytest.raises(F.FastFFTError):
        ft.InvFFT(torch_cuda.zeros(128 * 130, device="cuda"))
