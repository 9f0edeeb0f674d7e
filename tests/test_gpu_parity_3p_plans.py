"""2D plans at the lengths 3 * 2^k (384 ... 6144), 5 * 2^k (640 ... 5120) and 7 * 2^k (896 ... 3584), which the
reference rejects, against the FP64 oracle: forward, inverse (with a window origin), round
trip, and the fused correlation through the size-N kernels (single call) and the
reduced-size path (batched).
"""
import numpy as np
import pytest

import fastfft_b200 as F
from oracle import fastfft_oracle as O
from tests._util import RTOL_L2_FP32, RTOL_MAX_FP32, dev, empty, host, random_real, spectrum_view

pytestmark = pytest.mark.gpu


def make(fin, fout, iout):
    ft = F.FourierTransformer()
    ft.SetForwardFFTPlan(*fin, *fout)
    ft.SetInverseFFTPlan(*fout, *iout)
    return ft


FWD_CASES = [
    ((384, 384, 1), (384, 384, 1)),
    ((1536, 1536, 1), (1536, 1536, 1)),
    ((100, 200, 1), (768, 1536, 1)),         # zero padding into 3 * 2^k on both axes
    ((3072, 64, 1), (3072, 64, 1)),          # 3 * 2^k rows, power-of-two columns
    ((64, 6144, 1), (64, 6144, 1)),          # power-of-two rows, 6144-point columns
    ((1536, 768, 1), (384, 384, 1)),         # forward decrease: first outputs kept
    ((640, 640, 1), (640, 640, 1)),           # 5 * 2^k
    ((1280, 1280, 1), (1280, 1280, 1)),
    ((100, 300, 1), (640, 2560, 1)),          # zero padding into 5 * 2^k on both axes
    ((5120, 32, 1), (5120, 32, 1)),           # 5120-point rows
    ((32, 5120, 1), (32, 5120, 1)),           # 5120-point columns
    ((640, 1536, 1), (640, 1536, 1)),         # 5 * 2^k rows, 3 * 2^k columns
    ((2560, 1280, 1), (640, 640, 1)),         # forward decrease
    ((896, 896, 1), (896, 896, 1)),           # 7 * 2^k
    ((100, 300, 1), (896, 1792, 1)),          # zero padding into 7 * 2^k on both axes
    ((3584, 32, 1), (3584, 32, 1)),           # 3584-point rows
    ((32, 3584, 1), (32, 3584, 1)),           # 3584-point columns
    ((896, 1536, 1), (896, 1536, 1)),         # 7 * 2^k rows, 3 * 2^k columns
    ((1792, 896, 1), (640, 640, 1)),          # forward decrease
]


@pytest.mark.parametrize("fin,fout", FWD_CASES)
def test_forward_matches_oracle(torch_cuda, fin, fout):
    torch = torch_cuda
    x = random_real((fin[1], fin[0]), seed=fin[0] + 3 * fout[1])
    ft = make(fin, fout, fout)
    xin = dev(torch, O.real_to_padded(x, fin), ft.ReturnInputMemorySize())
    out = empty(torch, ft.ReturnFwdOutputMemorySize(), torch.float32)
    ft.FwdFFT(xin, out)
    got = spectrum_view(out, fout)
    ref = O.fwd(O.real_to_padded(x, fin), fin, fout)
    assert O.rel_l2(got, ref) <= RTOL_L2_FP32
    assert O.rel_max(got, ref) <= RTOL_MAX_FP32


INV_CASES = [
    ((1536, 1536, 1), (1536, 1536, 1), (0, 0)),
    ((768, 3072, 1), (700, 1000, 1), (0, 0)),
    ((1536, 1536, 1), (700, 600, 1), (16, 32)),   # window away from the origin
    ((1280, 1280, 1), (1280, 1280, 1), (0, 0)),
    ((640, 2560, 1), (600, 2000, 1), (0, 0)),
    ((2560, 640, 1), (1000, 500, 1), (40, 70)),
    ((1792, 1792, 1), (1792, 1792, 1), (0, 0)),
    ((896, 3584, 1), (800, 3000, 1), (20, 30)),
]


@pytest.mark.parametrize("iin,iout,origin", INV_CASES)
def test_inverse_matches_oracle(torch_cuda, iin, iout, origin):
    torch = torch_cuda
    rng = np.random.default_rng(iin[0] + iout[1])
    w, _ = O.padded_x(iin[0])
    spec = (rng.standard_normal((1, w, iin[1])) + 1j * rng.standard_normal((1, w, iin[1]))).astype(np.complex64)
    ft = make(iin, iin, iout)
    if origin != (0, 0):
        ft.SetInverseOutputOrigin(*origin)
    out = empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32)
    ft.InvFFT(dev(torch, spec.view(np.float32)), out)
    got = O.real_from_padded(host(out), iout)
    ref = O.real_from_padded(O.inv(spec, iin, iout, out_dtype=np.float64, origin=(*origin, 0)), iout)
    assert O.rel_l2(got, ref) <= RTOL_L2_FP32
    assert O.rel_max(got, ref) <= RTOL_MAX_FP32


def test_round_trip_1536(torch_cuda):
    torch = torch_cuda
    fin = fout = (1536, 1536, 1)
    x = random_real((1536, 1536), seed=77)
    ft = make(fin, fout, fout)
    n_max = max(ft.ReturnInputMemorySize(), ft.ReturnFwdOutputMemorySize())
    buf = dev(torch, O.real_to_padded(x, fin), n_max)
    ft.FwdFFT(buf)
    ft.InvFFT(buf)
    back = O.real_from_padded(host(buf), fout)[0]
    assert O.rel_l2(back, x * 1536.0 * 1536.0) <= RTOL_L2_FP32


def test_correlation_at_1536(torch_cuda):
    """200 x 150 template, 1536^2 image, 700 x 600 window: single calls run the size-N
    1536-point kernels, batched calls the reduced-size path (1024 x 768 here)."""
    torch = torch_cuda
    fin, fout, iout = (200, 150, 1), (1536, 1536, 1), (700, 600, 1)
    img = np.random.default_rng(78).standard_normal((1536, 1536))
    spec = O.fwd(O.real_to_padded(img, fout, dtype=np.float64), fout, fout).astype(np.complex64)
    d_spec = dev(torch, spec.view(np.float32))
    ts = [random_real((150, 200), seed=79 + i) for i in range(3)]
    ft = make(fin, fout, iout)
    assert ft.CorrelationSize() == (1024, 768)
    single = [empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32) for _ in ts]
    batched = [empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32) for _ in ts]
    ins = [dev(torch, O.real_to_padded(t, fin)) for t in ts]
    for t, o in zip(ins, single):
        ft.FwdImageInvFFT(t, d_spec, o)
    ft.FwdImageInvFFTMany(ins, d_spec, batched)
    p = O.Plan(fin, fout, fout, iout)
    for t, a, b in zip(ts, single, batched):
        ref = O.real_from_padded(O.fwd_image_inv(O.real_to_padded(t, fin), spec, p, out_dtype=np.float64), iout)
        for o in (a, b):
            got = O.real_from_padded(host(o), iout)
            assert O.rel_l2(got, ref) <= RTOL_L2_FP32
            assert O.rel_max(got, ref) <= RTOL_MAX_FP32


def test_round_trip_1280(torch_cuda):
    torch = torch_cuda
    fin = fout = (1280, 1280, 1)
    x = random_real((1280, 1280), seed=81)
    ft = make(fin, fout, fout)
    n_max = max(ft.ReturnInputMemorySize(), ft.ReturnFwdOutputMemorySize())
    buf = dev(torch, O.real_to_padded(x, fin), n_max)
    ft.FwdFFT(buf)
    ft.InvFFT(buf)
    back = O.real_from_padded(host(buf), fout)[0]
    assert O.rel_l2(back, x * 1280.0 * 1280.0) <= RTOL_L2_FP32


def test_correlation_at_1280(torch_cuda):
    """300 x 200 template, 1280^2 image, 900 x 700 window: single calls run the size-N
    1280-point kernels, batched calls the reduced-size path (1280 x 1024 here)."""
    torch = torch_cuda
    fin, fout, iout = (300, 200, 1), (1280, 1280, 1), (900, 700, 1)
    img = np.random.default_rng(82).standard_normal((1280, 1280))
    spec = O.fwd(O.real_to_padded(img, fout, dtype=np.float64), fout, fout).astype(np.complex64)
    d_spec = dev(torch, spec.view(np.float32))
    ts = [random_real((200, 300), seed=83 + i) for i in range(3)]
    ft = make(fin, fout, iout)
    assert ft.CorrelationSize() == (1280, 1024)
    single = [empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32) for _ in ts]
    batched = [empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32) for _ in ts]
    ins = [dev(torch, O.real_to_padded(t, fin)) for t in ts]
    for t, o in zip(ins, single):
        ft.FwdImageInvFFT(t, d_spec, o)
    ft.FwdImageInvFFTMany(ins, d_spec, batched)
    p = O.Plan(fin, fout, fout, iout)
    for t, a, b in zip(ts, single, batched):
        ref = O.real_from_padded(O.fwd_image_inv(O.real_to_padded(t, fin), spec, p, out_dtype=np.float64), iout)
        for o in (a, b):
            got = O.real_from_padded(host(o), iout)
            assert O.rel_l2(got, ref) <= RTOL_L2_FP32
            assert O.rel_max(got, ref) <= RTOL_MAX_FP32
