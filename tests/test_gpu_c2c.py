"""Complex-input (C2C) transforms against the FP64 oracle.

The reference declares complex InputType but its complex paths are stubs
(src/fastfft/FastFFT.cu:369-391, :722-793); the oracle's fwd_c2c / inv_c2c /
fwd_image_inv_c2c restate the real path's conventions for complex data (sign -1,
unnormalised, origin padding, [kz][kx][ky] spectra with every kx, rows of pitch x).
"""
import numpy as np
import pytest

import fastfft_b200 as F
from oracle import fastfft_oracle as O
from tests._util import RTOL_L2_FP32, RTOL_MAX_FP32, dev, empty, host

pytestmark = pytest.mark.gpu


def crand(shape, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def make(fin, fout, iout, input_dtype="complex64", origin=None):
    ft = F.FourierTransformer(input_dtype=input_dtype, rank=3 if fout[2] > 1 else 2)
    ft.SetForwardFFTPlan(*fin, *fout)
    ft.SetInverseFFTPlan(*fout, *iout)
    if origin is not None:
        ft.SetInverseOutputOrigin(*origin)
    return ft


def cbuf(torch, a, n_elems=None):
    return dev(torch, O.complex_to_buffer(a).view(np.float32), n_elems)


FWD = [
    ((64, 64, 1), (512, 512, 1)),
    ((100, 37, 1), (256, 128, 1)),
    ((4096, 16, 1), (4096, 16, 1)),
    ((512, 512, 1), (128, 256, 1)),          # decrease: the first outputs per axis
    ((16, 16, 16), (64, 64, 64)),
    ((64, 32, 16), (64, 32, 16)),
]


@pytest.mark.parametrize("fin,fout", FWD)
def test_forward_c2c(torch_cuda, fin, fout):
    torch = torch_cuda
    x = crand((fin[2], fin[1], fin[0]), sum(fin) + sum(fout))
    ft = make(fin, fout, fout)
    out = empty(torch, ft.ReturnFwdOutputMemorySize(), torch.float32)
    ft.FwdFFT(cbuf(torch, x), out, pre_op=F.KernelFunction.scale(0.5))
    ref = O.fwd_c2c(x, fin, fout, pre_op=(O.OP_SCALE, 0.5))
    got = host(out).view(np.complex64).reshape(ref.shape)
    assert O.rel_l2(got, ref) <= RTOL_L2_FP32
    assert O.rel_max(got, ref) <= RTOL_MAX_FP32


INV = [
    ((512, 512, 1), (512, 512, 1), (0, 0, 0)),
    ((256, 128, 1), (100, 37, 1), (0, 0, 0)),
    ((256, 128, 1), (100, 37, 1), (7, 50, 0)),
    ((64, 64, 64), (20, 30, 10), (5, 6, 3)),
]


@pytest.mark.parametrize("iin,iout,org", INV)
def test_inverse_c2c(torch_cuda, iin, iout, org):
    torch = torch_cuda
    spec = crand((iin[2], iin[0], iin[1]), sum(iin) + 3)     # [kz][kx][ky]
    ft = make(iin, iin, iout, origin=org)
    out = empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32)
    ft.InvFFT(cbuf(torch, spec), out, post_op=F.KernelFunction.scale(0.25))
    ref = O.inv_c2c(spec, iin, iout, post_op=(O.OP_SCALE, 0.25), origin=org)
    got = O.complex_from_buffer(host(out), iout)
    assert O.rel_l2(got, ref) <= RTOL_L2_FP32
    assert O.rel_max(got, ref) <= RTOL_MAX_FP32


@pytest.mark.parametrize("out_dtype", ["complex32", "complex_bf16"])
def test_round_trip_c2c_low_precision_output(torch_cuda, out_dtype):
    torch = torch_cuda
    fin, fout = (32, 32, 1), (128, 128, 1)
    x = crand((32, 32), 11) * 0.01
    ft = make(fin, fout, fout)
    ft.SetOutputDtype(out_dtype)
    spec = empty(torch, ft.ReturnFwdOutputMemorySize(), torch.float32)
    ft.FwdFFT(cbuf(torch, x), spec)
    tdt = torch.float16 if out_dtype == "complex32" else torch.bfloat16
    out = torch.zeros(ft.ReturnInvOutputMemorySize(), dtype=tdt, device="cuda")
    ft.InvFFT(spec, out, post_op=F.KernelFunction.scale(1.0 / (128 * 128)))
    got = O.complex_from_buffer(out.float().cpu().numpy(), fout)[0]
    want = np.zeros((128, 128), complex)
    want[:32, :32] = x
    assert O.rel_l2(got, want) <= (1e-3 if out_dtype == "complex32" else 8e-3)


XCORR = [
    ((48, 40, 1), (256, 256, 1), (100, 90, 1), None),
    ((64, 64, 1), (1024, 512, 1), (256, 128, 1), None),
    ((16, 16, 16), (64, 64, 64), (20, 20, 20), None),
    ((16, 16, 16), (64, 64, 64), (16, 16, 16), (24, 24, 24)),
]


@pytest.mark.parametrize("fin,fout,iout,org", XCORR)
def test_xcorr_c2c(torch_cuda, fin, fout, iout, org):
    torch = torch_cuda
    t = crand((fin[2], fin[1], fin[0]), 21)
    img = crand((fout[2], fout[1], fout[0]), 22)
    spec = O.fwd_c2c(img, fout, fout).astype(np.complex64)
    ft = make(fin, fout, iout, origin=org)
    out = empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32)
    ft.FwdImageInvFFT(cbuf(torch, t), dev(torch, spec.view(np.float32)), out)
    p = O.Plan(fin, fout, fout, iout)
    ref = O.fwd_image_inv_c2c(t, spec, p, origin=org or (0, 0, 0))
    got = O.complex_from_buffer(host(out), iout)
    assert O.rel_l2(got, ref) <= RTOL_L2_FP32
    assert O.rel_max(got, ref) <= RTOL_MAX_FP32
    flat = np.abs(got).ravel()
    assert int(np.argmax(flat)) == int(np.argmax(np.abs(ref).ravel()))


def test_xcorr_c2c_batched_calls_match_single(torch_cuda):
    """The batched entry points take the size-N path for complex input, template by template."""
    torch = torch_cuda
    fin, fout, iout = (40, 40, 1), (256, 256, 1), (64, 64, 1)
    spec = O.fwd_c2c(crand((256, 256), 31), fout, fout).astype(np.complex64)
    d_spec = dev(torch, spec.view(np.float32))
    ts = [cbuf(torch, crand((40, 40), 32 + i)) for i in range(3)]
    ft = make(fin, fout, iout)
    outs = [empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32) for _ in ts]
    ft.FwdImageInvFFTMany(ts, d_spec, outs)
    for t, o in zip(ts, outs):
        one = empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32)
        ft.FwdImageInvFFT(t, d_spec, one)
        assert torch.equal(one, o)
