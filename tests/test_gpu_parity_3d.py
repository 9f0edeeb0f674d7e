"""GPU parity of the 3D path against the FP64 oracle, through the C ABI.

Spectrum layout [kz][kx][ky] (ky contiguous); the inverse keeps a window at a settable
origin (the reference keeps the origin-anchored window and aborts on a 3D inverse
decrease, src/fastfft/FastFFT.cu:595-598).
"""
import numpy as np
import pytest

import fastfft_b200 as F
from oracle import fastfft_oracle as O
from tests._util import RTOL_L2_FP32, RTOL_MAX_FP32, dev, empty, host

pytestmark = pytest.mark.gpu


def make(fin, fout, iout, origin=None):
    ft = F.FourierTransformer(rank=3)
    ft.SetForwardFFTPlan(*fin, *fout)
    ft.SetInverseFFTPlan(*fout, *iout)
    if origin is not None:
        ft.SetInverseOutputOrigin(*origin)
    return ft


def spec_view(t, dims):
    x, y, z = dims
    w, _ = O.padded_x(x)
    return host(t)[: 2 * w * y * z].view(np.complex64).reshape(z, w, y)


FWD = [
    ((64, 64, 64), (256, 256, 256)),       # 64^3 zero-padded into a 256^3 R2C
    ((32, 32, 32), (32, 32, 32)),
    ((64, 32, 16), (64, 32, 16)),
    ((7, 9, 3), (32, 16, 16)),
    ((16, 16, 16), (128, 64, 32)),
    ((64, 64, 64), (32, 32, 32)),          # forward decrease: first outputs kept
    ((512, 16, 16), (512, 16, 16)),
]


@pytest.mark.parametrize("fin,fout", FWD)
def test_forward_3d(torch_cuda, fin, fout):
    torch = torch_cuda
    x = np.random.default_rng(sum(fin)).standard_normal((fin[2], fin[1], fin[0])).astype(np.float32)
    ft = make(fin, fout, fout)
    out = empty(torch, ft.ReturnFwdOutputMemorySize(), torch.float32)
    ft.FwdFFT(dev(torch, O.real_to_padded(x, fin)), out)
    got = spec_view(out, fout)
    ref = O.fwd(O.real_to_padded(x, fin), fin, fout)
    assert O.rel_l2(got, ref) <= RTOL_L2_FP32
    assert O.rel_max(got, ref) <= RTOL_MAX_FP32


INV = [
    ((256, 256, 256), (128, 128, 128), (64, 64, 64)),   # central 128^3 of a 256^3 C2R
    ((256, 256, 256), (128, 128, 128), (0, 0, 0)),
    ((32, 32, 32), (32, 32, 32), (0, 0, 0)),
    ((64, 32, 16), (30, 20, 10), (5, 6, 3)),
    ((16, 64, 32), (16, 64, 32), (0, 0, 0)),
]


@pytest.mark.parametrize("iin,iout,org", INV)
def test_inverse_3d(torch_cuda, iin, iout, org):
    torch = torch_cuda
    rng = np.random.default_rng(sum(iin) + sum(iout))
    w, _ = O.padded_x(iin[0])
    shape = (iin[2], w, iin[1])
    spec = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)
    ft = make(iin, iin, iout, origin=org)
    out = empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32)
    ft.InvFFT(dev(torch, spec.view(np.float32)), out)
    got = O.real_from_padded(host(out), iout)
    ref = O.real_from_padded(O.inv(spec, iin, iout, out_dtype=np.float64, origin=org), iout)
    assert O.rel_l2(got, ref) <= RTOL_L2_FP32
    assert O.rel_max(got, ref) <= RTOL_MAX_FP32


@pytest.mark.parametrize("org", [(0, 0, 0), (64, 64, 64)])
def test_round_trip_64_in_256_window_128(torch_cuda, org):
    """64^3 N(0,1) padded to a 256^3 R2C, then the 256^3 C2R keeping a 128^3 window.

    With the window at the origin it contains the volume (x 256^3); the central window
    does not overlap the zero-padded volume, so its exact values are 0 and the bound is
    absolute, relative to the round-trip scale.
    """
    torch = torch_cuda
    fin, fout, iout = (64, 64, 64), (256, 256, 256), (128, 128, 128)
    x = np.random.default_rng(O.SEED_BASE + 2).standard_normal((64, 64, 64)).astype(np.float32)
    ft = make(fin, fout, iout, origin=org)
    spec = empty(torch, ft.ReturnFwdOutputMemorySize(), torch.float32)
    ft.FwdFFT(dev(torch, O.real_to_padded(x, fin)), spec)
    out = empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32)
    ft.InvFFT(spec, out)
    got = O.real_from_padded(host(out), iout)
    ref_spec = O.fwd(O.real_to_padded(x, fin), fin, fout)
    assert O.rel_l2(spec_view(spec, fout), ref_spec) <= RTOL_L2_FP32
    scale = 256.0 ** 3 * np.abs(x).max()
    if org == (0, 0, 0):
        want = np.zeros((128, 128, 128))
        want[:64, :64, :64] = x * 256.0 ** 3
        assert O.rel_l2(got, want) <= RTOL_L2_FP32
    else:
        assert np.abs(got).max() <= 1e-6 * scale


@pytest.mark.parametrize("n", [16, 64, 128])
def test_kat_unit_impulse_3d(torch_cuda, n):
    torch = torch_cuda
    d = (n, n, n)
    x = np.zeros((n, n, n), np.float32)
    x[0, 0, 0] = 1
    ft = make(d, d, d)
    buf = dev(torch, O.real_to_padded(x, d), ft.ReturnFwdOutputMemorySize())
    ft.FwdFFT(buf)
    assert np.all(spec_view(buf, d) == np.complex64(1))
    ft.InvFFT(buf)
    r = O.real_from_padded(host(buf), d)
    assert r[0, 0, 0] == n ** 3 and np.count_nonzero(r) == 1


XCORR = [
    ((16, 16, 16), (64, 64, 64), (20, 20, 20), (0, 0, 0)),
    ((12, 10, 8), (32, 64, 16), (32, 64, 16), (0, 0, 0)),
    ((16, 16, 16), (64, 64, 64), (16, 16, 16), (24, 24, 24)),
]


@pytest.mark.parametrize("fin,fout,iout,org", XCORR)
def test_xcorr_3d(torch_cuda, fin, fout, iout, org):
    torch = torch_cuda
    rng = np.random.default_rng(7)
    t = rng.standard_normal((fin[2], fin[1], fin[0])).astype(np.float32)
    img = rng.standard_normal((fout[2], fout[1], fout[0]))
    spec = O.fwd(O.real_to_padded(img, fout, dtype=np.float64), fout, fout).astype(np.complex64)
    ft = make(fin, fout, iout, origin=org)
    out = empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32)
    ft.FwdImageInvFFT(dev(torch, O.real_to_padded(t, fin)), dev(torch, spec.view(np.float32)), out)
    got = O.real_from_padded(host(out), iout)
    ref = O.real_from_padded(O.fwd_image_inv(O.real_to_padded(t, fin), spec, O.Plan(fin, fout, fout, iout),
                                             out_dtype=np.float64, origin=org), iout)
    assert O.rel_l2(got, ref) <= RTOL_L2_FP32
