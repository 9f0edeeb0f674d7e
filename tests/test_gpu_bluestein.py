"""2D plans at lengths that are neither powers of two nor R * 2^k (any length in [17, 4096]),
which the reference rejects: the chirp-z (Bluestein) transforms on a power-of-two block FFT
of length M >= 2N - 1, against the FP64 oracle.  Forward (zero padding, odd lengths, mixed
with power-of-two axes, the shortest and longest lengths, forward decrease), inverse with a
window origin, round trip, the fused correlation through single and batched calls (the
batched call runs at the plan's size when an axis would correlate at a chirp-z length, and
through the reduced-size path when both axes correlate at a power of two or 3 * 2^k), the
half-precision storage types, the refusal of the fused peak search at such lengths, and
complex-input (C2C) plans (forward, inverse with an origin, correlation) and 3D plans
(forward with padding and decrease, inverse with a central window, correlation, C2C).
"""
import numpy as np
import pytest

import fastfft_b200 as F
from fastfft_b200 import _capi as C
from oracle import fastfft_oracle as O
from tests._util import RTOL_L2_FP32, RTOL_MAX_FP32, dev, empty, host, random_real, spectrum_view

pytestmark = pytest.mark.gpu

# the chirp-z DFT runs two M-point FFTs and three complex products per length-N transform;
# its FP32 error stays within the bounds of the power-of-two path
RTOL_L2_BLUE = RTOL_L2_FP32
RTOL_MAX_BLUE = RTOL_MAX_FP32


def make(fin, fout, iout):
    ft = F.FourierTransformer()
    ft.SetForwardFFTPlan(*fin, *fout)
    ft.SetInverseFFTPlan(*fout, *iout)
    return ft


FWD_CASES = [
    ((100, 100, 1), (1000, 1000, 1)),        # zero padding into 1000 on both axes
    ((1000, 1000, 1), (1000, 1000, 1)),
    ((77, 53, 1), (999, 1001, 1)),           # odd lengths
    ((1000, 512, 1), (1000, 512, 1)),        # chirp-z rows, power-of-two columns
    ((512, 1000, 1), (512, 1000, 1)),        # power-of-two rows, chirp-z columns
    ((300, 1536, 1), (300, 1536, 1)),        # chirp-z rows, 3 * 2^k columns
    ((17, 17, 1), (17, 17, 1)),              # shortest (M = 64)
    ((4095, 32, 1), (4095, 32, 1)),          # longest rows (M = 8192)
    ((32, 4095, 1), (32, 4095, 1)),          # longest columns
    ((1000, 600, 1), (300, 200, 1)),         # forward decrease: first outputs kept
]


@pytest.mark.parametrize("fin,fout", FWD_CASES)
def test_forward_matches_oracle(torch_cuda, fin, fout):
    torch = torch_cuda
    x = random_real((fin[1], fin[0]), seed=fin[0] + 7 * fout[1])
    ft = make(fin, fout, fout)
    xin = dev(torch, O.real_to_padded(x, fin), ft.ReturnInputMemorySize())
    out = empty(torch, ft.ReturnFwdOutputMemorySize(), torch.float32)
    ft.FwdFFT(xin, out)
    got = spectrum_view(out, fout)
    ref = O.fwd(O.real_to_padded(x, fin), fin, fout)
    assert O.rel_l2(got, ref) <= RTOL_L2_BLUE
    assert O.rel_max(got, ref) <= RTOL_MAX_BLUE


INV_CASES = [
    ((1000, 1000, 1), (1000, 1000, 1), (0, 0)),
    ((999, 1001, 1), (700, 800, 1), (10, 20)),    # odd lengths, window away from the origin
    ((1000, 512, 1), (600, 400, 1), (0, 0)),
    ((512, 1000, 1), (500, 900, 1), (5, 50)),
    ((4095, 64, 1), (4000, 64, 1), (95, 0)),
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
    assert O.rel_l2(got, ref) <= RTOL_L2_BLUE
    assert O.rel_max(got, ref) <= RTOL_MAX_BLUE


@pytest.mark.parametrize("n", [(1000, 1000), (999, 1001)])
def test_round_trip(torch_cuda, n):
    torch = torch_cuda
    fin = fout = (*n, 1)
    x = random_real((n[1], n[0]), seed=n[0])
    ft = make(fin, fout, fout)
    n_max = max(ft.ReturnInputMemorySize(), ft.ReturnFwdOutputMemorySize())
    buf = dev(torch, O.real_to_padded(x, fin), n_max)
    ft.FwdFFT(buf)
    ft.InvFFT(buf)
    back = O.real_from_padded(host(buf), fout)[0]
    assert O.rel_l2(back, x * float(n[0]) * float(n[1])) <= RTOL_L2_BLUE


def _image_spectrum(fout, seed):
    img = np.random.default_rng(seed).standard_normal((fout[1], fout[0]))
    return O.fwd(O.real_to_padded(img, fout, dtype=np.float64), fout, fout).astype(np.complex64)


@pytest.mark.parametrize("fin,fout,iout,corr", [
    ((100, 80, 1), (1000, 1000, 1), (700, 600, 1), (1000, 1000)),   # the x axis would correlate at 1000
    ((100, 100, 1), (1000, 1000, 1), (300, 300, 1), (512, 512)),    # reduced-size path from a 1000^2 image
    ((64, 50, 1), (999, 1001, 1), (500, 900, 1), (768, 1001)),      # y at 1001: full size
])
def test_correlation_matches_oracle(torch_cuda, fin, fout, iout, corr):
    torch = torch_cuda
    spec = _image_spectrum(fout, fout[0] + iout[0])
    d_spec = dev(torch, spec.view(np.float32))
    ts = [random_real((fin[1], fin[0]), seed=fin[0] + i) for i in range(3)]
    ft = make(fin, fout, iout)
    assert ft.CorrelationSize() == (corr if corr[0] < fout[0] and corr[1] < fout[1] else fout[:2])
    single = [empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32) for _ in ts]
    batched = [empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32) for _ in ts]
    ins = [dev(torch, O.real_to_padded(t, fin)) for t in ts]
    for t, o in zip(ins, single):
        ft.FwdImageInvFFT(t, d_spec, o)
    ft.FwdImageInvFFTMany(ins, d_spec, batched)
    torch.cuda.synchronize()
    p = O.Plan(fin, fout, fout, iout)
    for t, a, b in zip(ts, single, batched):
        ref = O.real_from_padded(O.fwd_image_inv(O.real_to_padded(t, fin), spec, p, out_dtype=np.float64), iout)
        for o in (a, b):
            got = O.real_from_padded(host(o), iout)
            assert O.rel_l2(got, ref) <= RTOL_L2_BLUE
            assert O.rel_max(got, ref) <= RTOL_MAX_BLUE


@pytest.mark.parametrize("in_dt,img_dt", [("float16", "complex32"), ("bfloat16", "complex_bf16")])
def test_low_precision_storage(torch_cuda, in_dt, img_dt):
    """Half-precision templates and image spectrum at 1000^2 (single and batched calls)."""
    torch = torch_cuda
    fin, fout, iout = (100, 100, 1), (1000, 1000, 1), (700, 700, 1)
    tdt = torch.float16 if in_dt == "float16" else torch.bfloat16
    spec = _image_spectrum(fout, 5) / 1000
    spec_q = torch.from_numpy(spec.view(np.float32).reshape(-1)).to(tdt)
    spec_deq = spec_q.float().numpy().view(np.complex64).reshape(spec.shape)
    t_q = torch.from_numpy(random_real((100, 100), seed=6).astype(np.float32)).to(tdt)
    t_deq = t_q.float().numpy()
    ft = F.FourierTransformer(input_dtype=in_dt, image_dtype=img_dt)
    ft.SetForwardFFTPlan(*fin, *fout)
    ft.SetInverseFFTPlan(*fout, *iout)
    ft.SetOutputDtype("float32")      # the output type otherwise follows the input type
    tin = torch.zeros(ft.ReturnInputMemorySize(), dtype=tdt)
    tin.view(100, -1)[:, :100] = t_q
    tin = tin.cuda()
    d_spec = spec_q.cuda()
    outs = [empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32) for _ in range(2)]
    ft.FwdImageInvFFT(tin, d_spec, outs[0])
    ft.FwdImageInvFFTMany([tin], d_spec, [outs[1]])
    torch.cuda.synchronize()
    p = O.Plan(fin, fout, fout, iout)
    ref = O.real_from_padded(O.fwd_image_inv(O.real_to_padded(t_deq, fin), spec_deq, p, out_dtype=np.float64), iout)
    for o in outs:
        assert O.rel_l2(O.real_from_padded(host(o), iout), ref) <= 2e-5


@pytest.mark.parametrize("out_dt", ["float16", "bfloat16"])
def test_low_precision_output(torch_cuda, out_dt):
    torch = torch_cuda
    fin, fout, iout = (100, 80, 1), (999, 1001, 1), (600, 700, 1)
    odt = torch.float16 if out_dt == "float16" else torch.bfloat16
    spec = _image_spectrum(fout, 9) / (1000 * 1000)
    ft = make(fin, fout, iout)
    ft.SetOutputDtype(out_dt)
    t = random_real((80, 100), seed=10)
    out = empty(torch, ft.ReturnInvOutputMemorySize(), odt)
    ft.FwdImageInvFFT(dev(torch, O.real_to_padded(t, fin)), dev(torch, spec.view(np.float32)), out)
    got = O.real_from_padded(out.float().cpu().numpy(), iout)
    p = O.Plan(fin, fout, fout, iout)
    ref = O.real_from_padded(O.fwd_image_inv(O.real_to_padded(t, fin), spec, p, out_dtype=np.float64), iout)
    tol = 1e-3 if out_dt == "float16" else 8e-3     # one rounding to 11 / 8 significant bits
    assert O.rel_l2(got, ref) <= tol


def test_peak_search_refused_at_chirp_z_inverse_rows(torch_cuda):
    torch = torch_cuda
    fin, fout, iout = (100, 80, 1), (1000, 1000, 1), (700, 600, 1)
    ft = make(fin, fout, iout)
    d_spec = empty(torch, ft.ReturnFwdOutputMemorySize(), torch.float32)
    ins = [empty(torch, ft.ReturnInputMemorySize(), torch.float32)]
    peaks = torch.zeros(1, dtype=torch.int64, device="cuda")
    with pytest.raises(F.FastFFTError) as e:
        ft.FwdImageInvFFTManyPeaks(ins, d_spec, peaks)
    assert e.value.status == C.ERR_UNSUPPORTED


# ---- complex input (C2C plans) at chirp-z lengths ----
def _crand(shape, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def _cmake(fin, fout, iout, origin=None):
    ft = F.FourierTransformer(input_dtype="complex64")
    ft.SetForwardFFTPlan(*fin, *fout)
    ft.SetInverseFFTPlan(*fout, *iout)
    if origin is not None:
        ft.SetInverseOutputOrigin(*origin)
    return ft


def _cbuf(torch, a, n_elems=None):
    return dev(torch, O.complex_to_buffer(a).view(np.float32), n_elems)


@pytest.mark.parametrize("fin,fout", [
    ((77, 53, 1), (999, 1001, 1)),
    ((1000, 1000, 1), (1000, 1000, 1)),
    ((100, 30, 1), (300, 512, 1)),           # chirp-z rows, power-of-two columns
    ((1000, 600, 1), (300, 200, 1)),         # forward decrease
])
def test_forward_c2c(torch_cuda, fin, fout):
    torch = torch_cuda
    x = _crand((1, fin[1], fin[0]), fin[0] + fout[1])
    ft = _cmake(fin, fout, fout)
    out = empty(torch, ft.ReturnFwdOutputMemorySize(), torch.float32)
    ft.FwdFFT(_cbuf(torch, x), out, pre_op=F.KernelFunction.scale(0.5))
    ref = O.fwd_c2c(x, fin, fout, pre_op=(O.OP_SCALE, 0.5))
    got = host(out)[: 2 * ref.size].view(np.complex64).reshape(ref.shape)
    assert O.rel_l2(got, ref) <= RTOL_L2_BLUE
    assert O.rel_max(got, ref) <= RTOL_MAX_BLUE


@pytest.mark.parametrize("iin,iout,org", [
    ((999, 1001, 1), (700, 800, 1), (10, 20, 0)),
    ((1000, 512, 1), (1000, 512, 1), (0, 0, 0)),
])
def test_inverse_c2c(torch_cuda, iin, iout, org):
    torch = torch_cuda
    spec = _crand((1, iin[0], iin[1]), iin[0] + 3)     # [kz][kx][ky]
    ft = _cmake(iin, iin, iout, origin=org)
    out = empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32)
    ft.InvFFT(_cbuf(torch, spec), out, post_op=F.KernelFunction.scale(0.25))
    ref = O.inv_c2c(spec, iin, iout, post_op=(O.OP_SCALE, 0.25), origin=org)
    got = O.complex_from_buffer(host(out), iout)
    assert O.rel_l2(got, ref) <= RTOL_L2_BLUE
    assert O.rel_max(got, ref) <= RTOL_MAX_BLUE


def test_correlation_c2c(torch_cuda):
    torch = torch_cuda
    fin, fout, iout = (100, 80, 1), (1000, 1000, 1), (700, 600, 1)
    t = _crand((1, fin[1], fin[0]), 21)
    img = _crand((1, fout[1], fout[0]), 22)
    spec = O.fwd_c2c(img, fout, fout).astype(np.complex64)
    ft = _cmake(fin, fout, iout)
    out = empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32)
    ft.FwdImageInvFFT(_cbuf(torch, t), dev(torch, spec.view(np.float32)), out)
    p = O.Plan(fin, fout, fout, iout)
    ref = O.fwd_image_inv_c2c(t, spec, p)
    got = O.complex_from_buffer(host(out), iout)
    assert O.rel_l2(got, ref) <= RTOL_L2_BLUE
    assert O.rel_max(got, ref) <= RTOL_MAX_BLUE
    assert int(np.argmax(np.abs(got).ravel())) == int(np.argmax(np.abs(ref).ravel()))


# ---- 3D plans at chirp-z lengths (within 512 per axis) ----
def _make3(fin, fout, iout, origin=None, input_dtype="float32"):
    ft = F.FourierTransformer(input_dtype=input_dtype, rank=3)
    ft.SetForwardFFTPlan(*fin, *fout)
    ft.SetInverseFFTPlan(*fout, *iout)
    if origin is not None:
        ft.SetInverseOutputOrigin(*origin)
    return ft


def _spec3(t, dims):
    x, y, z = dims
    w, _ = O.padded_x(x)
    return host(t)[: 2 * w * y * z].view(np.complex64).reshape(z, w, y)


@pytest.mark.parametrize("fin,fout", [
    ((16, 16, 16), (100, 60, 50)),           # chirp-z on every axis
    ((33, 20, 17), (33, 20, 17)),
    ((64, 30, 16), (64, 30, 16)),            # power-of-two x and z, chirp-z y
    ((100, 60, 50), (40, 30, 20)),           # forward decrease
])
def test_forward_3d(torch_cuda, fin, fout):
    torch = torch_cuda
    x = np.random.default_rng(sum(fin)).standard_normal((fin[2], fin[1], fin[0])).astype(np.float32)
    ft = _make3(fin, fout, fout)
    out = empty(torch, ft.ReturnFwdOutputMemorySize(), torch.float32)
    ft.FwdFFT(dev(torch, O.real_to_padded(x, fin)), out)
    ref = O.fwd(O.real_to_padded(x, fin), fin, fout)
    got = _spec3(out, fout)
    assert O.rel_l2(got, ref) <= RTOL_L2_BLUE
    assert O.rel_max(got, ref) <= RTOL_MAX_BLUE


@pytest.mark.parametrize("iin,iout,org", [
    ((100, 60, 50), (100, 60, 50), (0, 0, 0)),
    ((100, 60, 50), (40, 30, 20), (30, 15, 15)),     # central window
])
def test_inverse_3d(torch_cuda, iin, iout, org):
    torch = torch_cuda
    rng = np.random.default_rng(sum(iin) + sum(iout))
    w, _ = O.padded_x(iin[0])
    shape = (iin[2], w, iin[1])
    spec = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)
    ft = _make3(iin, iin, iout, origin=org)
    out = empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32)
    ft.InvFFT(dev(torch, spec.view(np.float32)), out)
    got = O.real_from_padded(host(out), iout)
    ref = O.real_from_padded(O.inv(spec, iin, iout, out_dtype=np.float64, origin=org), iout)
    assert O.rel_l2(got, ref) <= RTOL_L2_BLUE
    assert O.rel_max(got, ref) <= RTOL_MAX_BLUE


def test_correlation_3d(torch_cuda):
    torch = torch_cuda
    fin, fout, iout = (16, 12, 10), (100, 60, 50), (40, 30, 20)
    rng = np.random.default_rng(8)
    t = rng.standard_normal((fin[2], fin[1], fin[0])).astype(np.float32)
    img = rng.standard_normal((fout[2], fout[1], fout[0]))
    spec = O.fwd(O.real_to_padded(img, fout, dtype=np.float64), fout, fout).astype(np.complex64)
    ft = _make3(fin, fout, iout)
    out = empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32)
    ft.FwdImageInvFFT(dev(torch, O.real_to_padded(t, fin)), dev(torch, spec.view(np.float32)), out)
    got = O.real_from_padded(host(out), iout)
    ref = O.real_from_padded(O.fwd_image_inv(O.real_to_padded(t, fin), spec, O.Plan(fin, fout, fout, iout),
                                             out_dtype=np.float64), iout)
    assert O.rel_l2(got, ref) <= RTOL_L2_BLUE
    assert O.rel_max(got, ref) <= RTOL_MAX_BLUE


def test_forward_c2c_3d(torch_cuda):
    torch = torch_cuda
    fin, fout = (16, 16, 16), (100, 60, 50)
    x = _crand((fin[2], fin[1], fin[0]), 31)
    ft = _make3(fin, fout, fout, input_dtype="complex64")
    out = empty(torch, ft.ReturnFwdOutputMemorySize(), torch.float32)
    ft.FwdFFT(_cbuf(torch, x), out)
    ref = O.fwd_c2c(x, fin, fout)
    got = host(out)[: 2 * ref.size].view(np.complex64).reshape(ref.shape)
    assert O.rel_l2(got, ref) <= RTOL_L2_BLUE
    assert O.rel_max(got, ref) <= RTOL_MAX_BLUE
