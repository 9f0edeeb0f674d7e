"""Image reuse (fastfft_set_image_reuse): the reduced spectrum prepared for an image address
is kept across calls, and single FwdImageInvFFT calls take the reduced-size path.

The library's launch counter tells whether a call prepared the image (four launches) or
only ran the template passes (three launches: row R2C, fused column pass, row C2R).
"""
import numpy as np
import pytest

import fastfft_b200 as F
from oracle import fastfft_oracle as O
from tests._util import RTOL_L2_FP32, RTOL_MAX_FP32, dev, empty, host

pytestmark = pytest.mark.gpu

PREP, BATCH = 4, 3
FIN, FOUT, IOUT = (384, 384, 1), (2048, 2048, 1), (1024, 1024, 1)   # correlates at 1536^2


def plan():
    ft = F.FourierTransformer()
    ft.SetForwardFFTPlan(*FIN, *FOUT)
    ft.SetInverseFFTPlan(*FOUT, *IOUT)
    return ft


def spectrum(seed):
    img = np.random.default_rng(seed).standard_normal((FOUT[1], FOUT[0]))
    return O.fwd(O.real_to_padded(img, FOUT, dtype=np.float64), FOUT, FOUT).astype(np.complex64)


def oracle(t, spec):
    p = O.Plan(FIN, FOUT, FOUT, IOUT)
    return O.real_from_padded(O.fwd_image_inv(O.real_to_padded(t, FIN), spec, p, out_dtype=np.float64), IOUT)


def counted(ft, fn):
    before = ft.LaunchCount()
    fn()
    return ft.LaunchCount() - before


def test_single_calls_reuse_the_prepared_image(torch_cuda):
    torch = torch_cuda
    ft = plan()
    ft.SetImageReuse(True)
    assert ft.CorrelationSize() == (1536, 1536)
    specs = [spectrum(51), spectrum(52)]
    d_specs = [dev(torch, s.view(np.float32)) for s in specs]
    rng = np.random.default_rng(53)
    ts = [rng.standard_normal((384, 384)).astype(np.float32) for _ in range(4)]
    d_ts = [dev(torch, O.real_to_padded(t, FIN)) for t in ts]
    outs = [empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32) for _ in ts]
    which = [0, 0, 1, 0]        # image 0, again, a new image, image 0 again (prepared anew)
    expect = [PREP + BATCH, BATCH, PREP + BATCH, PREP + BATCH]
    for t, w, o, n in zip(d_ts, which, outs, expect):
        assert counted(ft, lambda: ft.FwdImageInvFFT(t, d_specs[w], o)) == n
    for t, w, o in zip(ts, which, outs):
        ref = oracle(t, specs[w])
        got = O.real_from_padded(host(o), IOUT)
        assert O.rel_l2(got, ref) <= RTOL_L2_FP32
        assert O.rel_max(got, ref) <= RTOL_MAX_FP32


def test_reuse_is_forgotten_on_request_and_stream_change(torch_cuda):
    torch = torch_cuda
    ft = plan()
    ft.SetImageReuse(True)
    d_spec = dev(torch, spectrum(54).view(np.float32))
    t = dev(torch, O.real_to_padded(np.random.default_rng(55).standard_normal((384, 384)).astype(np.float32), FIN))
    out = empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32)
    assert counted(ft, lambda: ft.FwdImageInvFFT(t, d_spec, out)) == PREP + BATCH
    assert counted(ft, lambda: ft.FwdImageInvFFT(t, d_spec, out)) == BATCH
    ft.SetImageReuse(True)                                   # forget
    assert counted(ft, lambda: ft.FwdImageInvFFT(t, d_spec, out)) == PREP + BATCH
    s = torch.cuda.Stream()
    ft.SetStream(s)                                          # another stream: forget
    with torch.cuda.stream(s):
        assert counted(ft, lambda: ft.FwdImageInvFFT(t, d_spec, out)) == PREP + BATCH
    s.synchronize()


def test_batched_calls_reuse_and_match_the_plain_path(torch_cuda):
    torch = torch_cuda
    a, b = plan(), plan()
    a.SetImageReuse(True)
    spec = spectrum(56)
    d_spec = dev(torch, spec.view(np.float32))
    rng = np.random.default_rng(57)
    ts = [dev(torch, O.real_to_padded(rng.standard_normal((384, 384)).astype(np.float32), FIN)) for _ in range(6)]
    out_a = [empty(torch, a.ReturnInvOutputMemorySize(), torch.float32) for _ in ts]
    out_b = [empty(torch, b.ReturnInvOutputMemorySize(), torch.float32) for _ in ts]
    a.FwdImageInvFFTMany(ts[:3], d_spec, out_a[:3])
    n = counted(a, lambda: a.FwdImageInvFFTMany(ts[3:], d_spec, out_a[3:]))
    assert n == BATCH                                        # 3 templates in one launch group
    b.FwdImageInvFFTMany(ts, d_spec, out_b)
    for x, y in zip(out_a, out_b):
        assert torch.equal(x, y)


def test_single_call_without_reuse_keeps_the_full_size_kernels(torch_cuda):
    torch = torch_cuda
    ft = plan()
    d_spec = dev(torch, spectrum(58).view(np.float32))
    t = dev(torch, O.real_to_padded(np.random.default_rng(59).standard_normal((384, 384)).astype(np.float32), FIN))
    out = empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32)
    assert counted(ft, lambda: ft.FwdImageInvFFT(t, d_spec, out)) == 3   # size-N R2C, fused columns, C2R
