"""The allocation-free correlation entry point against the regular one, through the C ABI.

fastfft_fwd_image_inv_2d_noalloc serves callers that cannot allocate device memory where
they correlate (a host application's pool owns the free memory; a steady-state loop must
not stall on cudaMalloc).  It keeps its intermediates in one fixed device array shared by
all calls, so this file runs last and checks two calls in a row (the second call must not
see the first one's leftovers) and the rejection of sizes beyond the array.
"""
import ctypes

import numpy as np
import pytest

import fastfft_b200 as F
from fastfft_b200 import _capi as C
from oracle import fastfft_oracle as O
from tests._util import RTOL_L2_FP32, dev, empty, host

pytestmark = pytest.mark.gpu


def _ref(op):
    return ctypes.byref(op) if op is not None else None


def _noalloc(lib, t, in_x, in_y, img, n_x, n_y, out, out_x, out_y, stream, pre=None, intra=None, post=None):
    intra = intra if intra is not None else C.fastfft_op(C.OP_CONJ_MUL, 1.0)
    return lib.fastfft_fwd_image_inv_2d_noalloc(t.data_ptr(), in_x, in_y, img.data_ptr(), n_x, n_y, out.data_ptr(),
                                                out_x, out_y, _ref(pre), _ref(intra), _ref(post), stream)


@pytest.mark.parametrize("fin,fout,iout", [((384, 384, 1), (4096, 4096, 1), (1024, 1024, 1)),
                                           ((48, 40, 1), (256, 128, 1), (200, 100, 1))])
def test_noalloc_matches_regular_entry_point(torch_cuda, fin, fout, iout):
    torch = torch_cuda
    lib = C.lib()
    rng = np.random.default_rng(31)
    img = rng.standard_normal((fout[1], fout[0]))
    spec = dev(torch, O.fwd(O.real_to_padded(img, fout, dtype=np.float64), fout, fout).astype(np.complex64)
               .view(np.float32))
    ft = F.FourierTransformer()
    ft.SetForwardFFTPlan(*fin, *fout)
    ft.SetInverseFFTPlan(*fout, *iout)
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):  # two calls in a row share the scratch array
        t = dev(torch, O.real_to_padded(rng.standard_normal((fin[1], fin[0])).astype(np.float32), fin))
        want = empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32)
        got = torch.full_like(want, float("nan"))
        ft.FwdImageInvFFT(t, spec, want)
        st = _noalloc(lib, t, fin[0], fin[1], spec, fout[0], fout[1], got, iout[0], iout[1], stream)
        assert st == C.OK, lib.fastfft_last_error(None)
        torch.cuda.synchronize()
        a = O.real_from_padded(host(got), iout)
        b = O.real_from_padded(host(want), iout)
        assert np.isfinite(a).all()
        assert O.rel_l2(a, b) <= RTOL_L2_FP32, f"call {call}"


def test_noalloc_rejects_sizes_beyond_its_scratch(torch_cuda):
    torch = torch_cuda
    lib = C.lib()
    t = torch.zeros(16, device="cuda")
    img = torch.zeros(16, device="cuda")
    out = torch.zeros(16, device="cuda")
    # 8192^2 with 384 template rows and a 1024-row window needs ~46 MB of scratch
    st = _noalloc(lib, t, 384, 384, img, 8192, 8192, out, 1024, 1024, None)
    assert st == C.ERR_UNSUPPORTED
    assert b"scratch" in lib.fastfft_last_error(None)
    st = _noalloc(lib, t, 384, 384, img, 4096, 4096, out, 5000, 1024, None)
    assert st == C.ERR_INVALID_DIMS


def test_noalloc_odd_sizes_and_functors(torch_cuda):
    """Odd template width and window height (odd pitches, the single-row C2R branch), with
    pre SCALE, CONJ_MUL_THEN_SCALE and post SCALE, against FwdImageInvFFT with the same
    functors."""
    torch = torch_cuda
    lib = C.lib()
    fin, fout, iout = (47, 41, 1), (256, 128, 1), (199, 101, 1)
    rng = np.random.default_rng(35)
    img = rng.standard_normal((fout[1], fout[0]))
    spec = dev(torch, O.fwd(O.real_to_padded(img, fout, dtype=np.float64), fout, fout).astype(np.complex64)
               .view(np.float32))
    ft = F.FourierTransformer()
    ft.SetForwardFFTPlan(*fin, *fout)
    ft.SetInverseFFTPlan(*fout, *iout)
    pre = C.fastfft_op(C.OP_SCALE, 0.5)
    intra = C.fastfft_op(C.OP_CONJ_MUL_THEN_SCALE, 0.25)
    post = C.fastfft_op(C.OP_SCALE, 2.0)
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        t = dev(torch, O.real_to_padded(rng.standard_normal((fin[1], fin[0])).astype(np.float32), fin))
        want = empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32)
        got = torch.full_like(want, float("nan"))
        ft.FwdImageInvFFT(t, spec, want, pre, intra, post)
        st = _noalloc(lib, t, fin[0], fin[1], spec, fout[0], fout[1], got, iout[0], iout[1], stream, pre, intra, post)
        assert st == C.OK, lib.fastfft_last_error(None)
        torch.cuda.synchronize()
        a = O.real_from_padded(host(got), iout)
        b = O.real_from_padded(host(want), iout)
        assert np.isfinite(a).all()
        assert O.rel_l2(a, b) <= RTOL_L2_FP32, f"call {call}"


def test_noalloc_steady_state_allocates_nothing(torch_cuda):
    """After the first call on the device, a call leaves the device's free memory unchanged."""
    torch = torch_cuda
    lib = C.lib()
    fin, fout, iout = (384, 384, 1), (4096, 4096, 1), (1024, 1024, 1)
    spec = torch.zeros(2 * (fout[0] // 2 + 1) * fout[1], device="cuda")
    t = torch.zeros(O.padded_memory_size(fin), device="cuda")
    out = torch.zeros(O.padded_memory_size(iout), device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    assert _noalloc(lib, t, fin[0], fin[1], spec, fout[0], fout[1], out, iout[0], iout[1], stream) == C.OK
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        assert _noalloc(lib, t, fin[0], fin[1], spec, fout[0], fout[1], out, iout[0], iout[1], stream) == C.OK
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after == free_before
