"""Seeded random sweep of plan shapes and functors against the FP64 oracle.

Each case draws a transform length per axis among powers of two, 3 * 2^k, 5 * 2^k and 7 * 2^k, a
template (forward input) no larger than the transform, a window (inverse output) no larger
than it, functors among NOOP / SCALE / CONJ_MUL / CONJ_MUL_THEN_SCALE, and runs the
correlation through the single call (size-N kernels), the batched call (reduced size where
shorter) and, for the same plan, a FwdFFT and an InvFFT.  Sizes stay small enough for the
oracle to finish in well under a second per case.
"""
import numpy as np
import pytest

import fastfft_b200 as F
from oracle import fastfft_oracle as O
from tests._util import RTOL_L2_FP32, dev, empty, host, spectrum_view

pytestmark = pytest.mark.gpu

LENGTHS = [64, 128, 256, 384, 512, 640, 768, 896, 1024, 1280, 1792]


def draw(seed):
    rng = np.random.default_rng(seed)
    nx, ny = (int(v) for v in rng.choice(LENGTHS, 2))
    lx, ly = int(rng.integers(1, nx + 1)), int(rng.integers(1, ny + 1))
    wx, wy = int(rng.integers(1, nx + 1)), int(rng.integers(1, ny + 1))
    pre = (O.OP_SCALE, float(rng.uniform(0.5, 2))) if rng.random() < 0.5 else (O.OP_NOOP, 1.0)
    intra = (O.OP_CONJ_MUL_THEN_SCALE, float(rng.uniform(0.5, 2))) if rng.random() < 0.5 else (O.OP_CONJ_MUL, 1.0)
    post = (O.OP_SCALE, float(rng.uniform(0.5, 2))) if rng.random() < 0.5 else (O.OP_NOOP, 1.0)
    return (lx, ly, 1), (nx, ny, 1), (wx, wy, 1), pre, intra, post


def op(kind_scale):
    kind, s = kind_scale
    K = F.KernelFunction
    return {O.OP_NOOP: K.noop(), O.OP_SCALE: K.scale(s), O.OP_CONJ_MUL: K.conj_mul(),
            O.OP_CONJ_MUL_THEN_SCALE: K.conj_mul_then_scale(s)}[kind]


@pytest.mark.parametrize("seed", range(48))
def test_random_plan(torch_cuda, seed):
    torch = torch_cuda
    fin, fout, iout, pre, intra, post = draw(1000 + seed)
    rng = np.random.default_rng(seed)
    t = rng.standard_normal((fin[1], fin[0])).astype(np.float32)
    img = rng.standard_normal((fout[1], fout[0]))
    spec = O.fwd(O.real_to_padded(img, fout, dtype=np.float64), fout, fout).astype(np.complex64)
    ft = F.FourierTransformer()
    ft.SetForwardFFTPlan(*fin, *fout)
    ft.SetInverseFFTPlan(*fout, *iout)
    p = O.Plan(fin, fout, fout, iout)
    t_pad = O.real_to_padded(t, fin)
    ref = O.real_from_padded(O.fwd_image_inv(t_pad, spec, p, pre, intra, post, out_dtype=np.float64), iout)
    d_t, d_spec = dev(torch, t_pad), dev(torch, spec.view(np.float32))
    single = empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32)
    ft.FwdImageInvFFT(d_t, d_spec, single, op(pre), op(intra), op(post))
    batched = [empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32) for _ in range(2)]
    ft.FwdImageInvFFTMany([d_t, d_t], d_spec, batched, op(pre), op(intra), op(post))
    for o in [single] + batched:
        got = O.real_from_padded(host(o), iout)
        assert O.rel_l2(got, ref) <= RTOL_L2_FP32, (fin, fout, iout, pre, intra, post, ft.CorrelationSize())
    # forward and inverse of the same plan
    spec_out = empty(torch, ft.ReturnFwdOutputMemorySize(), torch.float32)
    ft.FwdFFT(d_t, spec_out, op(pre))
    want = O.fwd(t_pad, fin, fout, pre)
    assert O.rel_l2(spectrum_view(spec_out, fout), want) <= RTOL_L2_FP32
    out = empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32)
    ft.InvFFT(d_spec, out, None, op(post))
    want = O.real_from_padded(O.inv(spec, fout, iout, post, out_dtype=np.float64), iout)
    assert O.rel_l2(O.real_from_padded(host(out), iout), want) <= RTOL_L2_FP32
