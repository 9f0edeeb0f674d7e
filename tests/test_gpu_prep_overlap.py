"""The reduced-size path prepares each image on a second stream of the plan, overlapping the
templates' row R2C, and joins it before the fused column pass.  These tests stress the
ordering: several images per call with small launch groups (a preparation must wait for the
column passes that still read the previous image's spectrum), back-to-back calls without a
host synchronisation, and the whole call captured in a CUDA graph.
"""
import numpy as np
import pytest

import fastfft_b200 as F
from oracle import fastfft_oracle as O
from tests._util import RTOL_L2_FP32, RTOL_MAX_FP32, dev, empty, host

pytestmark = pytest.mark.gpu

FIN, FOUT, IOUT = (64, 64, 1), (1024, 1024, 1), (200, 200, 1)     # correlates at 384^2


def plan():
    ft = F.FourierTransformer()
    ft.SetForwardFFTPlan(*FIN, *FOUT)
    ft.SetInverseFFTPlan(*FOUT, *IOUT)
    return ft


def spectrum(seed):
    img = np.random.default_rng(seed).standard_normal((FOUT[1], FOUT[0]))
    return O.fwd(O.real_to_padded(img, FOUT, dtype=np.float64), FOUT, FOUT).astype(np.complex64)


def check(outs, ts, which, specs):
    p = O.Plan(FIN, FOUT, FOUT, IOUT)
    for o, t, w in zip(outs, ts, which):
        ref = O.real_from_padded(O.fwd_image_inv(O.real_to_padded(t, FIN), specs[w], p, out_dtype=np.float64), IOUT)
        got = O.real_from_padded(host(o), IOUT)
        assert O.rel_l2(got, ref) <= RTOL_L2_FP32
        assert O.rel_max(got, ref) <= RTOL_MAX_FP32


def test_interleaved_images_back_to_back(torch_cuda):
    torch = torch_cuda
    ft = plan()
    assert ft.CorrelationSize() == (384, 384)
    ft.SetTemplatesPerLaunch(4)
    specs = [spectrum(300 + i) for i in range(3)]
    d_specs = [dev(torch, s.view(np.float32)) for s in specs]
    rng = np.random.default_rng(310)
    ts = [rng.standard_normal((64, 64)).astype(np.float32) for _ in range(14)]
    d_ts = [dev(torch, O.real_to_padded(t, FIN)) for t in ts]
    which_a = [i % 3 for i in range(14)]
    which_b = [(2 * i + 1) % 3 for i in range(14)]
    outs_a = [empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32) for _ in ts]
    outs_b = [empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32) for _ in ts]
    # two calls in a row, no synchronisation in between: the second call's first preparation
    # forks after the first call's last column pass
    ft.FwdImageInvFFTMany(d_ts, [d_specs[w] for w in which_a], outs_a)
    ft.FwdImageInvFFTMany(d_ts, [d_specs[w] for w in which_b], outs_b)
    torch.cuda.synchronize()
    check(outs_a, ts, which_a, specs)
    check(outs_b, ts, which_b, specs)


def test_graph_capture_replays_the_call(torch_cuda):
    torch = torch_cuda
    ft = plan()
    specs = [spectrum(320), spectrum(321)]
    d_specs = [dev(torch, s.view(np.float32)) for s in specs]
    rng = np.random.default_rng(322)
    ts = [rng.standard_normal((64, 64)).astype(np.float32) for _ in range(6)]
    d_ts = [dev(torch, O.real_to_padded(t, FIN)) for t in ts]
    which = [0, 1, 1, 0, 1, 0]
    outs = [empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32) for _ in ts]
    ft.FwdImageInvFFTMany(d_ts, [d_specs[w] for w in which], outs)      # allocates, tunes nothing
    torch.cuda.synchronize()
    for o in outs:
        o.zero_()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        ft.FwdImageInvFFTMany(d_ts, [d_specs[w] for w in which], outs)
    graph.replay()
    torch.cuda.synchronize()
    check(outs, ts, which, specs)
    # new template contents through the same graph
    ts2 = [rng.standard_normal((64, 64)).astype(np.float32) for _ in range(6)]
    for d, t in zip(d_ts, ts2):
        d.copy_(torch.from_numpy(O.real_to_padded(t, FIN).reshape(-1)).to(d.device))
    graph.replay()
    torch.cuda.synchronize()
    check(outs, ts2, which, specs)
    del graph
