"""Split-precision tensor-core option of the batched correlation (fastfft_set_tensor_core_dft):
the radix-16 passes of the fused column pass at length 1536 run as BF16 hi/lo matrix products
with FP32 accumulation.  The bound for this form is 1e-4 relative L2 against FP64, and the
peak must stay where the FP32 path puts it.
"""
import numpy as np
import pytest

import fastfft_b200 as F
from oracle import fastfft_oracle as O
from tests._util import dev, empty, host

pytestmark = pytest.mark.gpu

RTOL_L2_TC = 1e-4

FIN, FOUT, IOUT = (64, 200, 1), (2048, 2048, 1), (200, 1100, 1)    # correlates at (384, 1536)


def plan(tc):
    ft = F.FourierTransformer()
    ft.SetForwardFFTPlan(*FIN, *FOUT)
    ft.SetInverseFFTPlan(*FOUT, *IOUT)
    ft.SetTensorCoreDFT(tc)
    return ft


def test_active_only_where_the_pass_has_that_form(torch_cuda):
    assert plan(True).TensorCoreDFTActive()
    assert not plan(False).TensorCoreDFTActive()
    other = F.FourierTransformer()
    other.SetForwardFFTPlan(64, 64, 1, 1024, 1024, 1)
    other.SetInverseFFTPlan(1024, 1024, 1, 256, 256, 1)              # correlates at 384^2
    other.SetTensorCoreDFT(True)
    assert not other.TensorCoreDFTActive()
    forced = plan(True)
    forced.SetFullSizeCorrelation(True)
    assert not forced.TensorCoreDFTActive()


def test_split_precision_matches_oracle_and_fp32_peaks(torch_cuda):
    torch = torch_cuda
    img = O.gaussian_blob_image(2048, n_blobs=8, seed=41)
    spec = O.image_spectrum_fp32(img)
    d_spec = dev(torch, spec.view(np.float32))
    rng = np.random.default_rng(42)
    # templates cut from the image at lags inside the window, plus noise: a clear peak there
    ts = []
    for i in range(5):
        y0, x0 = rng.integers(0, IOUT[1] - 100), rng.integers(0, IOUT[0] - 20)
        t = img[y0:y0 + FIN[1], x0:x0 + FIN[0]].astype(np.float32) + 0.1 * rng.standard_normal((FIN[1], FIN[0]))
        ts.append(t.astype(np.float32))
    d_ts = [dev(torch, O.real_to_padded(t, FIN)) for t in ts]
    tc, fp = plan(True), plan(False)
    out_tc = [empty(torch, tc.ReturnInvOutputMemorySize(), torch.float32) for _ in ts]
    out_fp = [empty(torch, fp.ReturnInvOutputMemorySize(), torch.float32) for _ in ts]
    tc.FwdImageInvFFTMany(d_ts, d_spec, out_tc)
    fp.FwdImageInvFFTMany(d_ts, d_spec, out_fp)
    torch.cuda.synchronize()
    p = O.Plan(FIN, FOUT, FOUT, IOUT)
    for t, a, b in zip(ts, out_tc, out_fp):
        ref = O.real_from_padded(O.fwd_image_inv(O.real_to_padded(t, FIN), spec, p, out_dtype=np.float64), IOUT)
        got_tc = O.real_from_padded(host(a), IOUT)
        got_fp = O.real_from_padded(host(b), IOUT)
        err_tc = O.rel_l2(got_tc, ref)
        assert err_tc <= RTOL_L2_TC
        assert err_tc > O.rel_l2(got_fp, ref)            # the split form is the less accurate one
        assert O.peak(got_tc)[0] == O.peak(got_fp)[0] == O.peak(ref)[0]


def test_low_precision_image_with_tensor_core_passes(torch_cuda):
    torch = torch_cuda
    spec = O.image_spectrum_fp32(O.gaussian_blob_image(2048, n_blobs=4, seed=43)) / 2048
    ft = F.FourierTransformer(image_dtype="complex_bf16")
    ft.SetForwardFFTPlan(*FIN, *FOUT)
    ft.SetInverseFFTPlan(*FOUT, *IOUT)
    ft.SetTensorCoreDFT(True)
    assert ft.TensorCoreDFTActive()
    spec_bf = torch.from_numpy(spec.view(np.float32).copy()).to(torch.bfloat16).cuda()
    spec_deq = spec_bf.float().cpu().numpy().view(np.complex64).reshape(spec.shape)
    t = np.random.default_rng(44).standard_normal((FIN[1], FIN[0])).astype(np.float32)
    out = empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32)
    ft.FwdImageInvFFTMany([dev(torch, O.real_to_padded(t, FIN))], spec_bf, [out])
    torch.cuda.synchronize()
    p = O.Plan(FIN, FOUT, FOUT, IOUT)
    ref = O.real_from_padded(O.fwd_image_inv(O.real_to_padded(t, FIN), spec_deq, p, out_dtype=np.float64), IOUT)
    assert O.rel_l2(O.real_from_padded(host(out), IOUT), ref) <= RTOL_L2_TC


HEAD_FIN, HEAD_FOUT, HEAD_IOUT = (384, 384, 1), (2048, 2048, 1), (1024, 1024, 1)   # correlates at 1536^2


def _plan(fin, fout, iout, tc):
    ft = F.FourierTransformer()
    ft.SetForwardFFTPlan(*fin, *fout)
    ft.SetInverseFFTPlan(*fout, *iout)
    ft.SetTensorCoreDFT(tc)
    return ft


def _blob_case(torch, seed):
    img = O.gaussian_blob_image(HEAD_FOUT[0], n_blobs=12, seed=seed)
    spec = O.image_spectrum_fp32(img)
    return img, spec, dev(torch, spec.view(np.float32))


@pytest.mark.parametrize("intra", ["conj_mul_then_scale", "noop"])
def test_benchmark_shape_partial_work_item(torch_cuda, intra):
    """384^2 templates and 1024^2 windows (the 1536^2 correlation of the benchmark workload), 6
    templates: the tensor-core pass takes 4 templates per work item, so the second item is half
    empty (CONJ_MUL_THEN_SCALE).  With NOOP the call is a round trip of the template, which the
    reduced size would scale differently: it runs at the plan's size."""
    torch = torch_cuda
    img, spec, d_spec = _blob_case(torch, 51)
    rng = np.random.default_rng(52)
    ts = []
    for i in range(6):
        y0, x0 = rng.integers(0, 600, size=2)
        ts.append((img[y0:y0 + 384, x0:x0 + 384] + 0.2 * rng.standard_normal((384, 384))).astype(np.float32))
    op = F.KernelFunction.conj_mul_then_scale(0.125) if intra != "noop" else F.KernelFunction.noop()
    oop = (O.OP_CONJ_MUL_THEN_SCALE, 0.125) if intra != "noop" else (O.OP_NOOP, 1.0)
    tc, fp = _plan(HEAD_FIN, HEAD_FOUT, HEAD_IOUT, True), _plan(HEAD_FIN, HEAD_FOUT, HEAD_IOUT, False)
    assert tc.TensorCoreDFTActive() and tc.CorrelationSize() == (1536, 1536)
    d_ts = [dev(torch, O.real_to_padded(t, HEAD_FIN)) for t in ts]
    out_tc = [empty(torch, tc.ReturnInvOutputMemorySize(), torch.float32) for _ in ts]
    out_fp = [empty(torch, fp.ReturnInvOutputMemorySize(), torch.float32) for _ in ts]
    tc.FwdImageInvFFTMany(d_ts, d_spec, out_tc, intra_op=op)
    fp.FwdImageInvFFTMany(d_ts, d_spec, out_fp, intra_op=op)
    torch.cuda.synchronize()
    p = O.Plan(HEAD_FIN, HEAD_FOUT, HEAD_FOUT, HEAD_IOUT)
    for t, a, b in zip(ts, out_tc, out_fp):
        ref = O.real_from_padded(O.fwd_image_inv(O.real_to_padded(t, HEAD_FIN), spec, p, intra_op=oop,
                                                 out_dtype=np.float64), HEAD_IOUT)
        got_tc = O.real_from_padded(host(a), HEAD_IOUT)
        assert O.rel_l2(got_tc, ref) <= RTOL_L2_TC
        if intra != "noop":
            assert O.peak(got_tc)[0] == O.peak(O.real_from_padded(host(b), HEAD_IOUT))[0] == O.peak(ref)[0]


def test_uneven_template_rows_in_one_work_item(torch_cuda):
    """Templates of 258..384 rows share the 1536-point class, so one work item mixes lengths
    (the tensor-core pass zero-fills each template's rows beyond its own)."""
    torch = torch_cuda
    img, spec, d_spec = _blob_case(torch, 53)
    rng = np.random.default_rng(54)
    sizes = [(384, 384), (384, 300), (384, 262), (200, 384), (384, 333), (384, 258), (300, 300)]
    ts = [rng.standard_normal((y, x)).astype(np.float32) for x, y in sizes]
    ft = _plan(HEAD_FIN, HEAD_FOUT, HEAD_IOUT, True)
    ins = [dev(torch, O.real_to_padded(t, (x, y, 1))) for t, (x, y) in zip(ts, sizes)]
    outs = [empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32) for _ in ts]
    ft.FwdImageInvFFTManySized(ins, sizes, d_spec, outs)
    torch.cuda.synchronize()
    for t, (x, y), o in zip(ts, sizes, outs):
        p = O.Plan((x, y, 1), HEAD_FOUT, HEAD_FOUT, HEAD_IOUT)
        ref = O.real_from_padded(O.fwd_image_inv(O.real_to_padded(t, (x, y, 1)), spec, p, out_dtype=np.float64),
                                 HEAD_IOUT)
        assert O.rel_l2(O.real_from_padded(host(o), HEAD_IOUT), ref) <= RTOL_L2_TC, (x, y)


def test_tall_templates_fall_back_to_fp32(torch_cuda):
    """Templates of more than 512 rows (the tensor-core pass reads n < 512) run the FP32 pass."""
    ft = _plan((64, 520, 1), (2048, 2048, 1), (64, 1000, 1), True)
    assert ft.CorrelationSize()[1] == 1536
    assert not ft.TensorCoreDFTActive()


@pytest.mark.parametrize("per_launch,groups", [(3, 2), (5, 1), (16, 2)])
def test_several_launches_and_groups_in_flight(torch_cuda, per_launch, groups):
    """The tensor-core pass with several launches per call and two groups in flight on two
    streams (each launch takes whole SMs and all of their tensor memory while it runs):
    windows identical to one launch of the same pass."""
    torch = torch_cuda
    img, spec, d_spec = _blob_case(torch, 55)
    rng = np.random.default_rng(56)
    ts = [rng.standard_normal((384, 384)).astype(np.float32) for _ in range(11)]
    d_ts = [dev(torch, O.real_to_padded(t, HEAD_FIN)) for t in ts]
    results = []
    for pl, gr in ((64, 1), (per_launch, groups)):
        ft = _plan(HEAD_FIN, HEAD_FOUT, HEAD_IOUT, True)
        ft.SetTemplatesPerLaunch(pl)
        ft.SetPipelinedGroups(gr)
        assert ft.TensorCoreDFTActive()
        outs = [empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32) for _ in ts]
        ft.FwdImageInvFFTMany(d_ts, d_spec, outs)
        torch.cuda.synchronize()
        results.append([host(o) for o in outs])
    for a, b in zip(*results):
        assert np.array_equal(a, b)


def test_longest_template_and_widest_window(torch_cuda):
    """The pass's limits: 512-row templates (F1 reads n1 < 16 of 32-row steps) and a 1025-row
    window (the inverse keeps n1 < 48, N = 96 of the last product), L + W - 1 = 1536 exactly."""
    torch = torch_cuda
    fin, fout, iout = (64, 512, 1), (2048, 2048, 1), (300, 1025, 1)
    ft = _plan(fin, fout, iout, True)
    assert ft.CorrelationSize()[1] == 1536 and ft.TensorCoreDFTActive()
    img = O.gaussian_blob_image(2048, n_blobs=8, seed=57)
    spec = O.image_spectrum_fp32(img)
    d_spec = dev(torch, spec.view(np.float32))
    rng = np.random.default_rng(58)
    ts = [rng.standard_normal((fin[1], fin[0])).astype(np.float32) for _ in range(5)]
    outs = [empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32) for _ in ts]
    ft.FwdImageInvFFTMany([dev(torch, O.real_to_padded(t, fin)) for t in ts], d_spec, outs)
    torch.cuda.synchronize()
    p = O.Plan(fin, fout, fout, iout)
    for t, o in zip(ts, outs):
        ref = O.real_from_padded(O.fwd_image_inv(O.real_to_padded(t, fin), spec, p, out_dtype=np.float64), iout)
        assert O.rel_l2(O.real_from_padded(host(o), iout), ref) <= RTOL_L2_TC
