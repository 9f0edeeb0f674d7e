"""Batched correlation (fastfft_fwd_image_inv_many) against the FP64 oracle.

The batched call correlates at the smallest exact size M >= L + W - 1 per axis (a power
of two or 3 * 2^k) when M < N; these tests check that the retained window equals the size-N correlation
the reference defines (FwdImageInvFFT, conj(T) * I, origin-anchored crop).
"""
import numpy as np
import pytest

import fastfft_b200 as F
from oracle import fastfft_oracle as O
from tests._util import RTOL_L2_FP32, RTOL_MAX_FP32, dev, empty, host

pytestmark = pytest.mark.gpu


def plan(fin, fout, iout, **kw):
    ft = F.FourierTransformer(**kw)
    ft.SetForwardFFTPlan(*fin, *fout)
    ft.SetInverseFFTPlan(*fout, *iout)
    return ft


def image_spectrum(fout, seed):
    img = np.random.default_rng(seed).standard_normal((fout[1], fout[0]))
    return O.fwd(O.real_to_padded(img, fout, dtype=np.float64), fout, fout).astype(np.complex64)


CASES = [
    ((48, 48, 1), (512, 512, 1), (40, 40, 1), (128, 128)),
    ((100, 60, 1), (1024, 512, 1), (130, 70, 1), (256, 256)),
    ((128, 128, 1), (4096, 4096, 1), (512, 512, 1), (768, 768)),     # 639 -> 3 * 256
    ((256, 256, 1), (1024, 1024, 1), (512, 512, 1), (768, 768)),
    ((256, 256, 1), (512, 512, 1), (300, 300, 1), (512, 512)),       # 555 > 512: full size
    ((33, 200, 1), (64, 2048, 1), (30, 100, 1), (64, 384)),
]


@pytest.mark.parametrize("fin,fout,iout,msize", CASES)
def test_many_matches_oracle(torch_cuda, fin, fout, iout, msize):
    torch = torch_cuda
    ft = plan(fin, fout, iout)
    assert ft.CorrelationSize() == msize
    specs = [image_spectrum(fout, s) for s in (1, 2)]
    d_specs = [dev(torch, s.view(np.float32)) for s in specs]
    rng = np.random.default_rng(5)
    ts = [rng.standard_normal((fin[1], fin[0])).astype(np.float32) for _ in range(5)]
    which = [0, 1, 0, 0, 1]                      # interleaved images: grouping must keep pairs
    ins = [dev(torch, O.real_to_padded(t, fin)) for t in ts]
    outs = [empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32) for _ in ts]
    ft.FwdImageInvFFTMany(ins, [d_specs[w] for w in which], outs)
    p = O.Plan(fin, fout, fout, iout)
    for t, w, o in zip(ts, which, outs):
        ref = O.real_from_padded(O.fwd_image_inv(O.real_to_padded(t, fin), specs[w], p, out_dtype=np.float64), iout)
        got = O.real_from_padded(host(o), iout)
        assert O.rel_l2(got, ref) <= RTOL_L2_FP32
        assert O.rel_max(got, ref) <= RTOL_MAX_FP32


def test_many_equals_full_size_path(torch_cuda):
    torch = torch_cuda
    fin, fout, iout = (64, 64, 1), (1024, 1024, 1), (200, 200, 1)
    spec = dev(torch, image_spectrum(fout, 9).view(np.float32))
    t = dev(torch, O.real_to_padded(np.random.default_rng(3).standard_normal((64, 64)).astype(np.float32), fin))
    a = plan(fin, fout, iout)
    b = plan(fin, fout, iout)
    b.SetFullSizeCorrelation(True)
    assert a.CorrelationSize() == (384, 384) and b.CorrelationSize() == (1024, 1024)
    oa, ob, oc = (empty(torch, a.ReturnInvOutputMemorySize(), torch.float32) for _ in range(3))
    a.FwdImageInvFFTMany([t], spec, [oa])
    b.FwdImageInvFFTMany([t], spec, [ob])
    a.FwdImageInvFFT(t, spec, oc)                       # single call: size-N kernels
    ra, rb, rc = (O.real_from_padded(host(x), iout) for x in (oa, ob, oc))
    assert np.array_equal(rb, rc)
    assert O.rel_l2(ra, rc) <= RTOL_L2_FP32


def test_many_headline_shape_peak(torch_cuda):
    """384^2 template, 4096^2 image (noise + blobs), 1024^2 window: computed at 1536^2."""
    torch = torch_cuda
    n, L, W = 4096, 384, 1024
    spec = O.image_spectrum_fp32(O.gaussian_blob_image(n))
    t = O.normal_template(L, O.SEED_BASE + 1).astype(np.float32)
    fin, fout, iout = (L, L, 1), (n, n, 1), (W, W, 1)
    ft = plan(fin, fout, iout)
    assert ft.CorrelationSize() == (1536, 1536)
    out = empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32)
    ft.FwdImageInvFFTMany([dev(torch, O.real_to_padded(t, fin))], dev(torch, spec.view(np.float32)), [out])
    got = O.real_from_padded(host(out), iout)[0]
    p = O.Plan(fin, fout, fout, iout)
    ref = O.real_from_padded(O.fwd_image_inv(O.real_to_padded(t, fin), spec, p, out_dtype=np.float64), iout)[0]
    assert O.rel_l2(got, ref) <= RTOL_L2_FP32
    gi, _, _ = O.peak(got)
    ri, _, _ = O.peak(ref)
    assert gi == ri


@pytest.mark.parametrize("img_dt", ["complex32", "complex_bf16"])
def test_many_low_precision_image(torch_cuda, img_dt):
    torch = torch_cuda
    fin, fout, iout = (96, 96, 1), (1024, 1024, 1), (256, 256, 1)
    tdt = torch.float16 if img_dt == "complex32" else torch.bfloat16
    spec = image_spectrum(fout, 4) / 1024
    spec_q = torch.from_numpy(spec.view(np.float32).reshape(-1)).to(tdt)
    spec_deq = spec_q.float().numpy().view(np.complex64).reshape(spec.shape)
    ft = plan(fin, fout, iout, image_dtype=img_dt)
    t = np.random.default_rng(8).standard_normal((96, 96)).astype(np.float32)
    out = empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32)
    ft.FwdImageInvFFTMany([dev(torch, O.real_to_padded(t, fin))], spec_q.cuda(), [out])
    p = O.Plan(fin, fout, fout, iout)
    ref = O.real_from_padded(O.fwd_image_inv(O.real_to_padded(t, fin), spec_deq, p, out_dtype=np.float64), iout)
    assert O.rel_l2(O.real_from_padded(host(out), iout), ref) <= RTOL_L2_FP32


@pytest.mark.parametrize("force_full", [False, True])
def test_many_sized_uneven_templates(torch_cuda, force_full):
    """Uneven template sizes in one call (one plan for the largest), against the oracle."""
    torch = torch_cuda
    fmax, fout, iout = (96, 96, 1), (1024, 1024, 1), (128, 128, 1)
    ft = plan(fmax, fout, iout)
    ft.SetFullSizeCorrelation(force_full)
    assert ft.CorrelationSize() == ((1024, 1024) if force_full else (256, 256))
    spec = image_spectrum(fout, 12)
    d_spec = dev(torch, spec.view(np.float32))
    rng = np.random.default_rng(13)
    sizes = [(32, 32), (96, 96), (48, 64), (96, 40), (64, 64), (17, 95), (96, 96), (33, 33), (80, 20), (64, 96)]
    ts = [rng.standard_normal((y, x)).astype(np.float32) for x, y in sizes]
    ins = [dev(torch, O.real_to_padded(t, (x, y, 1))) for t, (x, y) in zip(ts, sizes)]
    outs = [empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32) for _ in ts]
    ft.FwdImageInvFFTManySized(ins, sizes, d_spec, outs)
    for t, (x, y), o in zip(ts, sizes, outs):
        p = O.Plan((x, y, 1), fout, fout, iout)
        ref = O.real_from_padded(O.fwd_image_inv(O.real_to_padded(t, (x, y, 1)), spec, p, out_dtype=np.float64), iout)
        got = O.real_from_padded(host(o), iout)
        assert O.rel_l2(got, ref) <= RTOL_L2_FP32, (x, y)


def test_many_sized_rejects_oversized_template(torch_cuda):
    ft = plan((64, 64, 1), (512, 512, 1), (64, 64, 1))
    t = torch_cuda.zeros(8192, device="cuda")
    spec = torch_cuda.zeros(2 * 257 * 512, device="cuda")
    out = torch_cuda.zeros(66 * 64, device="cuda")
    with pytest.raises(F.FastFFTError) as e:
        ft.FwdImageInvFFTManySized([t], [(65, 64)], spec, [out])
    assert "larger than the plan" in str(e.value)


@pytest.mark.parametrize("per_launch", [1, 3, 16])
def test_templates_per_launch_setting(torch_cuda, per_launch):
    torch = torch_cuda
    fin, fout, iout = (40, 40, 1), (512, 512, 1), (64, 64, 1)
    ft = plan(fin, fout, iout)
    ft.SetTemplatesPerLaunch(per_launch)
    assert ft.TemplatesPerLaunch() == per_launch
    spec = image_spectrum(fout, 21)
    d_spec = dev(torch, spec.view(np.float32))
    rng = np.random.default_rng(2)
    ts = [rng.standard_normal((40, 40)).astype(np.float32) for _ in range(7)]
    outs = [empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32) for _ in ts]
    ft.FwdImageInvFFTMany([dev(torch, O.real_to_padded(t, fin)) for t in ts], d_spec, outs)
    p = O.Plan(fin, fout, fout, iout)
    for t, o in zip(ts, outs):
        ref = O.real_from_padded(O.fwd_image_inv(O.real_to_padded(t, fin), spec, p, out_dtype=np.float64), iout)
        assert O.rel_l2(O.real_from_padded(host(o), iout), ref) <= RTOL_L2_FP32


@pytest.mark.parametrize("write_windows,force_full", [(False, False), (True, False), (False, True)])
def test_many_peaks_match_oracle_argmax(torch_cuda, write_windows, force_full):
    """Fused peak search: max and first-occurrence argmax of every window, bit-exact index."""
    torch = torch_cuda
    fin, fout, iout = (64, 64, 1), (1024, 1024, 1), (200, 150, 1)
    ft = plan(fin, fout, iout)
    ft.SetFullSizeCorrelation(force_full)
    img = O.gaussian_blob_image(1024, n_blobs=6, seed=5)
    spec = O.image_spectrum_fp32(img)
    d_spec = dev(torch, spec.view(np.float32))
    rng = np.random.default_rng(17)
    sizes = [(64, 64), (40, 64), (64, 33), (20, 20), (64, 64), (50, 60)]
    ts = [rng.standard_normal((y, x)).astype(np.float32) for x, y in sizes]
    ins = [dev(torch, O.real_to_padded(t, (x, y, 1))) for t, (x, y) in zip(ts, sizes)]
    outs = [empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32) for _ in ts] if write_windows else None
    peaks = torch.zeros(len(ts), dtype=torch.int64, device="cuda")
    ft.FwdImageInvFFTManyPeaks(ins, d_spec, peaks, sizes=sizes, outputs=outs)
    vals, idx = F.decode_peaks(peaks)
    for i, (t, (x, y)) in enumerate(zip(ts, sizes)):
        p = O.Plan((x, y, 1), fout, fout, iout)
        ref = O.real_from_padded(O.fwd_image_inv(O.real_to_padded(t, (x, y, 1)), spec, p, out_dtype=np.float64),
                                 iout)[0]
        ri, rtop, margin = O.peak(ref)
        if margin > 1e-4 * abs(rtop):
            assert idx[i] == ri, i
        assert abs(vals[i] - rtop) <= 1e-5 * abs(rtop)
        if write_windows:
            got = O.real_from_padded(host(outs[i]), iout)[0]
            assert O.rel_l2(got, ref) <= RTOL_L2_FP32
            assert O.peak(got)[0] == idx[i]


def test_launches_beyond_sixteen_templates(torch_cuda):
    """70 templates at 64 per launch (two launches, template slots past 16): windows and
    fused peaks against the oracle."""
    torch = torch_cuda
    fin, fout, iout = (40, 40, 1), (512, 512, 1), (64, 64, 1)
    ft = plan(fin, fout, iout)
    ft.SetTemplatesPerLaunch(64)
    assert ft.TemplatesPerLaunch() == 64
    spec = O.image_spectrum_fp32(O.gaussian_blob_image(512, n_blobs=4, seed=23))
    d_spec = dev(torch, spec.view(np.float32))
    rng = np.random.default_rng(24)
    ts = [rng.standard_normal((40, 40)).astype(np.float32) for _ in range(70)]
    ins = [dev(torch, O.real_to_padded(t, fin)) for t in ts]
    outs = [empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32) for _ in ts]
    peaks = torch.zeros(len(ts), dtype=torch.int64, device="cuda")
    ft.FwdImageInvFFTManyPeaks(ins, d_spec, peaks, outputs=outs)
    vals, idx = F.decode_peaks(peaks)
    p = O.Plan(fin, fout, fout, iout)
    for i in (0, 16, 17, 40, 63, 64, 69):
        ref = O.real_from_padded(O.fwd_image_inv(O.real_to_padded(ts[i], fin), spec, p, out_dtype=np.float64), iout)
        got = O.real_from_padded(host(outs[i]), iout)
        assert O.rel_l2(got, ref) <= RTOL_L2_FP32, i
        assert O.peak(got[0])[0] == idx[i], i


def test_uneven_templates_use_their_own_size_class(torch_cuda):
    """128^2 and 384^2 templates with 512^2 windows in one call: the 128s correlate at 768
    (128 + 511 <= 3 * 256), the 384s at the plan's 1024; one image preparation per class."""
    torch = torch_cuda
    fmax, fout, iout = (384, 384, 1), (2048, 2048, 1), (512, 512, 1)
    ft = plan(fmax, fout, iout)
    assert ft.CorrelationSize() == (1024, 1024)
    spec = image_spectrum(fout, 25)
    d_spec = dev(torch, spec.view(np.float32))
    rng = np.random.default_rng(26)
    sizes = [(128, 128), (384, 384), (128, 128), (384, 384), (128, 128), (128, 128)]
    ts = [rng.standard_normal((y, x)).astype(np.float32) for x, y in sizes]
    ins = [dev(torch, O.real_to_padded(t, (x, y, 1))) for t, (x, y) in zip(ts, sizes)]
    outs = [empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32) for _ in ts]
    before = ft.LaunchCount()
    ft.FwdImageInvFFTManySized(ins, sizes, d_spec, outs)
    assert ft.LaunchCount() - before == 2 * 4 + 2 * 3      # two preparations, one batch per class
    for t, (x, y), o in zip(ts, sizes, outs):
        p = O.Plan((x, y, 1), fout, fout, iout)
        ref = O.real_from_padded(O.fwd_image_inv(O.real_to_padded(t, (x, y, 1)), spec, p, out_dtype=np.float64), iout)
        got = O.real_from_padded(host(o), iout)
        assert O.rel_l2(got, ref) <= RTOL_L2_FP32, (x, y)
        assert O.rel_max(got, ref) <= RTOL_MAX_FP32, (x, y)


@pytest.mark.parametrize("per_launch", [1, 3, 5])
def test_pipelined_groups_match_single_stream(torch_cuda, per_launch):
    """Two groups in flight (alternating streams, own intermediate slices) give bit-identical
    windows and peaks to one group in flight: interleaved images, uneven sizes (size classes,
    one image preparation per class), an odd number of groups, and a CUDA graph replay."""
    torch = torch_cuda
    fmax, fout, iout = (96, 96, 1), (1024, 1024, 1), (128, 128, 1)
    specs = [dev(torch, image_spectrum(fout, s).view(np.float32)) for s in (21, 22)]
    rng = np.random.default_rng(23)
    sizes = [(96, 96), (32, 32), (96, 96), (64, 48), (96, 96), (17, 95), (96, 80), (33, 33), (96, 96), (80, 20),
             (96, 96)]
    which = [0, 1, 0, 0, 1, 0, 1, 1, 0, 0, 1]
    ins = [dev(torch, O.real_to_padded(rng.standard_normal((y, x)).astype(np.float32), (x, y, 1))) for x, y in sizes]
    results = []
    for groups in (1, 2):
        ft = plan(fmax, fout, iout)
        ft.SetTemplatesPerLaunch(per_launch)
        ft.SetPipelinedGroups(groups)
        assert ft.PipelinedGroups() == groups
        outs = [empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32) for _ in sizes]
        peaks = torch.zeros(len(sizes), dtype=torch.int64, device="cuda")
        ft.FwdImageInvFFTManySized(ins, sizes, [specs[w] for w in which], outs)
        ft.FwdImageInvFFTManyPeaks(ins, [specs[w] for w in which], peaks, sizes=sizes)
        graph_outs = [empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32) for _ in sizes]
        ft.FwdImageInvFFTManySized(ins, sizes, [specs[w] for w in which], graph_outs)
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            ft.FwdImageInvFFTManySized(ins, sizes, [specs[w] for w in which], graph_outs)
        for o in graph_outs:
            o.zero_()
        g.replay()
        torch.cuda.synchronize()
        del g
        for a, b in zip(outs, graph_outs):
            assert torch.equal(a, b)
        results.append(([host(o) for o in outs], host(peaks)))
    for a, b in zip(results[0][0], results[1][0]):
        assert np.array_equal(a, b)
    assert np.array_equal(results[0][1], results[1][1])


def test_templates_per_block_setting(torch_cuda):
    """Every templates-per-block choice of the fused column pass gives bit-identical windows
    (only the grouping of templates into blocks changes), at 1536 and at 640 points (a plan whose
    columns are 640 long, reduced along x only)."""
    torch = torch_cuda
    for fin, fout, iout in (((384, 384, 1), (2048, 2048, 1), (1024, 1024, 1)),
                            ((16, 128, 1), (64, 640, 1), (16, 512, 1))):
        spec = dev(torch, image_spectrum(fout, 27).view(np.float32))
        rng = np.random.default_rng(28)
        ins = [dev(torch, O.real_to_padded(rng.standard_normal((fin[1], fin[0])).astype(np.float32), fin))
               for _ in range(11)]
        ref = None
        for tpb in (0, 1, 2, 5, 16):
            ft = plan(fin, fout, iout)
            ft.SetTemplatesPerLaunch(11)
            ft.SetTemplatesPerBlock(tpb)
            if tpb:
                assert ft.TemplatesPerBlock() == min(tpb, 11)
            outs = [empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32) for _ in ins]
            ft.FwdImageInvFFTMany(ins, spec, outs)
            got = [host(o) for o in outs]
            if ref is None:
                ref = got
            else:
                for a, b in zip(ref, got):
                    assert np.array_equal(a, b), tpb
