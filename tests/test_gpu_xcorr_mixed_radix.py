"""Batched correlation at the mixed-radix lengths 3 * 2^k, 5 * 2^k and 7 * 2^k against the FP64 oracle.

When 3 * 2^k (2^k in [128, 2048]) reaches L + W - 1 before the next power of two, the batched
call correlates at that length (R radix-16 sub-FFTs and a radix-R pass per transform); 5 * 2^k
(2^k in [128, 1024]) and 7 * 2^k (2^k in [128, 512]) lengths run where the plan's own N is one
(along an axis without reduction, or with the other axis reduced).  These tests drive every such length along each axis through all four
kernels that have a 3 * 2^k form (row R2C, fused column pass, row C2R, and the forward
column pass of the image preparation) and compare the retained windows with the size-N
correlation that the reference defines.
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


def oracle_window(t, fin, spec, fout, iout):
    p = O.Plan(fin, fout, fout, iout)
    return O.real_from_padded(O.fwd_image_inv(O.real_to_padded(t, fin), spec, p, out_dtype=np.float64), iout)


# (template, transform, window, expected correlation size)
CASES3 = [
    ((96, 96, 1), (1024, 1024, 1), (256, 256, 1), (384, 384)),        # 351 -> 3 * 128
    ((200, 200, 1), (1024, 1024, 1), (150, 150, 1), (384, 384)),      # 349 -> 3 * 128, template longer than P
    ((200, 150, 1), (1024, 1024, 1), (500, 600, 1), (768, 768)),      # 699, 749 -> 3 * 256
    ((384, 384, 1), (2048, 2048, 1), (1024, 1024, 1), (1536, 1536)),  # 1407 -> 3 * 512
    ((1000, 16, 1), (4096, 64, 1), (2000, 16, 1), (3072, 32)),        # 2999 -> 3 * 1024 along x
    ((16, 1000, 1), (64, 4096, 1), (16, 2000, 1), (32, 3072)),        # ... along y
    ((2000, 8, 1), (8192, 32, 1), (4000, 8, 1), (6144, 16)),          # 5999 -> 3 * 2048 along x
    ((8, 2000, 1), (32, 8192, 1), (8, 4000, 1), (16, 6144)),          # ... along y
]


CASES5 = [
    ((128, 128, 1), (640, 640, 1), (512, 512, 1), (640, 640)),          # plan at 5 * 128 (639 needs all of it)
    ((300, 300, 1), (1280, 1280, 1), (900, 900, 1), (1280, 1280)),      # plan at 5 * 256
    ((300, 200, 1), (2048, 1024, 1), (500, 600, 1), (1024, 1024)),      # 799 -> 1024 on both axes
    ((1000, 16, 1), (2560, 64, 1), (1500, 16, 1), (2560, 32)),          # 5 * 512 rows, reduced along y
    ((16, 1000, 1), (64, 2560, 1), (16, 1500, 1), (32, 2560)),          # 5 * 512 fused column pass
    ((2000, 8, 1), (5120, 32, 1), (3000, 8, 1), (5120, 16)),            # 5 * 1024 rows
    ((8, 2000, 1), (32, 5120, 1), (8, 3000, 1), (16, 5120)),            # 5 * 1024 fused column pass
    ((200, 150, 1), (1024, 1024, 1), (440, 600, 1), (768, 768)),        # 639, 749 -> 3 * 256
]


CASES7 = [
    ((100, 100, 1), (896, 896, 1), (751, 751, 1), (896, 896)),          # plan at 7 * 128 (850 needs all of it)
    ((300, 300, 1), (1792, 1792, 1), (1401, 1401, 1), (1792, 1792)),    # plan at 7 * 256
    ((1000, 16, 1), (3584, 64, 1), (2301, 16, 1), (3584, 32)),          # 7 * 512 rows, reduced along y
    ((16, 1000, 1), (64, 3584, 1), (16, 2301, 1), (32, 3584)),          # 7 * 512 fused column pass
]


@pytest.mark.parametrize("fin,fout,iout,msize", CASES3 + CASES5 + CASES7)
def test_mixed_radix_sizes_match_oracle(torch_cuda, fin, fout, iout, msize):
    torch = torch_cuda
    ft = plan(fin, fout, iout)
    assert ft.CorrelationSize() == msize
    spec = image_spectrum(fout, 31)
    d_spec = dev(torch, spec.view(np.float32))
    rng = np.random.default_rng(32)
    ts = [rng.standard_normal((fin[1], fin[0])).astype(np.float32) for _ in range(3)]
    outs = [empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32) for _ in ts]
    ft.FwdImageInvFFTMany([dev(torch, O.real_to_padded(t, fin)) for t in ts], d_spec, outs)
    for t, o in zip(ts, outs):
        ref = oracle_window(t, fin, spec, fout, iout)
        got = O.real_from_padded(host(o), iout)
        assert O.rel_l2(got, ref) <= RTOL_L2_FP32
        assert O.rel_max(got, ref) <= RTOL_MAX_FP32


def test_mixed_radix_equals_power_of_two_path(torch_cuda):
    """The 1536^2 correlation agrees with the size-N (2048^2) kernels on the window."""
    torch = torch_cuda
    fin, fout, iout = (384, 384, 1), (2048, 2048, 1), (1024, 1024, 1)
    d_spec = dev(torch, image_spectrum(fout, 40).view(np.float32))
    t = dev(torch, O.real_to_padded(np.random.default_rng(41).standard_normal((384, 384)).astype(np.float32), fin))
    a = plan(fin, fout, iout)
    b = plan(fin, fout, iout)
    b.SetFullSizeCorrelation(True)
    assert a.CorrelationSize() == (1536, 1536) and b.CorrelationSize() == (2048, 2048)
    oa, ob = (empty(torch, a.ReturnInvOutputMemorySize(), torch.float32) for _ in range(2))
    a.FwdImageInvFFTMany([t], d_spec, [oa])
    b.FwdImageInvFFTMany([t], d_spec, [ob])
    ra, rb = (O.real_from_padded(host(x), iout) for x in (oa, ob))
    assert O.rel_l2(ra, rb) <= RTOL_L2_FP32


@pytest.mark.parametrize("write_windows", [False, True])
def test_mixed_radix_uneven_templates_and_peaks(torch_cuda, write_windows):
    """Uneven template sizes and the fused peak search at 768^2."""
    torch = torch_cuda
    fmax, fout, iout = (200, 150, 1), (1024, 1024, 1), (500, 600, 1)
    ft = plan(fmax, fout, iout)
    assert ft.CorrelationSize() == (768, 768)
    img = O.gaussian_blob_image(1024, n_blobs=6, seed=7)
    spec = O.image_spectrum_fp32(img)
    d_spec = dev(torch, spec.view(np.float32))
    rng = np.random.default_rng(33)
    sizes = [(200, 150), (64, 64), (17, 150), (200, 3), (99, 101), (128, 128), (1, 1), (150, 149), (33, 77)]
    ts = [rng.standard_normal((y, x)).astype(np.float32) for x, y in sizes]
    ins = [dev(torch, O.real_to_padded(t, (x, y, 1))) for t, (x, y) in zip(ts, sizes)]
    outs = [empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32) for _ in ts] if write_windows else None
    peaks = torch.zeros(len(ts), dtype=torch.int64, device="cuda")
    ft.FwdImageInvFFTManyPeaks(ins, d_spec, peaks, sizes=sizes, outputs=outs)
    vals, idx = F.decode_peaks(peaks)
    for i, (t, (x, y)) in enumerate(zip(ts, sizes)):
        ref = oracle_window(t, (x, y, 1), spec, fout, iout)[0]
        ri, rtop, margin = O.peak(ref)
        if margin > 1e-4 * abs(rtop):
            assert idx[i] == ri, i
        assert abs(vals[i] - rtop) <= 1e-5 * abs(rtop), i
        if write_windows:
            got = O.real_from_padded(host(outs[i]), iout)[0]
            assert O.rel_l2(got, ref) <= RTOL_L2_FP32, (x, y)
            assert O.peak(got)[0] == idx[i]


@pytest.mark.parametrize("in_dt,img_dt", [("float16", "complex32"), ("bfloat16", "complex_bf16")])
def test_mixed_radix_low_precision_storage(torch_cuda, in_dt, img_dt):
    torch = torch_cuda
    fin, fout, iout = (96, 96, 1), (1024, 1024, 1), (256, 256, 1)
    tdt = torch.float16 if in_dt == "float16" else torch.bfloat16
    rng = np.random.default_rng(34)
    t_q = torch.from_numpy(rng.standard_normal((96, 96)).astype(np.float32)).to(tdt)
    t_deq = t_q.float().numpy()
    spec = image_spectrum(fout, 35) / 1024
    spec_q = torch.from_numpy(spec.view(np.float32).reshape(-1)).to(tdt)
    spec_deq = spec_q.float().numpy().view(np.complex64).reshape(spec.shape)
    ft = plan(fin, fout, iout, input_dtype=in_dt, image_dtype=img_dt)
    ft.SetOutputDtype("float32")      # the output type otherwise follows the input type
    assert ft.CorrelationSize() == (384, 384)
    tin = torch.zeros(ft.ReturnInputMemorySize(), dtype=tdt)
    tin.view(96, -1)[:, :96] = t_q
    out = empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32)
    ft.FwdImageInvFFTMany([tin.cuda()], spec_q.cuda(), [out])
    ref = oracle_window(t_deq, fin, spec_deq, fout, iout)
    assert O.rel_l2(O.real_from_padded(host(out), iout), ref) <= 2e-5


@pytest.mark.parametrize("out_dt", ["float16", "bfloat16"])
def test_mixed_radix_low_precision_output(torch_cuda, out_dt):
    torch = torch_cuda
    fin, fout, iout = (200, 150, 1), (1024, 1024, 1), (500, 600, 1)
    odt = torch.float16 if out_dt == "float16" else torch.bfloat16
    spec = image_spectrum(fout, 36) / (1024 * 1024)
    ft = plan(fin, fout, iout)
    ft.SetOutputDtype(out_dt)
    t = np.random.default_rng(37).standard_normal((150, 200)).astype(np.float32)
    out = empty(torch, ft.ReturnInvOutputMemorySize(), odt)
    ft.FwdImageInvFFTMany([dev(torch, O.real_to_padded(t, fin))], dev(torch, spec.view(np.float32)), [out])
    got = O.real_from_padded(out.float().cpu().numpy(), iout)
    ref = oracle_window(t, fin, spec, fout, iout)
    tol = 1e-3 if out_dt == "float16" else 8e-3     # one rounding to 11 / 8 significant bits
    assert O.rel_l2(got, ref) <= tol


@pytest.mark.parametrize("per_launch", [1, 5, 16])
def test_mixed_radix_templates_per_launch(torch_cuda, per_launch):
    torch = torch_cuda
    fin, fout, iout = (384, 384, 1), (2048, 2048, 1), (1024, 1024, 1)
    ft = plan(fin, fout, iout)
    ft.SetTemplatesPerLaunch(per_launch)
    spec = image_spectrum(fout, 38)
    d_spec = dev(torch, spec.view(np.float32))
    rng = np.random.default_rng(39)
    ts = [rng.standard_normal((384, 384)).astype(np.float32) for _ in range(7)]
    outs = [empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32) for _ in ts]
    ft.FwdImageInvFFTMany([dev(torch, O.real_to_padded(t, fin)) for t in ts], d_spec, outs)
    for i in (0, 3, 6):
        ref = oracle_window(ts[i], fin, spec, fout, iout)
        assert O.rel_l2(O.real_from_padded(host(outs[i]), iout), ref) <= RTOL_L2_FP32


def test_fused_pass_just_under_48k_shared_memory(torch_cuda):
    """256^2 templates at 768^2, 8 per launch: the fused pass's dynamic shared memory is
    49,040 B, under 48 KB by itself but over it with the kernel's static shared memory, so
    the launcher has to raise the attribute."""
    torch = torch_cuda
    fin, fout, iout = (256, 256, 1), (1024, 1024, 1), (512, 512, 1)
    ft = plan(fin, fout, iout)
    ft.SetTemplatesPerLaunch(8)
    assert ft.CorrelationSize() == (768, 768)
    spec = image_spectrum(fout, 42)
    d_spec = dev(torch, spec.view(np.float32))
    rng = np.random.default_rng(43)
    ts = [rng.standard_normal((256, 256)).astype(np.float32) for _ in range(8)]
    outs = [empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32) for _ in ts]
    ft.FwdImageInvFFTMany([dev(torch, O.real_to_padded(t, fin)) for t in ts], d_spec, outs)
    for i in (0, 7):
        ref = oracle_window(ts[i], fin, spec, fout, iout)
        assert O.rel_l2(O.real_from_padded(host(outs[i]), iout), ref) <= RTOL_L2_FP32
