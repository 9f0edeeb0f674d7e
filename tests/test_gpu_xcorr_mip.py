"""Fused maximum projection across templates (fastfft_fwd_image_inv_many_mip).

Every retained pixel of the projection keeps the best score over the templates and the
first template that reached it.  The oracle is the per-template FP64 window of the
reference's correlation, reduced per pixel with argmax (first index on ties).
"""
import numpy as np
import pytest

import fastfft_b200 as F
from oracle import fastfft_oracle as O
from tests._util import dev, empty, host

pytestmark = pytest.mark.gpu


def plan(fin, fout, iout):
    ft = F.FourierTransformer()
    ft.SetForwardFFTPlan(*fin, *fout)
    ft.SetInverseFFTPlan(*fout, *iout)
    return ft


def templates(sizes, seed):
    rng = np.random.default_rng(seed)
    return [rng.standard_normal((y, x)).astype(np.float32) for x, y in sizes]


def oracle_projection(ts, sizes, spec, fout, iout):
    """(best value, best template, top-2 margin) per pixel of the FP64 windows."""
    wins = []
    for t, (x, y) in zip(ts, sizes):
        p = O.Plan((x, y, 1), fout, fout, iout)
        wins.append(O.real_from_padded(O.fwd_image_inv(O.real_to_padded(t, (x, y, 1)), spec, p,
                                                       out_dtype=np.float64), iout)[0])
    w = np.stack(wins)                       # [template][y][x]
    best = np.argmax(w, axis=0)              # first template on ties
    top = np.take_along_axis(w, best[None], 0)[0]
    srt = np.sort(w, axis=0)
    margin = srt[-1] - srt[-2] if len(ts) > 1 else np.full(top.shape, np.inf)
    return top, best, margin, w


def check_projection(mip, ts, sizes, spec, fout, iout):
    vals, idx = F.decode_peaks(mip)
    wx, wy = iout[0], iout[1]
    vals = vals.reshape(wy, wx)
    idx = idx.reshape(wy, wx)
    top, best, margin, _ = oracle_projection(ts, sizes, spec, fout, iout)
    scale = np.abs(top).max()
    assert np.abs(vals - top).max() <= 5e-5 * scale
    sure = margin > 1e-3 * scale               # pixels whose best template is not a near tie
    assert sure.mean() > 0.5
    assert np.array_equal(idx[sure], best[sure])
    return vals, idx


CASES = [
    ((200, 150, 1), (1024, 1024, 1), (500, 600, 1), (768, 768)),   # 3 * 256 on both axes
    ((64, 64, 1), (1024, 1024, 1), (400, 440, 1), (512, 512)),     # 463, 503 -> powers of two
]


@pytest.mark.parametrize("fmax,fout,iout,msize", CASES)
def test_projection_matches_oracle(torch_cuda, fmax, fout, iout, msize):
    torch = torch_cuda
    ft = plan(fmax, fout, iout)
    assert ft.CorrelationSize() == msize
    spec = O.image_spectrum_fp32(O.gaussian_blob_image(1024, n_blobs=6, seed=11))
    d_spec = dev(torch, spec.view(np.float32))
    sizes = [(fmax[0], fmax[1]), (fmax[0] // 2, fmax[1]), (33, 17), (fmax[0], fmax[1] // 3), (fmax[0], fmax[1]),
             (8, 8), (fmax[0] - 1, fmax[1] - 1)]
    ts = templates(sizes, 12)
    ins = [dev(torch, O.real_to_padded(t, (x, y, 1))) for t, (x, y) in zip(ts, sizes)]
    mip = torch.zeros(iout[0] * iout[1], dtype=torch.int64, device="cuda")
    ft.FwdImageInvFFTManyMip(ins, d_spec, mip, sizes=sizes)
    check_projection(mip, ts, sizes, spec, fout, iout)


def test_projection_streams_across_calls(torch_cuda):
    """Two calls numbered with index_base give exactly the projection of one call."""
    torch = torch_cuda
    fin, fout, iout = (200, 150, 1), (1024, 1024, 1), (500, 600, 1)
    ft = plan(fin, fout, iout)
    spec = O.image_spectrum_fp32(O.gaussian_blob_image(1024, n_blobs=4, seed=13))
    d_spec = dev(torch, spec.view(np.float32))
    ts = templates([(200, 150)] * 9, 14)
    ins = [dev(torch, O.real_to_padded(t, fin)) for t in ts]
    one = torch.zeros(500 * 600, dtype=torch.int64, device="cuda")
    two = torch.zeros_like(one)
    ft.FwdImageInvFFTManyMip(ins, d_spec, one)
    ft.FwdImageInvFFTManyMip(ins[:4], d_spec, two, index_base=0)
    ft.FwdImageInvFFTManyMip(ins[4:], d_spec, two, index_base=4)
    assert torch.equal(one, two)
    check_projection(one, ts, [(200, 150)] * 9, spec, fout, iout)


def test_projection_with_windows_and_full_size_path(torch_cuda):
    """Windows written beside the projection equal FwdImageInvFFTMany's; the size-N kernels
    give the same projection within the FP32 bounds."""
    torch = torch_cuda
    fin, fout, iout = (96, 96, 1), (1024, 1024, 1), (256, 256, 1)
    spec = O.image_spectrum_fp32(O.gaussian_blob_image(1024, n_blobs=5, seed=15))
    d_spec = dev(torch, spec.view(np.float32))
    ts = templates([(96, 96)] * 5, 16)
    ins = [dev(torch, O.real_to_padded(t, fin)) for t in ts]
    a = plan(fin, fout, iout)
    wins = [empty(torch, a.ReturnInvOutputMemorySize(), torch.float32) for _ in ts]
    ref_wins = [empty(torch, a.ReturnInvOutputMemorySize(), torch.float32) for _ in ts]
    mip_a = torch.zeros(256 * 256, dtype=torch.int64, device="cuda")
    a.FwdImageInvFFTManyMip(ins, d_spec, mip_a, outputs=wins)
    a.FwdImageInvFFTMany(ins, d_spec, ref_wins)
    for w, r in zip(wins, ref_wins):
        assert torch.equal(w, r)
    b = plan(fin, fout, iout)
    b.SetFullSizeCorrelation(True)
    mip_b = torch.zeros_like(mip_a)
    b.FwdImageInvFFTManyMip(ins, d_spec, mip_b)
    check_projection(mip_a, ts, [(96, 96)] * 5, spec, fout, iout)
    check_projection(mip_b, ts, [(96, 96)] * 5, spec, fout, iout)


def test_projection_rejects_bad_arguments(torch_cuda):
    torch = torch_cuda
    ft = plan((64, 64, 1), (512, 512, 1), (64, 64, 1))
    t = torch.zeros(ft.ReturnInputMemorySize(), device="cuda")
    spec = torch.zeros(2 * 257 * 512, device="cuda")
    with pytest.raises(ValueError):
        ft.FwdImageInvFFTManyMip([t], spec, torch.zeros(10, dtype=torch.int64, device="cuda"))
    with pytest.raises(F.FastFFTError):
        ft.FwdImageInvFFTManyMip([t], spec, torch.zeros(64 * 64, dtype=torch.int64, device="cuda"), index_base=-1)
