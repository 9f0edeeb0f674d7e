"""FwdFFT writing a normalised, quantised spectrum (fastfft_set_spectrum_output): FP16 or BF16
storage of scale x the spectrum, rounded once in the last pass, against the FP64 oracle; and
that spectrum as the image of the batched correlation with the matching image_dtype.
"""
import numpy as np
import pytest

import fastfft_b200 as F
from oracle import fastfft_oracle as O
from tests._util import RTOL_L2_FP32, RTOL_MAX_FP32, dev, empty, host, random_real

pytestmark = pytest.mark.gpu

# relative L2 of one rounding to the storage format (unit roundoff 2^-11 and 2^-8)
RTOL_STORE = {"complex32": 1e-3, "complex_bf16": 8e-3}


def stored(torch, t, dtype, n_complex):
    tdt = torch.float16 if dtype == "complex32" else torch.bfloat16
    return t.view(tdt)[: 2 * n_complex].float().cpu().numpy().view(np.complex64)


@pytest.mark.parametrize("dtype", ["complex32", "complex_bf16"])
@pytest.mark.parametrize("fin,fout", [((64, 64, 1), (512, 512, 1)), ((200, 100, 1), (1536, 1536, 1)),
                                      ((32, 32, 32), (64, 64, 64))])
def test_quantised_spectrum_matches_oracle(torch_cuda, dtype, fin, fout):
    torch = torch_cuda
    scale = 1.0 / fout[0]
    shape = (fin[2], fin[1], fin[0]) if fin[2] > 1 else (fin[1], fin[0])
    x = random_real(shape, seed=fin[0] + fout[0] + len(dtype))
    ft = F.FourierTransformer(rank=3 if fin[2] > 1 else 2)
    ft.SetForwardFFTPlan(*fin, *fout)
    ft.SetInverseFFTPlan(*fout, *fout)
    ft.SetSpectrumOutput(dtype, scale)
    xin = dev(torch, O.real_to_padded(x, fin), ft.ReturnInputMemorySize())
    out = empty(torch, ft.ReturnFwdOutputMemorySize(), torch.float32)
    ft.FwdFFT(xin, out)
    torch.cuda.synchronize()
    w, _ = O.padded_x(fout[0])
    got = stored(torch, out, dtype, w * fout[1] * fout[2]).reshape(fout[2], w, fout[1])
    ref = O.fwd(O.real_to_padded(x, fin), fin, fout) * scale
    assert O.rel_l2(got, ref) <= RTOL_STORE[dtype]


@pytest.mark.parametrize("dtype", ["complex32", "complex_bf16"])
def test_quantised_image_spectrum_drives_the_correlation(torch_cuda, dtype):
    torch = torch_cuda
    fin, fout, iout = (96, 96, 1), (1024, 1024, 1), (256, 256, 1)       # correlates at 384^2
    img = O.gaussian_blob_image(1024, n_blobs=6, seed=61)
    prep = F.FourierTransformer()
    prep.SetForwardFFTPlan(*fout, *fout)
    prep.SetInverseFFTPlan(*fout, *fout)
    prep.SetSpectrumOutput(dtype, 1.0 / 1024)
    d_img = dev(torch, O.real_to_padded(img.astype(np.float32), fout), prep.ReturnInputMemorySize())
    spec = empty(torch, prep.ReturnFwdOutputMemorySize(), torch.float32)
    prep.FwdFFT(d_img, spec)
    torch.cuda.synchronize()
    w, _ = O.padded_x(fout[0])
    spec_deq = stored(torch, spec, dtype, w * fout[1]).reshape(1, w, fout[1])
    ft = F.FourierTransformer(image_dtype=dtype)
    ft.SetForwardFFTPlan(*fin, *fout)
    ft.SetInverseFFTPlan(*fout, *iout)
    rng = np.random.default_rng(62)
    ts = [rng.standard_normal((96, 96)).astype(np.float32) for _ in range(3)]
    outs = [empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32) for _ in ts]
    ft.FwdImageInvFFTMany([dev(torch, O.real_to_padded(t, fin)) for t in ts], spec, outs)
    torch.cuda.synchronize()
    p = O.Plan(fin, fout, fout, iout)
    for t, o in zip(ts, outs):
        ref = O.real_from_padded(O.fwd_image_inv(O.real_to_padded(t, fin), spec_deq, p, out_dtype=np.float64), iout)
        got = O.real_from_padded(host(o), iout)
        assert O.rel_l2(got, ref) <= RTOL_L2_FP32
        assert O.rel_max(got, ref) <= RTOL_MAX_FP32
