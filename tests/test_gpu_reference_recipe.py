"""FwdImageInvFFT against the reference's own validation recipe on non-symmetric data.

The reference checks its padded correlation against cuFFT (src/tests/padded_convolution_FastFFT_vs_cuFFT.cu:317-378):
the template clipped into the top-left of a zeroed N x N buffer (ClipIntoTopLeft,
src/fastfft/FastFFT.cu:1766-1778), an in-place R2C, and an in-place C2R whose load callback
forms conj(template spectrum) x image spectrum (src/fastfft/Image.cu:315-343).  That recipe runs
here as a standalone program (fastfft_b200/csrc/comparator/cufft_recipe_bench.cu, statically
linked cuFFT) on a random template of non-power-of-two size and a random image, and the window
of its N x N output must equal ours: the single call (size-N kernels) and the batched call
(reduced correlation size).  This pins the conjugation direction, the spectrum layout and the
window origin against the reference's recipe rather than against the symmetric known answers.
"""
import json
import os
import subprocess
import tempfile

import numpy as np
import pytest

import fastfft_b200 as F
from oracle import fastfft_oracle as O
from tests._util import dev, empty, host

pytestmark = pytest.mark.gpu

RTOL_L2 = 1e-5


def _recipe_window(n, template, spec_kxky, w):
    from fastfft_b200.build import build_comparator

    exe = build_comparator()
    if exe is None:
        pytest.skip("no static cuFFT in this toolkit")
    L = template.shape[0]
    with tempfile.TemporaryDirectory() as d:
        np.ascontiguousarray(template, dtype=np.float32).tofile(os.path.join(d, "template.f32"))
        # the recipe's image spectrum is [ky][kx] (N rows of N/2+1); ours is [kx][ky]
        kykx = np.ascontiguousarray(spec_kxky.reshape(n // 2 + 1, n).T, dtype=np.complex64)
        kykx.tofile(os.path.join(d, "image_kykx.c64"))
        p = subprocess.run([str(exe), d, str(n), str(L), "1", "1", str(w)], capture_output=True, text=True, timeout=300)
        r = json.loads(p.stdout.strip().splitlines()[-1])
        assert "ms_per_execution" in r, p.stdout + p.stderr
        return np.fromfile(os.path.join(d, "corr.f32"), dtype=np.float32).reshape(w, n + 2)[:, :w]


@pytest.mark.parametrize("n,L,W", [(1024, 100, 300), (1536, 200, 700)])
def test_windows_equal_the_reference_cufft_recipe(torch_cuda, n, L, W):
    torch = torch_cuda
    rng = np.random.default_rng(n + L)
    img = (O.gaussian_blob_image(n, n_blobs=10, seed=n) + 0.3 * rng.standard_normal((n, n))).astype(np.float32)
    spec = O.image_spectrum_fp32(img)                                     # [kx][ky] complex64
    t = (rng.standard_normal((L, L)) + np.linspace(0, 1, L)[None, :]).astype(np.float32)   # no symmetry
    ref = _recipe_window(n, t, spec, W)

    fin, fout, iout = (L, L, 1), (n, n, 1), (W, W, 1)
    d_spec = dev(torch, spec.view(np.float32))
    d_t = dev(torch, O.real_to_padded(t, fin))
    for batched in (False, True):
        ft = F.FourierTransformer()
        ft.SetForwardFFTPlan(*fin, *fout)
        ft.SetInverseFFTPlan(*fout, *iout)
        out = empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32)
        if batched:
            ft.FwdImageInvFFTMany([d_t], d_spec, [out])
        else:
            ft.FwdImageInvFFT(d_t, d_spec, out)
        torch.cuda.synchronize()
        got = O.real_from_padded(host(out), iout)[0]
        assert O.rel_l2(got, ref) <= RTOL_L2, (batched, ft.CorrelationSize())
        assert np.unravel_index(np.argmax(got), got.shape) == np.unravel_index(np.argmax(ref), ref.shape)
