"""Parity at the full shapes of the two benchmarked workload families.

* Uneven batch: a 4096^2 image (N(0,1) noise + 20 Gaussian blobs), templates of
  128^2, 192^2, 256^2 and 384^2 (five per size, N(0,1), seeded) zero-padded to 4096^2,
  512^2 windows, all in one FwdImageInvFFTManySized call; FP32 storage (relative L2
  <= 1e-5 against FP64) and BF16 storage (<= 1e-4 against FP64 of the stored inputs).
* Low-precision correlation with the tensor-core DFT: a 384^2 template and the 4096^2
  image spectrum stored in FP16 or BF16 (spectrum scaled by 1/4096), the fused column
  pass's radix-16 stages on the tensor cores in split precision, 1024^2 window; relative
  L2 <= 1e-4 against FP64 of the stored inputs, and the peak where the FP32 path puts it.

Every window's peak index must equal the FP64 oracle's (or, where the oracle's top two
values lie closer together than the measured error, point at a value within that error of
the top).  The oracle is the size-4096 formulation of the reference's FwdImageInvFFT
(conj(T) x I, inverse cropped at the origin).
"""
import numpy as np
import pytest

import fastfft_b200 as F
from oracle import fastfft_oracle as O
from tests._util import RTOL_L2_FP32, RTOL_MAX_FP32, dev, empty, host

pytestmark = pytest.mark.gpu

N = 4096
RTOL_L2_LOW = 1e-4          # BF16/FP16 storage and the split-precision tensor-core form
UNEVEN_EDGES = (128, 192, 256, 384)
PER_EDGE = 5
WORKERS = O.cpu_workers()


@pytest.fixture(scope="module")
def image():
    img = O.gaussian_blob_image(N)
    spec = O.image_spectrum_fp32(img)            # [kx][ky], complex64
    return img, spec


def check_peak(got, ref):
    gi = O.peak(got)[0]
    ri, rtop, margin = O.peak(ref)
    err = float(np.max(np.abs(got - ref)))
    if margin > 4 * err:
        assert gi == ri
    else:  # a near tie in the oracle itself: the chosen lag must be one of the tied values
        assert ref.ravel()[gi] >= rtop - 2 * err


def oracle_window(t_pad, fin, spec, iout):
    p = O.Plan(fin, (N, N, 1), (N, N, 1), iout)
    return O.real_from_padded(O.fwd_image_inv(t_pad, spec, p, out_dtype=np.float64, workers=WORKERS), iout)[0]


@pytest.mark.parametrize("storage", ["float32", "bfloat16"])
def test_uneven_batch_full_shape(torch_cuda, image, storage):
    torch = torch_cuda
    _, spec = image
    W = 512
    L = max(UNEVEN_EDGES)
    rng = np.random.default_rng(O.SEED_BASE + 5)
    edges = [e for e in UNEVEN_EDGES for _ in range(PER_EDGE)]
    rng.shuffle(edges)
    tdt = torch.float32 if storage == "float32" else torch.bfloat16
    if storage == "float32":
        ft = F.FourierTransformer()
        spec_dev = dev(torch, spec.view(np.float32))
        spec_used = spec
    else:
        ft = F.FourierTransformer(input_dtype="bfloat16", image_dtype="complex_bf16")
        spec_q = torch.from_numpy((spec / N).view(np.float32).reshape(-1).copy()).to(torch.bfloat16)
        spec_dev = spec_q.cuda()
        spec_used = spec_q.float().numpy().view(np.complex64).reshape(spec.shape)
    ft.SetForwardFFTPlan(L, L, 1, N, N, 1)
    ft.SetInverseFFTPlan(N, N, 1, W, W, 1)
    ft.SetOutputDtype("float32")
    ts, ins, sizes = [], [], []
    for e in edges:
        t = rng.standard_normal((e, e)).astype(np.float32)
        t_dev = dev(torch, O.real_to_padded(t, (e, e, 1)), dtype=tdt)
        ts.append(t_dev.float().cpu().numpy())                  # the stored values, dequantized
        ins.append(t_dev)
        sizes.append((e, e))
    outs = [empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32) for _ in edges]
    ft.FwdImageInvFFTManySized(ins, sizes, spec_dev, outs)
    torch.cuda.synchronize()
    bound = RTOL_L2_FP32 if storage == "float32" else RTOL_L2_LOW
    for e, t_pad, o in zip(edges, ts, outs):
        ref = oracle_window(t_pad, (e, e, 1), spec_used, (W, W, 1))
        got = O.real_from_padded(host(o), (W, W, 1))[0]
        assert O.rel_l2(got, ref) <= bound, e
        if storage == "float32":
            assert O.rel_max(got, ref) <= RTOL_MAX_FP32, e
        check_peak(got, ref)


@pytest.mark.parametrize("storage", ["float16", "bfloat16"])
def test_low_precision_tensor_core_full_shape(torch_cuda, image, storage):
    torch = torch_cuda
    _, spec = image
    L, W = 384, 1024
    fin, iout = (L, L, 1), (W, W, 1)
    tdt = torch.float16 if storage == "float16" else torch.bfloat16
    img_dt = "complex32" if storage == "float16" else "complex_bf16"
    t = O.normal_template(L, O.SEED_BASE + 4).astype(np.float32)
    t_pad = O.real_to_padded(t, fin)

    fp = F.FourierTransformer()
    fp.SetForwardFFTPlan(*fin, N, N, 1)
    fp.SetInverseFFTPlan(N, N, 1, *iout)
    out_fp = empty(torch, fp.ReturnInvOutputMemorySize(), torch.float32)
    fp.FwdImageInvFFTMany([dev(torch, t_pad)], dev(torch, spec.view(np.float32)), [out_fp])

    ft = F.FourierTransformer(input_dtype=storage, image_dtype=img_dt)
    ft.SetForwardFFTPlan(*fin, N, N, 1)
    ft.SetInverseFFTPlan(N, N, 1, *iout)
    ft.SetOutputDtype("float32")
    ft.SetTensorCoreDFT(True)
    assert ft.TensorCoreDFTActive()
    spec_q = torch.from_numpy((spec / N).view(np.float32).reshape(-1).copy()).to(tdt)
    t_q = dev(torch, t_pad, dtype=tdt)
    out = empty(torch, ft.ReturnInvOutputMemorySize(), torch.float32)
    ft.FwdImageInvFFTMany([t_q], spec_q.cuda(), [out])
    torch.cuda.synchronize()

    spec_deq = spec_q.float().numpy().view(np.complex64).reshape(spec.shape)
    ref = oracle_window(t_q.float().cpu().numpy(), fin, spec_deq, iout)
    got = O.real_from_padded(host(out), iout)[0]
    assert O.rel_l2(got, ref) <= RTOL_L2_LOW
    check_peak(got, ref)
    got_fp = O.real_from_padded(host(out_fp), iout)[0]
    assert O.peak(got)[0] == O.peak(got_fp)[0]
