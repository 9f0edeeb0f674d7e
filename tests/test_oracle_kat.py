"""The host oracle against the reference's known-answer tests and an independent DFT.

Pins oracle/fastfft_oracle.py before it is used as the checker:
  - unit impulse (src/tests/unit_impulse_test.cu:89-179)
  - constant image (src/tests/constant_image_test.cu:78-191)
  - padded convolution impulse control (src/tests/padded_convolution_FastFFT_vs_cuFFT.cu:169-265)
  - functor scaling (src/tests/preop_functor_scale_test.cu:200-364)
  - FFTW-free smoke test (src/tests/non_cuda_compilation_unit.cu:16-84)
  - golden vectors from a matrix DFT (tests/golden/make_golden.py)
"""
import os

import numpy as np
import pytest

from oracle import fastfft_oracle as O

SIZES = [32, 64, 128, 256, 512]          # reference test_size (tests.h:11), trimmed for the CPU suite
HERE = os.path.dirname(os.path.abspath(__file__))


def impulse(n, val=1.0):
    a = np.zeros((n, n))
    a[0, 0] = val
    return a


@pytest.mark.parametrize("n_in,n_out", [(a, b) for a in SIZES for b in SIZES if b >= a])
def test_unit_impulse_increase(n_in, n_out):
    plan = O.Plan((n_in, n_in, 1), (n_out, n_out, 1), (n_out, n_out, 1), (n_out, n_out, 1))
    x = O.real_to_padded(impulse(n_in), plan.fwd_in)
    s = O.fwd(x, plan.fwd_in, plan.fwd_out)
    # forward: every coefficient is exactly 1 -> sum |X| = number of complex elements
    assert np.sum(np.abs(s)) == pytest.approx(s.size, abs=1e-8)
    r = O.real_from_padded(O.inv(s, plan.inv_in, plan.inv_out), plan.inv_out)
    # round trip: sum of real output = Nx*Ny exactly (unit_impulse_test.cu:175-179)
    assert r.sum() == n_out * n_out
    assert r[0, 0, 0] == n_out * n_out


@pytest.mark.parametrize("n", SIZES)
def test_constant_image(n):
    plan = O.Plan((n, n, 1), (n, n, 1), (n, n, 1), (n, n, 1))
    x = O.real_to_padded(np.ones((n, n)), plan.fwd_in)
    s = O.fwd(x, plan.fwd_in, plan.fwd_out)
    assert s[0, 0, 0] == pytest.approx(n * n)
    rest = np.abs(s).ravel()[1:]
    assert rest.max() < 1e-9 * n * n
    r = O.real_from_padded(O.inv(s, plan.inv_in, plan.inv_out), plan.inv_out)
    # round trip sum N^4 (constant_image_test.cu:186-191)
    assert r.sum() == pytest.approx(float(n) ** 4, rel=1e-12)


@pytest.mark.parametrize("n_in,n_out", [(32, 32), (32, 128), (64, 256), (128, 512)])
def test_padded_convolution_impulse(n_in, n_out):
    # template impulse 2.0 padded to n_out; image impulse 3.0 transformed at n_out
    plan = O.Plan((n_in, n_in, 1), (n_out, n_out, 1), (n_out, n_out, 1), (n_out, n_out, 1))
    t = O.real_to_padded(impulse(n_in, 2.0), plan.fwd_in)
    img = O.fwd(O.real_to_padded(impulse(n_out, 3.0), plan.fwd_out), plan.fwd_out, plan.fwd_out)
    out = O.real_from_padded(O.fwd_image_inv(t, img, plan), plan.inv_out)
    assert out[0, 0, 0] == n_out * n_out * 2.0 * 3.0
    out[0, 0, 0] = 0
    assert np.all(out == 0)


@pytest.mark.parametrize("n", [64, 256])
def test_functor_scaling(n):
    plan = O.Plan((n, n, 1), (n, n, 1), (n, n, 1), (n, n, 1))
    sf = float(n * n * 2 * 3)
    t = O.real_to_padded(impulse(n, 2.0), plan.fwd_in)
    img = O.fwd(O.real_to_padded(impulse(n, 3.0), plan.fwd_in), plan.fwd_in, plan.fwd_out)
    noop = O.real_from_padded(O.fwd_image_inv(t, img, plan), plan.inv_out)
    assert noop[0, 0, 0] == sf
    pre = O.real_from_padded(O.fwd_image_inv(t, img, plan, pre_op=(O.OP_SCALE, 1.0 / sf)), plan.inv_out)
    assert pre[0, 0, 0] == pytest.approx(1.0, rel=1e-12)
    intra = O.real_from_padded(
        O.fwd_image_inv(t, img, plan, intra_op=(O.OP_CONJ_MUL_THEN_SCALE, 1.0 / sf)), plan.inv_out)
    assert intra[0, 0, 0] == pytest.approx(1.0, rel=1e-12)


def test_smoke_64_round_trip():
    plan = O.Plan((64, 64, 1), (64, 64, 1), (64, 64, 1), (64, 64, 1))
    x = O.real_to_padded(impulse(64), plan.fwd_in)
    r = O.real_from_padded(O.inv(O.fwd(x, plan.fwd_in, plan.fwd_out), plan.inv_in, plan.inv_out), plan.inv_out)
    assert r[0, 0, 0] == 4096.0


def _matrix_dft(n, sign):
    k = np.arange(n)
    return np.exp(sign * 2j * np.pi * np.outer(k, k) / n)


def test_oracle_against_matrix_dft_nonsymmetric():
    # non-symmetric input, non-power-of-2 L: pins layout [kx][ky] and the sign convention
    rng = np.random.default_rng(7)
    L, N = 24, 64
    a = rng.standard_normal((L, L)).astype(np.float32).astype(np.float64)
    full = np.zeros((N, N))
    full[:L, :L] = a
    F = _matrix_dft(N, -1)
    s_yx = F @ full @ F.T                     # [ky][kx]
    expect = s_yx[:, : N // 2 + 1].T          # [kx][ky]
    plan = O.Plan((L, L, 1), (N, N, 1), (N, N, 1), (N, N, 1))
    got = O.fwd(O.real_to_padded(a, plan.fwd_in), plan.fwd_in, plan.fwd_out)[0]
    assert O.rel_l2(got, expect) < 1e-13


def test_oracle_xcorr_definition():
    # c[r] = N * sum_x T(x) I(x + r) mod N
    rng = np.random.default_rng(11)
    L, N, W = 5, 16, 7
    t = rng.standard_normal((L, L))
    img = rng.standard_normal((N, N))
    plan = O.Plan((L, L, 1), (N, N, 1), (N, N, 1), (W, W, 1))
    spec = O.fwd(O.real_to_padded(img, (N, N, 1)), (N, N, 1), (N, N, 1))
    got = O.real_from_padded(O.fwd_image_inv(O.real_to_padded(t, plan.fwd_in), spec, plan), plan.inv_out)[0]
    want = np.zeros((W, W))
    for ry in range(W):
        for rx in range(W):
            acc = 0.0
            for y in range(L):
                for x in range(L):
                    acc += t[y, x] * img[(y + ry) % N, (x + rx) % N]
            want[ry, rx] = N * N * acc
    assert np.allclose(got, want, rtol=1e-6, atol=1e-6 * np.abs(want).max())


@pytest.mark.parametrize("name", ["fwd_32_to_128", "xcorr_48_to_128_w40"])
def test_oracle_against_golden(name):
    g = np.load(os.path.join(HERE, "golden", f"{name}.npz"))
    plan = O.Plan(tuple(g["fwd_in"]), tuple(g["fwd_out"]), tuple(g["inv_in"]), tuple(g["inv_out"]))
    if name.startswith("fwd"):
        got = O.fwd(g["input"], plan.fwd_in, plan.fwd_out)
        assert O.rel_l2(got, g["spectrum"]) < 1e-13
        back = O.inv(got, plan.inv_in, plan.inv_out, out_dtype=np.float64)
        assert O.rel_l2(back, g["round_trip"]) < 1e-13
    else:
        got = O.fwd_image_inv(g["input"], g["image_spectrum"], plan, out_dtype=np.float64)
        assert O.rel_l2(got, g["output"]) < 1e-12


def test_padded_sizes_match_reference_formula():
    # ReturnPaddedMemorySize (FastFFT.h:363-404)
    assert O.padded_x(384) == (193, 386)
    assert O.padded_x(385) == (193, 386)
    assert O.padded_memory_size((4096, 4096, 1)) == 4098 * 4096
    assert O.padded_memory_size((1024, 1024, 1)) == 1026 * 1024
    assert O.padded_memory_size((64, 64, 64)) == 66 * 64 * 64
