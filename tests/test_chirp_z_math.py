"""The chirp-z (Bluestein) identities the chirp-z kernels rely on, checked in FP64 numpy on CPU.

The kernels evaluate a length-N DFT as X[k] = c_k sum_n (x_n c_n) conj(c_(k-n)) with
c_n = exp(-i pi n^2 / N), a circular convolution of length M >= 2N - 1 (a power of two, at
least 64) done as IFFT_M(FFT_M(a) FFT_M(b)), with the filter spectrum FFT_M(b) / M tabulated
per N as (1 + sum_(0<m<N) 2 cos(2 pi m k / M) conj(c_m)) / M, the chirp exponent reduced as
n^2 mod 2N, and the inverse taken as conj(DFT(conj X)).  This restates those tables and steps
and compares them with numpy's DFT.
"""
import numpy as np
import pytest


def blue_m(n):
    m = 64
    while m < 2 * n - 1:
        m *= 2
    return m


def chirp(n):
    e = (np.arange(n, dtype=np.int64) ** 2) % (2 * n)
    return np.exp(-1j * np.pi * e / n)


def filter_spectrum(n, m):
    """FFT_M(b) / M for b_0 = 1, b_m = b_(M-m) = conj(c_m), 0 < m < N: the direct cosine sum."""
    c = chirp(n)
    k = np.arange(m)[:, None]
    j = np.arange(1, n)[None, :]
    w = 2.0 * np.cos(2.0 * np.pi * ((j * k) % m) / m)
    return (1.0 + w @ np.conj(c[1:])) / m


def chirp_z_dft(x, inverse=False):
    n = x.shape[-1]
    m = blue_m(n)
    c = chirp(n)
    filt = filter_spectrum(n, m)
    v = np.conj(x) if inverse else x
    a = np.zeros(m, complex)
    a[:n] = v * c
    y = np.fft.ifft(np.fft.fft(a) * filt) * m      # unnormalised inverse of the M-point FFT
    out = y[:n] * c
    return np.conj(out) if inverse else out


@pytest.mark.parametrize("n", [17, 31, 100, 321, 999, 1000, 1001])
def test_filter_table_equals_fft_of_b(n):
    m = blue_m(n)
    c = chirp(n)
    b = np.zeros(m, complex)
    b[0] = 1.0
    b[1:n] = np.conj(c[1:])
    b[m - n + 1:] = np.conj(c[1:])[::-1]
    np.testing.assert_allclose(filter_spectrum(n, m), np.fft.fft(b) / m, rtol=0, atol=1e-12)


@pytest.mark.parametrize("n", [17, 33, 100, 257, 999, 1000, 4095])
def test_chirp_z_equals_dft(n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    ref = np.fft.fft(x)
    got = chirp_z_dft(x)
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-12
    inv = chirp_z_dft(ref, inverse=True)                     # unnormalised inverse
    assert np.linalg.norm(inv - n * x) / np.linalg.norm(n * x) < 1e-12


def test_chirp_exponent_reduction():
    """exp(-i pi n^2 / N) depends on n^2 only mod 2N, so the reduced exponent is exact."""
    for n in (17, 1000, 4095):
        k = np.arange(n, dtype=np.int64)
        direct = np.exp(-1j * np.pi * (k.astype(np.float64) ** 2 / n))
        np.testing.assert_allclose(chirp(n), direct, rtol=0, atol=1e-6 * max(1, n * n / 1e6))


def test_m_covers_the_linear_convolution():
    for n in range(17, 4096, 37):
        m = blue_m(n)
        assert m >= 2 * n - 1 and m & (m - 1) == 0 and m <= 8192
