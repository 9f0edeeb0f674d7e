"""Generate the golden vectors in tests/golden/ with a matrix DFT (independent of numpy.fft).

Run: python tests/golden/make_golden.py
The vectors pin the spectrum layout [kx][ky], the forward sign, the unnormalised
inverse, zero padding at the origin and the origin-anchored crop, using seeded
non-symmetric inputs with non-power-of-two L and W.
"""
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def mdft(n, sign):
    k = np.arange(n)
    return np.exp(sign * 2j * np.pi * np.outer(k, k) / n)


def pad_rows(a, x):
    w = (x + (2 if x % 2 == 0 else 1)) // 2
    out = np.zeros((a.shape[0], 2 * w))
    out[:, : a.shape[1]] = a
    return out.reshape(-1)


def fwd_full(a, n):
    full = np.zeros((n, n))
    full[: a.shape[0], : a.shape[1]] = a
    F = mdft(n, -1)
    return F @ full @ F.T  # [ky][kx]


def inv_full(s_yx_half, n):
    # Hermitian-extend along kx, then unnormalised inverse DFT; keep the real part
    full = np.zeros((n, n), dtype=complex)
    h = n // 2
    full[:, : h + 1] = s_yx_half
    for kx in range(h + 1, n):
        full[:, kx] = np.conj(s_yx_half[(-np.arange(n)) % n, n - kx])
    G = mdft(n, +1)
    return (G @ full @ G.T).real


def main():
    rng = np.random.default_rng(20261203)
    # forward 32 -> 128 and round trip
    L, N = 32, 128
    a = rng.standard_normal((L, L)).astype(np.float32).astype(np.float64)
    s = fwd_full(a, N)
    spec = np.ascontiguousarray(s[:, : N // 2 + 1].T[None])  # [kz][kx][ky]
    rt = inv_full(s[:, : N // 2 + 1], N)
    np.savez_compressed(os.path.join(HERE, "fwd_32_to_128.npz"), fwd_in=(L, L, 1), fwd_out=(N, N, 1),
                        inv_in=(N, N, 1), inv_out=(N, N, 1), input=pad_rows(a, L), spectrum=spec,
                        round_trip=pad_rows(rt, N))
    # cross-correlation 48 -> 128, window 40 x 40
    L, N, W = 48, 128, 40
    t = rng.standard_normal((L, L)).astype(np.float32).astype(np.float64)
    img = rng.standard_normal((N, N))
    si = fwd_full(img, N)[:, : N // 2 + 1]       # [ky][kx]
    st = fwd_full(t, N)[:, : N // 2 + 1]
    c = inv_full(np.conj(st) * si, N)[:W, :W]
    np.savez_compressed(os.path.join(HERE, "xcorr_48_to_128_w40.npz"), fwd_in=(L, L, 1), fwd_out=(N, N, 1),
                        inv_in=(N, N, 1), inv_out=(W, W, 1), input=pad_rows(t, L),
                        image_spectrum=np.ascontiguousarray(si.T[None]).astype(np.complex128), output=pad_rows(c, W))


if __name__ == "__main__":
    main()
