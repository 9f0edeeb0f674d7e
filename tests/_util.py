"""Shared helpers for the parity tests (device buffers via torch, oracle comparisons)."""
from __future__ import annotations

import numpy as np

from oracle import fastfft_oracle as O

RTOL_L2_FP32 = 1e-5       # relative L2 error bound of the FP32 path against the FP64 oracle
RTOL_MAX_FP32 = 5e-5      # max |err| / max |ref|


def dev(torch, a: np.ndarray, n_elems: int | None = None, dtype=None):
    """Copy a numpy array to a zero-initialised CUDA tensor of at least n_elems elements."""
    a = np.ascontiguousarray(a)
    t = torch.from_numpy(a.reshape(-1).copy())
    if dtype is not None:
        t = t.to(dtype)
    if n_elems is not None and n_elems > t.numel():
        z = torch.zeros(n_elems, dtype=t.dtype)
        z[: t.numel()] = t
        t = z
    return t.cuda()


def empty(torch, n: int, dtype):
    return torch.zeros(n, dtype=dtype, device="cuda")


def host(t) -> np.ndarray:
    return t.detach().cpu().numpy()


def spectrum_view(t, plan_dims_out) -> np.ndarray:
    """Complex64 spectrum [kz][kx][ky] from a float32 device buffer."""
    x, y, z = plan_dims_out
    w, _ = O.padded_x(x)
    a = host(t)[: 2 * w * y * z].view(np.complex64)
    return a.reshape(z, w, y)


def random_real(shape, seed):
    return np.random.default_rng(seed).standard_normal(shape).astype(np.float32)
