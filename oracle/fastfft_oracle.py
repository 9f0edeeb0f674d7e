"""Host oracle for FastFFT's size-changing FFT / padded cross-correlation path.

TEST INFRASTRUCTURE ONLY.  Nothing in the product (``fastfft_b200``) imports this
module; only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg use it, and only as the checker (or as the timed CPU baseline), never as the
thing being measured on the GPU.

It restates, in numpy (FP64 by default), the semantics of the reference's
``FourierTransformer`` path:

* buffer sizes and the FFTW pitch ``2*(x/2+1)``        -- include/FastFFT.h:363-404
* size-change classification and validation            -- src/fastfft/FastFFT.cu:803-930 (ValidateDimensions)
* forward sign -1, unnormalised transforms             -- src/fastfft/FastFFT.cu:3117-3124
* zero padding at the origin (forward increase)        -- include/FastFFT.cuh:881-915 (io::load), :428-448
* 2D spectrum layout [kx][ky], ky contiguous           -- FastFFT.cu:3216-3218, kernel indexing :46,
                                                          store_r2c_transposed_xy FastFFT.cuh:769-811
* 3D spectrum layout [kz][kx][ky]                      -- Return1DFFTAddress_YZ_transpose_strided_Z
                                                          memory_addressing.h:86-96 + C2C pass :1433-1475
* C2R reads the transposed layout, writes pitched rows -- FastFFT.cuh:831-848, :1135-1148
* decrease keeps the first outputs per axis            -- store_r2c_reduced FastFFT.cuh:547-565,
                                                          C2C_FWD_NONE_INV_DECREASE store :1340-1342
* functors NOOP / SCALE / CONJ_MUL / CONJ_MUL_THEN_SCALE -- include/detail/functors.h:15-80
  (CONJ_MUL: (tx*Ix + ty*Iy, tx*Iy - ty*Ix) = conj(T) * I, functors.h:30-40)

Parity of this restatement is pinned by the reference's own known-answer tests
(src/tests/unit_impulse_test.cu, constant_image_test.cu,
padded_convolution_FastFFT_vs_cuFFT.cu, preop_functor_scale_test.cu,
non_cuda_compilation_unit.cu), which tests/test_oracle_kat.py replays, and by an
independent naive-DFT check at small sizes.  The reference's cuFFTDx arithmetic
cannot be run or linked here, so non-symmetric layouts are pinned by the cited
addressing code plus the FP64 DFT definition.
"""
from __future__ import annotations

import os
from dataclasses import dataclass

import numpy as np

# Functor kinds, mirroring KernelFunction::IKF_t (include/detail/functors.h:15-80).
OP_NOOP = 0
OP_SCALE = 1
OP_CONJ_MUL = 2
OP_CONJ_MUL_THEN_SCALE = 3

SIZE_INCREASE = "increase"
SIZE_DECREASE = "decrease"
SIZE_NO_CHANGE = "no_change"


def is_power_of_two(v: int) -> bool:
    return v >= 1 and (v & (v - 1)) == 0


def padded_x(x: int) -> tuple[int, int]:
    """(w, pitch) for a real row of logical length x.

    Restates ReturnPaddedMemorySize (include/FastFFT.h:363-404): w is the number of
    complex elements after an R2C along x, and the real pitch is 2*w elements.
    """
    jump = 2 if x % 2 == 0 else 1
    w = (x + jump) // 2
    return w, 2 * w


def padded_memory_size(dims: tuple[int, int, int], real_input: bool = True) -> int:
    """Number of InputType elements the reference reserves for dims (x, y, z)."""
    x, y, z = dims
    if real_input:
        w, _ = padded_x(x)
        return 2 * w * y * z
    return 2 * x * y * z


def classify(din: tuple[int, int, int], dout: tuple[int, int, int]) -> str:
    """Size-change type of one direction (FastFFT.cu:803-850)."""
    if any(o > i for i, o in zip(din, dout)):
        if not all(o >= i for i, o in zip(din, dout)):
            raise ValueError("if padding, all dimensions must be >=")
        return SIZE_INCREASE
    if any(o < i for i, o in zip(din, dout)):
        return SIZE_DECREASE
    return SIZE_NO_CHANGE


@dataclass
class Plan:
    """Forward + inverse plan; dims are (x, y, z) as passed to Set{Forward,Inverse}FFTPlan."""

    fwd_in: tuple[int, int, int]
    fwd_out: tuple[int, int, int]
    inv_in: tuple[int, int, int]
    inv_out: tuple[int, int, int]

    def __post_init__(self):
        if tuple(self.fwd_out) != tuple(self.inv_in):
            raise ValueError("fwd out must match inv in")
        self.fwd_change = classify(self.fwd_in, self.fwd_out)
        self.inv_change = classify(self.inv_in, self.inv_out)
        self.rank = 3 if (self.fwd_in[2] > 1 or self.fwd_out[2] > 1) else 2

    @property
    def n(self) -> tuple[int, int, int]:
        """Transform size per axis (x, y, z): the larger of forward in/out."""
        return tuple(max(a, b) for a, b in zip(self.fwd_in, self.fwd_out))

    def input_memory_size(self) -> int:
        return padded_memory_size(self.fwd_in)

    def fwd_output_memory_size(self) -> int:
        return padded_memory_size(self.fwd_out)

    def inv_output_memory_size(self) -> int:
        return padded_memory_size(self.inv_out)


# ---------------------------------------------------------------------------
# Layout helpers
# ---------------------------------------------------------------------------

def real_from_padded(buf: np.ndarray, dims: tuple[int, int, int]) -> np.ndarray:
    """View a flat FFTW-padded real buffer as a (z, y, x) array of the logical values."""
    x, y, z = dims
    _, pitch = padded_x(x)
    a = np.asarray(buf)[: pitch * y * z].reshape(z, y, pitch)
    return a[:, :, :x]


def real_to_padded(a: np.ndarray, dims: tuple[int, int, int], dtype=np.float32) -> np.ndarray:
    """Flat FFTW-padded buffer (pitch 2*(x/2+1)) holding a (z, y, x) array; pad slots are 0."""
    x, y, z = dims
    _, pitch = padded_x(x)
    out = np.zeros((z, y, pitch), dtype=dtype)
    out[:, :, :x] = np.asarray(a).reshape(z, y, x)
    return out.reshape(-1)


def spectrum_from_zyx(s_zyx: np.ndarray) -> np.ndarray:
    """numpy rfftn output [kz][ky][kx] -> reference layout [kz][kx][ky] (ky contiguous)."""
    return np.ascontiguousarray(np.transpose(s_zyx, (0, 2, 1)))


def spectrum_to_zyx(s_ref: np.ndarray) -> np.ndarray:
    """Reference layout [kz][kx][ky] -> numpy [kz][ky][kx]."""
    return np.ascontiguousarray(np.transpose(s_ref, (0, 2, 1)))


# ---------------------------------------------------------------------------
# Functors (include/detail/functors.h:15-80)
# ---------------------------------------------------------------------------

def apply_scale(a: np.ndarray, kind: int, scale: float) -> np.ndarray:
    if kind == OP_SCALE:
        return a * scale
    return a


def apply_intra(t: np.ndarray, img: np.ndarray, kind: int, scale: float) -> np.ndarray:
    """Intra-op on (template spectrum, image spectrum): CONJ_MUL = conj(t) * img."""
    if kind == OP_CONJ_MUL:
        return np.conj(t) * img
    if kind == OP_CONJ_MUL_THEN_SCALE:
        return np.conj(t) * img * scale
    if kind == OP_NOOP:
        return t
    raise ValueError(f"intra op kind {kind} not supported")


# ---------------------------------------------------------------------------
# Transforms
# ---------------------------------------------------------------------------

def _fft_backend(workers: int | None):
    if workers is None:
        return np.fft, {}
    import scipy.fft as sfft  # pocketfft, multithreaded

    return sfft, {"workers": workers}


def fwd(x_padded: np.ndarray, fwd_in, fwd_out, pre_op=(OP_NOOP, 1.0), dtype=np.float64,
        workers: int | None = None) -> np.ndarray:
    """FwdFFT: real input (FFTW-padded, dims fwd_in) -> spectrum [kz][kx][ky].

    The transform size per axis is max(in, out).  Increase: the input sits at the
    origin of a zero array.  Decrease: the full input is transformed and only the
    first out.y (ky), out.z (kz) and out.x/2+1 (kx) outputs are kept.
    Returns a complex array of shape (out.z, out.w, out.y).
    """
    fwd_in = tuple(fwd_in)
    fwd_out = tuple(fwd_out)
    nx, ny, nz = (max(a, b) for a, b in zip(fwd_in, fwd_out))
    src = real_from_padded(x_padded, fwd_in).astype(dtype)
    src = apply_scale(src, pre_op[0], pre_op[1])
    full = np.zeros((nz, ny, nx), dtype=dtype)
    full[: fwd_in[2], : fwd_in[1], : fwd_in[0]] = src
    be, kw = _fft_backend(workers)
    s = be.rfftn(full, axes=(0, 1, 2) if nz > 1 else (1, 2), **kw)
    wout, _ = padded_x(fwd_out[0])
    s = s[: fwd_out[2], : fwd_out[1], :wout]
    return spectrum_from_zyx(s)


def inv(s_ref: np.ndarray, inv_in, inv_out, post_op=(OP_NOOP, 1.0), dtype=np.float64,
        out_dtype=np.float32, workers: int | None = None, origin=(0, 0, 0)) -> np.ndarray:
    """InvFFT: spectrum [kz][kx][ky] of size inv_in -> real output, FFTW-padded, dims inv_out.

    Unnormalised (a forward/inverse round trip scales by Nx*Ny*Nz).  Decrease keeps
    the window [origin, origin + out) per axis (origin (0,0,0) is the reference's
    behaviour).  The imaginary parts of the kx = 0 and kx = N/2 bins are ignored,
    as in any C2R of a Hermitian spectrum.
    """
    inv_in = tuple(inv_in)
    inv_out = tuple(inv_out)
    nx, ny, nz = inv_in
    w, _ = padded_x(nx)
    s = np.asarray(s_ref).reshape(nz, w, ny).astype(np.complex128 if dtype == np.float64 else np.complex64)
    be, kw = _fft_backend(workers)
    axes = (0, 1, 2) if nz > 1 else (1, 2)
    zyx = spectrum_to_zyx(s)
    shape = (nz, ny, nx) if nz > 1 else (ny, nx)
    if nz == 1:
        zyx = zyx[0]
    r = be.irfftn(zyx, s=shape, axes=axes if nz > 1 else (0, 1), **kw)
    r = r * (nx * ny * nz)
    if nz == 1:
        r = r[None]
    ox, oy, oz = origin
    r = r[oz: oz + inv_out[2], oy: oy + inv_out[1], ox: ox + inv_out[0]]
    r = apply_scale(r, post_op[0], post_op[1])
    return real_to_padded(r, inv_out, dtype=out_dtype)


def fwd_image_inv(t_padded: np.ndarray, image_spectrum: np.ndarray, plan: Plan,
                  pre_op=(OP_NOOP, 1.0), intra_op=(OP_CONJ_MUL, 1.0), post_op=(OP_NOOP, 1.0),
                  dtype=np.float64, out_dtype=np.float32, workers: int | None = None,
                  origin=(0, 0, 0)) -> np.ndarray:
    """FwdImageInvFFT: pad template, forward, intra-op against the image spectrum, inverse.

    Output = irfftn(conj(rfftn(T_pad)) * I_hat) * N (unnormalised), cropped to inv_out.
    Equivalently c[r] = N * sum_x T(x) I(x + r) (mod N), N = Nx*Ny*Nz.
    """
    t_hat = fwd(t_padded, plan.fwd_in, plan.fwd_out, pre_op, dtype=dtype, workers=workers)
    img = np.asarray(image_spectrum).reshape(t_hat.shape)
    prod = apply_intra(t_hat, img.astype(t_hat.dtype), intra_op[0], intra_op[1])
    return inv(prod, plan.inv_in, plan.inv_out, post_op, dtype=dtype, out_dtype=out_dtype,
               workers=workers, origin=origin)


# ---------------------------------------------------------------------------
# Complex-input (C2C) transforms.  The reference declares complex InputType but leaves its
# complex paths as stubs (src/fastfft/FastFFT.cu:369-391, 3D cross-correlation :722-793);
# these follow the conventions of its real path: sign -1 forward, unnormalised, zero padding
# at the origin, the transposed spectrum layout [kz][kx][ky] (kx now over all N_x), the
# window of a decrease at the origin (or at `origin`), complex rows of pitch x
# (ReturnPaddedMemorySize's complex branch, include/FastFFT.h:381-384).
# ---------------------------------------------------------------------------

def complex_memory_size(dims: tuple[int, int, int]) -> int:
    """Scalar components the reference reserves for complex dims (x, y, z): 2 x y z."""
    x, y, z = dims
    return 2 * x * y * z


def complex_from_buffer(buf: np.ndarray, dims: tuple[int, int, int]) -> np.ndarray:
    """View a flat complex buffer (interleaved re, im; rows of pitch x) as a (z, y, x) array."""
    x, y, z = dims
    a = np.asarray(buf).reshape(-1)
    if not np.iscomplexobj(a):
        a = a[: 2 * x * y * z].astype(np.float64).view(np.complex128)
    return a[: x * y * z].reshape(z, y, x)


def complex_to_buffer(a: np.ndarray, dtype=np.complex64) -> np.ndarray:
    """Flat interleaved buffer of a complex (z, y, x) array (rows of pitch x)."""
    return np.ascontiguousarray(np.asarray(a).reshape(-1).astype(dtype))


def fwd_c2c(x: np.ndarray, fwd_in, fwd_out, pre_op=(OP_NOOP, 1.0), dtype=np.complex128) -> np.ndarray:
    """C2C FwdFFT: complex (z, y, x) input of dims fwd_in -> spectrum [kz][kx][ky] of dims
    fwd_out (first outputs per axis kept on a decrease), shape (out.z, out.x, out.y)."""
    fwd_in, fwd_out = tuple(fwd_in), tuple(fwd_out)
    nx, ny, nz = (max(a, b) for a, b in zip(fwd_in, fwd_out))
    src = apply_scale(np.asarray(x, dtype=dtype).reshape(fwd_in[2], fwd_in[1], fwd_in[0]), pre_op[0], pre_op[1])
    full = np.zeros((nz, ny, nx), dtype=dtype)
    full[: fwd_in[2], : fwd_in[1], : fwd_in[0]] = src
    s = np.fft.fftn(full, axes=(0, 1, 2) if nz > 1 else (1, 2))
    s = s[: fwd_out[2], : fwd_out[1], : fwd_out[0]]
    return spectrum_from_zyx(s)


def inv_c2c(s_ref: np.ndarray, inv_in, inv_out, post_op=(OP_NOOP, 1.0), origin=(0, 0, 0)) -> np.ndarray:
    """C2C InvFFT: spectrum [kz][kx][ky] of dims inv_in -> complex (z, y, x) window of dims
    inv_out at `origin`, unnormalised (a round trip scales by Nx Ny Nz)."""
    nx, ny, nz = tuple(inv_in)
    s = np.asarray(s_ref, dtype=np.complex128).reshape(nz, nx, ny)
    r = np.fft.ifftn(spectrum_to_zyx(s), axes=(0, 1, 2) if nz > 1 else (1, 2)) * (nx * ny * nz)
    ox, oy, oz = origin
    r = r[oz: oz + inv_out[2], oy: oy + inv_out[1], ox: ox + inv_out[0]]
    return apply_scale(r, post_op[0], post_op[1])


def fwd_image_inv_c2c(t: np.ndarray, image_spectrum: np.ndarray, plan: Plan, pre_op=(OP_NOOP, 1.0),
                      intra_op=(OP_CONJ_MUL, 1.0), post_op=(OP_NOOP, 1.0), origin=(0, 0, 0)) -> np.ndarray:
    """C2C FwdImageInvFFT: conj(fft(T_pad)) x image spectrum (full [kz][kx][ky] layout), inverse,
    window.  c[r] = N sum_x conj(T(x)) I(x + r) (mod N)."""
    t_hat = fwd_c2c(t, plan.fwd_in, plan.fwd_out, pre_op)
    img = np.asarray(image_spectrum).reshape(t_hat.shape)
    prod = apply_intra(t_hat, img.astype(np.complex128), intra_op[0], intra_op[1])
    return inv_c2c(prod, plan.inv_in, plan.inv_out, post_op, origin=origin)


# ---------------------------------------------------------------------------
# Metrics
# ---------------------------------------------------------------------------

def rel_l2(a: np.ndarray, ref: np.ndarray) -> float:
    a = np.asarray(a, dtype=np.complex128 if np.iscomplexobj(a) or np.iscomplexobj(ref) else np.float64)
    ref = np.asarray(ref, dtype=a.dtype)
    den = np.linalg.norm(ref.ravel())
    return float(np.linalg.norm((a - ref).ravel()) / (den if den > 0 else 1.0))


def rel_max(a: np.ndarray, ref: np.ndarray) -> float:
    a = np.asarray(a)
    ref = np.asarray(ref)
    den = np.max(np.abs(ref)) if ref.size else 1.0
    return float(np.max(np.abs(a - ref)) / (den if den > 0 else 1.0))


def peak(window: np.ndarray) -> tuple[int, float, float]:
    """(flat argmax with first-occurrence tie break, top value, top1 - top2 margin)."""
    flat = np.asarray(window).ravel()
    idx = int(np.argmax(flat))
    top = float(flat[idx])
    rest = np.delete(flat, idx)
    margin = top - float(rest.max()) if rest.size else float("inf")
    return idx, top, margin


# ---------------------------------------------------------------------------
# Seeded synthetic inputs for the workloads
# ---------------------------------------------------------------------------

SEED_BASE = 20261203


def gaussian_blob_image(n: int, n_blobs: int = 20, sigma: float = 8.0, amp: float = 5.0,
                        seed: int = SEED_BASE + 2) -> np.ndarray:
    """n x n image of N(0,1) noise plus Gaussian blobs at seeded centres in [32, n-32)."""
    rng = np.random.default_rng(seed)
    img = rng.standard_normal((n, n))
    lo, hi = min(32, n // 4), max(n - 32, 3 * n // 4)
    centres = rng.uniform(lo, hi, size=(n_blobs, 2))
    r = int(np.ceil(4 * sigma))
    yy, xx = np.mgrid[-r: r + 1, -r: r + 1]
    for cy, cx in centres:
        iy, ix = int(np.floor(cy)), int(np.floor(cx))
        fy, fx = cy - iy, cx - ix
        g = amp * np.exp(-((yy - fy) ** 2 + (xx - fx) ** 2) / (2 * sigma * sigma))
        y0, x0 = iy - r, ix - r
        ys = slice(max(y0, 0), min(y0 + 2 * r + 1, n))
        xs = slice(max(x0, 0), min(x0 + 2 * r + 1, n))
        img[ys, xs] += g[ys.start - y0: ys.stop - y0, xs.start - x0: xs.stop - x0]
    return img


def normal_template(edge: int, seed: int) -> np.ndarray:
    return np.random.default_rng(seed).standard_normal((edge, edge))


def image_spectrum_fp32(img: np.ndarray) -> np.ndarray:
    """FP64 R2C of a 2D image, rounded to complex64, in the [kx][ky] layout (shape (1, w, n))."""
    n = img.shape[0]
    padded = real_to_padded(img, (img.shape[1], n, 1), dtype=np.float64)
    s = fwd(padded, (img.shape[1], n, 1), (img.shape[1], n, 1))
    return s.astype(np.complex64)


def cpu_workers() -> int:
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)


# ---------------------------------------------------------------------------
# Radial operations on square 2D half spectra (image-spectrum preparation; no reference
# counterpart: these define the semantics fastfft_radial_power / fastfft_apply_radial_filter
# implement)
# ---------------------------------------------------------------------------

def radial_index(n: int, n_bins: int) -> np.ndarray:
    """Bin of every element of an n x n half spectrum [kx][ky]: floor(sqrt(kx^2 + sy^2)) with
    the signed ky (sy = ky - n above n/2), clipped to n_bins - 1."""
    kx = np.arange(n // 2 + 1, dtype=np.int64)[:, None]
    ky = np.arange(n, dtype=np.int64)[None, :]
    sy = np.where(ky <= n // 2, ky, ky - n)
    r = np.floor(np.sqrt((kx * kx + sy * sy).astype(np.float64))).astype(np.int64)
    return np.minimum(r, n_bins - 1)


def radial_power(spec: np.ndarray, n: int, n_bins: int) -> np.ndarray:
    """Mean |S|^2 per radius over the full spectrum (columns 0 < kx < n/2 count twice)."""
    s = np.asarray(spec).reshape(n // 2 + 1, n)
    idx = radial_index(n, n_bins)
    w = np.full((n // 2 + 1, 1), 2.0)
    w[0] = w[-1] = 1.0
    w = np.broadcast_to(w, s.shape)
    sums = np.bincount(idx.ravel(), weights=(w * np.abs(s) ** 2).ravel(), minlength=n_bins)
    wts = np.bincount(idx.ravel(), weights=w.ravel(), minlength=n_bins)
    return np.where(wts > 0, sums / np.where(wts > 0, wts, 1), 0.0)


def radial_filter(spec: np.ndarray, n: int, filt: np.ndarray, scale: float = 1.0) -> np.ndarray:
    s = np.asarray(spec).reshape(n // 2 + 1, n)
    return s * (np.asarray(filt, dtype=np.float64)[radial_index(n, len(filt))] * scale)
