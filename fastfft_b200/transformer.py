"""Python mirror of FastFFT::FourierTransformer over the C ABI.

Method names, argument order and meaning follow the reference class
(include/FastFFT.h:84-219): SetForwardFFTPlan / SetInverseFFTPlan, FwdFFT, InvFFT,
FwdImageInvFFT, Return*MemorySize, Return*Dimensions, Wait.  Buffers are device
pointers: torch CUDA tensors or raw integer addresses.  Where the reference calls
std::abort() on a user error, this class raises FastFFTError with the library's
message.

Work is queued on torch's current CUDA stream unless a stream was set explicitly
with SetStream (the reference always uses cudaStreamPerThread, usage.md:13).
"""
from __future__ import annotations

import ctypes

from . import _capi as C

_REAL_DTYPES = {"float32": C.DTYPE_F32, "float16": C.DTYPE_F16, "bfloat16": C.DTYPE_BF16}
_CPLX_DTYPES = {"complex64": C.DTYPE_C64, "complex32": C.DTYPE_C32H, "chalf": C.DTYPE_C32H,
                "complex_bf16": C.DTYPE_C32BF}
# InputType: real (R2C / C2R transforms) or complex (C2C transforms; the reference declares
# complex InputType but leaves its paths as stubs, src/fastfft/FastFFT.cu:369-391)
_INPUT_DTYPES = {**_REAL_DTYPES, **_CPLX_DTYPES}


def _dtype_code(name, table):
    name = str(name).replace("torch.", "")
    if name not in table:
        raise ValueError(f"unsupported dtype {name}; expected one of {sorted(table)}")
    return table[name]


class KernelFunction:
    """Functor descriptors, mirroring KernelFunction::my_functor (include/detail/functors.h)."""

    @staticmethod
    def noop():
        return C.fastfft_op(C.OP_NOOP, 1.0)

    @staticmethod
    def scale(s: float):
        return C.fastfft_op(C.OP_SCALE, float(s))

    @staticmethod
    def conj_mul():
        return C.fastfft_op(C.OP_CONJ_MUL, 1.0)

    @staticmethod
    def conj_mul_then_scale(s: float):
        return C.fastfft_op(C.OP_CONJ_MUL_THEN_SCALE, float(s))


def _ptr(x) -> int | None:
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        if hasattr(x, "is_cuda") and not x.is_cuda:
            raise ValueError("FastFFT buffers must be CUDA device memory")
        return x.data_ptr()
    raise TypeError(f"cannot take a device pointer of {type(x)}")


def _opref(op):
    return ctypes.byref(op) if op is not None else None


def decode_peaks(peaks):
    """(values float32, flat indices int64) of keys written by FwdImageInvFFTManyPeaks (host numpy)."""
    import numpy as np

    k = np.asarray(peaks.cpu() if hasattr(peaks, "cpu") else peaks).astype(np.int64).view(np.uint64)
    ordered = (k >> np.uint64(32)).astype(np.uint32)
    bits = np.where(ordered & np.uint32(0x80000000), ordered & np.uint32(0x7FFFFFFF), ~ordered).astype(np.uint32)
    index = (np.uint64(0xFFFFFFFF) - (k & np.uint64(0xFFFFFFFF))).astype(np.int64)
    return bits.view(np.float32), index


class FourierTransformer:
    def __init__(self, compute_dtype="float32", input_dtype="float32", image_dtype="complex64", rank=2):
        self._lib = C.lib()
        self._h = C.Handle()
        st = self._lib.fastfft_create(ctypes.byref(self._h), _dtype_code(compute_dtype, {"float32": 0}),
                                      _dtype_code(input_dtype, _INPUT_DTYPES),
                                      _dtype_code(image_dtype, _CPLX_DTYPES), int(rank))
        if st != C.OK:
            raise C.FastFFTError(st, self._lib.fastfft_last_error(None).decode())
        self._stream = None
        self.rank = rank
        self.complex_input = str(input_dtype).replace("torch.", "") in _CPLX_DTYPES

    def __del__(self):
        h = getattr(self, "_h", None)
        lib = getattr(self, "_lib", None)
        if h is not None and h.value and lib is not None:
            try:
                lib.fastfft_destroy(h)
            except Exception:  # interpreter shutdown: the library may already be gone
                pass
            self._h = None     # (module globals such as C.Handle may be gone at shutdown)

    # -- helpers ---------------------------------------------------------
    def _check(self, st):
        if st != C.OK:
            raise C.FastFFTError(st, self._lib.fastfft_last_error(self._h).decode())

    def _bind_stream(self):
        if self._stream is not None:
            return
        try:
            import torch
        except ImportError:  # pragma: no cover - torch is part of the image
            return
        if torch.cuda.is_available():
            self._check(self._lib.fastfft_set_stream(self._h, ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))

    # -- plans -----------------------------------------------------------
    def SetForwardFFTPlan(self, ix, iy, iz, ox, oy, oz, is_padded_output=True):
        self._check(self._lib.fastfft_set_forward_plan(self._h, ix, iy, iz, ox, oy, oz, int(bool(is_padded_output))))

    def SetInverseFFTPlan(self, ix, iy, iz, ox, oy, oz, is_padded_output=True):
        self._check(self._lib.fastfft_set_inverse_plan(self._h, ix, iy, iz, ox, oy, oz, int(bool(is_padded_output))))

    def SetStream(self, stream):
        """Fix the work stream (a torch.cuda.Stream, a raw cudaStream_t, or None for cudaStreamPerThread)."""
        raw = getattr(stream, "cuda_stream", stream)
        self._stream = stream if stream is not None else 0
        self._check(self._lib.fastfft_set_stream(self._h, ctypes.c_void_p(raw) if raw else None))

    def SetInverseOutputOrigin(self, ox, oy, oz=0):
        """First retained output of an inverse size decrease (default 0, the reference's window)."""
        self._check(self._lib.fastfft_set_inverse_output_origin(self._h, ox, oy, oz))

    def SetOutputDtype(self, dtype):
        """Storage of the inverse's output: real for real-input plans, complex for complex-input plans."""
        table = _CPLX_DTYPES if self.complex_input else _REAL_DTYPES
        self._check(self._lib.fastfft_set_output_dtype(self._h, _dtype_code(dtype, table)))

    # -- transforms ------------------------------------------------------
    def FwdFFT(self, input_ptr, output_ptr=None, pre_op=None, intra_op=None):
        self._bind_stream()
        self._check(self._lib.fastfft_fwd(self._h, _ptr(input_ptr), _ptr(output_ptr), _opref(pre_op), _opref(intra_op)))

    def InvFFT(self, input_ptr, output_ptr=None, intra_op=None, post_op=None):
        self._bind_stream()
        self._check(self._lib.fastfft_inv(self._h, _ptr(input_ptr), _ptr(output_ptr), _opref(intra_op), _opref(post_op)))

    def FwdImageInvFFT(self, input_ptr, image_to_search, output_ptr=None, pre_op=None, intra_op=None, post_op=None):
        if intra_op is None:
            intra_op = KernelFunction.conj_mul()
        self._bind_stream()
        self._check(self._lib.fastfft_fwd_image_inv(self._h, _ptr(input_ptr), _ptr(image_to_search), _ptr(output_ptr),
                                                    _opref(pre_op), _opref(intra_op), _opref(post_op)))

    def FwdImageInvFFTMany(self, inputs, images, outputs=None, pre_op=None, intra_op=None, post_op=None):
        """FwdImageInvFFT over a list of templates in one library call.

        images is one image (searched by every template) or a list with one image per
        template; outputs is a list of the same length as inputs, or None (in place).
        """
        n = len(inputs)
        if not isinstance(images, (list, tuple)):
            images = [images] * n
        if len(images) != n or (outputs is not None and len(outputs) != n):
            raise ValueError("inputs, images and outputs must have the same length")
        if intra_op is None:
            intra_op = KernelFunction.conj_mul()
        arr = ctypes.c_void_p * n
        ins = arr(*[_ptr(x) for x in inputs])
        ims = arr(*[_ptr(x) for x in images])
        outs = arr(*[_ptr(x) for x in outputs]) if outputs is not None else None
        self._bind_stream()
        self._check(self._lib.fastfft_fwd_image_inv_many(self._h, n, ins, ims, outs, _opref(pre_op), _opref(intra_op),
                                                         _opref(post_op)))

    def FwdImageInvFFTManySized(self, inputs, sizes, images, outputs=None, pre_op=None, intra_op=None,
                                post_op=None):
        """FwdImageInvFFTMany for templates of uneven sizes: sizes[i] = (x, y) of template i."""
        n = len(inputs)
        if not isinstance(images, (list, tuple)):
            images = [images] * n
        if len(sizes) != n or len(images) != n or (outputs is not None and len(outputs) != n):
            raise ValueError("inputs, sizes, images and outputs must have the same length")
        if intra_op is None:
            intra_op = KernelFunction.conj_mul()
        arr = ctypes.c_void_p * n
        dims = (ctypes.c_int * (2 * n))(*[int(v) for xy in sizes for v in xy])
        ins = arr(*[_ptr(x) for x in inputs])
        ims = arr(*[_ptr(x) for x in images])
        outs = arr(*[_ptr(x) for x in outputs]) if outputs is not None else None
        self._bind_stream()
        self._check(self._lib.fastfft_fwd_image_inv_many_sized(self._h, n, ins, dims, ims, outs, _opref(pre_op),
                                                               _opref(intra_op), _opref(post_op)))

    def FwdImageInvFFTManyPeaks(self, inputs, images, peaks, sizes=None, outputs=None, pre_op=None, intra_op=None,
                                post_op=None):
        """Batched correlation with a fused peak search into `peaks` (int64 CUDA tensor, one per
        template; decode with decode_peaks).  outputs None: the windows are not written."""
        n = len(inputs)
        if not isinstance(images, (list, tuple)):
            images = [images] * n
        if len(images) != n or (outputs is not None and len(outputs) != n) or (sizes is not None and len(sizes) != n):
            raise ValueError("inputs, images, sizes and outputs must have the same length")
        if peaks.numel() < n or peaks.element_size() != 8:
            raise ValueError("peaks must hold one 64-bit value per template")
        if intra_op is None:
            intra_op = KernelFunction.conj_mul()
        arr = ctypes.c_void_p * n
        dims = (ctypes.c_int * (2 * n))(*[int(v) for xy in sizes for v in xy]) if sizes is not None else None
        ins = arr(*[_ptr(x) for x in inputs])
        ims = arr(*[_ptr(x) for x in images])
        outs = arr(*[_ptr(x) for x in outputs]) if outputs is not None else None
        self._bind_stream()
        self._check(self._lib.fastfft_fwd_image_inv_many_peaks(self._h, n, ins, dims, ims, outs, _ptr(peaks),
                                                               _opref(pre_op), _opref(intra_op), _opref(post_op)))

    def FwdImageInvFFTManyMip(self, inputs, images, mip, sizes=None, outputs=None, index_base=0, pre_op=None,
                              intra_op=None, post_op=None):
        """Batched correlation with a fused maximum projection across templates: every
        retained pixel of mip (int64 CUDA tensor of out_x * out_y keys, row-major; zero it
        before the first call) keeps the best score over the templates and its template
        number index_base + i (decode with decode_peaks).  The array accumulates across
        calls.  outputs None: the windows are not written."""
        n = len(inputs)
        if not isinstance(images, (list, tuple)):
            images = [images] * n
        if len(images) != n or (outputs is not None and len(outputs) != n) or (sizes is not None and len(sizes) != n):
            raise ValueError("inputs, images, sizes and outputs must have the same length")
        out_x, out_y = self.ReturnInvOutputDimensions()[:2]
        if mip.numel() < out_x * out_y or mip.element_size() != 8:
            raise ValueError("mip must hold one 64-bit value per window pixel (out_x * out_y)")
        if intra_op is None:
            intra_op = KernelFunction.conj_mul()
        arr = ctypes.c_void_p * n
        dims = (ctypes.c_int * (2 * n))(*[int(v) for xy in sizes for v in xy]) if sizes is not None else None
        ins = arr(*[_ptr(x) for x in inputs])
        ims = arr(*[_ptr(x) for x in images])
        outs = arr(*[_ptr(x) for x in outputs]) if outputs is not None else None
        self._bind_stream()
        self._check(self._lib.fastfft_fwd_image_inv_many_mip(self._h, n, ins, dims, ims, outs, _ptr(mip),
                                                             int(index_base), _opref(pre_op), _opref(intra_op),
                                                             _opref(post_op)))

    def SetTemplatesPerLaunch(self, n):
        self._check(self._lib.fastfft_set_templates_per_launch(self._h, int(n)))

    def TemplatesPerLaunch(self):
        v = ctypes.c_int()
        self._check(self._lib.fastfft_templates_per_launch(self._h, ctypes.byref(v)))
        return v.value

    def SetTemplatesPerBlock(self, n):
        """Templates one block of the batched fused column pass serves (0: the built-in choice)."""
        self._check(self._lib.fastfft_set_templates_per_block(self._h, int(n)))

    def TemplatesPerBlock(self):
        v = ctypes.c_int()
        self._check(self._lib.fastfft_templates_per_block(self._h, ctypes.byref(v)))
        return v.value

    def SetPipelinedGroups(self, n):
        """1 or 2 groups of templates in flight in the batched reduced-size path (2: consecutive
        groups alternate between two streams, each group's intermediates small enough for L2)."""
        self._check(self._lib.fastfft_set_pipelined_groups(self._h, int(n)))

    def PipelinedGroups(self):
        v = ctypes.c_int()
        self._check(self._lib.fastfft_pipelined_groups(self._h, ctypes.byref(v)))
        return v.value

    def SetImageReuse(self, enable=True):
        """Declare that image spectra do not change while in use: the reduced spectrum prepared
        for an image address is reused by later calls naming the same address (single
        FwdImageInvFFT calls then also correlate at the reduced size).  Calling it again, or
        changing the plan or stream, forgets the prepared image."""
        self._check(self._lib.fastfft_set_image_reuse(self._h, int(bool(enable))))

    def SetSpectrumOutput(self, dtype="complex64", scale=1.0):
        """FwdFFT writes its spectrum as `dtype` ("complex64", "complex32" or "complex_bf16"),
        every value multiplied by `scale` and rounded once: the normalised, quantised image
        spectrum for FwdImageInvFFT with a matching image_dtype."""
        self._check(self._lib.fastfft_set_spectrum_output(self._h, _dtype_code(dtype, _CPLX_DTYPES), float(scale)))

    def RadialPower(self, spectrum, n, power):
        """power[r] (float32 device tensor of n_bins) = mean |S|^2 over the elements of the n x n
        complex64 half spectrum `spectrum` at radius r = floor(sqrt(kx^2 + ky^2)); the last bin
        also holds every larger radius."""
        self._bind_stream()
        self._check(self._lib.fastfft_radial_power(self._h, _ptr(spectrum), int(n), _ptr(power), int(power.numel())))

    def ApplyRadialFilter(self, spectrum, output, n, filt):
        """output = spectrum x filt[r] (radius as in RadialPower), written in the storage and
        scale set by SetSpectrumOutput; in place only with complex64 storage."""
        self._bind_stream()
        self._check(self._lib.fastfft_apply_radial_filter(self._h, _ptr(spectrum), _ptr(output), int(n), _ptr(filt),
                                                          int(filt.numel())))

    def SetTensorCoreDFT(self, enable=True):
        """Run the radix-16 passes of the batched correlation's fused column pass on the tensor
        cores in BF16 split precision (about 1e-5 relative L2 against FP64) where the pass has
        that form (correlation length 1536 along y); slower than the FP32 default."""
        self._check(self._lib.fastfft_set_tensor_core_dft(self._h, int(bool(enable))))

    def TensorCoreDFTActive(self):
        v = ctypes.c_int()
        self._check(self._lib.fastfft_tensor_core_dft_active(self._h, ctypes.byref(v)))
        return bool(v.value)

    def SetFullSizeCorrelation(self, force=True):
        """Make FwdImageInvFFTMany use the size-N kernels even when a smaller size is exact."""
        self._check(self._lib.fastfft_set_full_size_correlation(self._h, int(bool(force))))

    def CorrelationSize(self):
        d = (ctypes.c_int * 2)()
        self._check(self._lib.fastfft_correlation_size(self._h, d))
        return tuple(d)

    # -- accounting and profiling ------------------------------------------
    def LaunchCount(self):
        return self._ll(self._lib.fastfft_launch_count)

    def ProfileStart(self, max_calls):
        self._check(self._lib.fastfft_profile_start(self._h, int(max_calls)))

    def ProfileStop(self):
        """Returns ([ms of pass 0, 1, 2 summed over the recorded calls], n_calls)."""
        ms = (ctypes.c_double * 3)()
        n = ctypes.c_longlong()
        self._check(self._lib.fastfft_profile_stop(self._h, ms, 3, ctypes.byref(n)))
        return list(ms), n.value

    def Wait(self):
        self._check(self._lib.fastfft_wait(self._h))

    # -- queries ---------------------------------------------------------
    def _ll(self, fn):
        v = ctypes.c_longlong()
        self._check(fn(self._h, ctypes.byref(v)))
        return v.value

    def ReturnInputMemorySize(self):
        return self._ll(self._lib.fastfft_input_memory_size)

    def ReturnFwdOutputMemorySize(self):
        return self._ll(self._lib.fastfft_fwd_output_memory_size)

    def ReturnInvOutputMemorySize(self):
        return self._ll(self._lib.fastfft_inv_output_memory_size)

    def ReturnBufferBytes(self):
        return self._ll(self._lib.fastfft_buffer_bytes)

    def _dims(self, fn):
        d = (ctypes.c_int * 4)()
        self._check(fn(self._h, d))
        return tuple(d)

    def ReturnFwdInputDimensions(self):
        return self._dims(self._lib.fastfft_fwd_input_dims)

    def ReturnFwdOutputDimensions(self):
        return self._dims(self._lib.fastfft_fwd_output_dims)

    def ReturnInvInputDimensions(self):
        return self._dims(self._lib.fastfft_inv_input_dims)

    def ReturnInvOutputDimensions(self):
        return self._dims(self._lib.fastfft_inv_output_dims)
