"""ctypes binding of libfastfft_b200.so (declarations in include/fastfft_capi.h).

The shared library is built in-tree (``python -m fastfft_b200.build``) and loaded from
this package directory.  There is no fallback implementation: if the library is
missing, importing this module raises.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libfastfft_b200.so"

# fastfft_status
OK = 0
ERR_INVALID_ARGUMENT = 1
ERR_INVALID_DIMS = 2
ERR_UNSUPPORTED = 3
ERR_NOT_PLANNED = 4
ERR_CUDA = 5
ERR_ALLOC = 6
ERR_TIMEOUT = 7

# fastfft_dtype
DTYPE_F32 = 0
DTYPE_F16 = 1
DTYPE_BF16 = 2
DTYPE_C64 = 3
DTYPE_C32H = 4
DTYPE_C32BF = 5

# fastfft_op_kind
OP_NOOP = 0
OP_SCALE = 1
OP_CONJ_MUL = 2
OP_CONJ_MUL_THEN_SCALE = 3


class fastfft_op(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("scale", ctypes.c_float)]


Handle = ctypes.c_void_p
_st = ctypes.c_int
_sz = ctypes.c_size_t
_vp = ctypes.c_void_p
_op = ctypes.POINTER(fastfft_op)
_dims = ctypes.POINTER(ctypes.c_int)
_ll = ctypes.POINTER(ctypes.c_longlong)

# name -> (restype, argtypes); the set of exported entry points of the C ABI
SIGNATURES = {
    "fastfft_create": (_st, [ctypes.POINTER(Handle), ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "fastfft_destroy": (_st, [Handle]),
    "fastfft_set_forward_plan": (_st, [Handle, _sz, _sz, _sz, _sz, _sz, _sz, ctypes.c_int]),
    "fastfft_set_inverse_plan": (_st, [Handle, _sz, _sz, _sz, _sz, _sz, _sz, ctypes.c_int]),
    "fastfft_set_stream": (_st, [Handle, _vp]),
    "fastfft_set_output_dtype": (_st, [Handle, ctypes.c_int]),
    "fastfft_set_inverse_output_origin": (_st, [Handle, _sz, _sz, _sz]),
    "fastfft_fwd": (_st, [Handle, _vp, _vp, _op, _op]),
    "fastfft_inv": (_st, [Handle, _vp, _vp, _op, _op]),
    "fastfft_fwd_image_inv": (_st, [Handle, _vp, _vp, _vp, _op, _op, _op]),
    "fastfft_fwd_image_inv_many": (_st, [Handle, ctypes.c_int, ctypes.POINTER(_vp), ctypes.POINTER(_vp),
                                         ctypes.POINTER(_vp), _op, _op, _op]),
    "fastfft_launch_count": (_st, [Handle, _ll]),
    "fastfft_fwd_image_inv_many_sized": (_st, [Handle, ctypes.c_int, ctypes.POINTER(_vp), ctypes.POINTER(ctypes.c_int),
                                               ctypes.POINTER(_vp), ctypes.POINTER(_vp), _op, _op, _op]),
    "fastfft_set_templates_per_launch": (_st, [Handle, ctypes.c_int]),
    "fastfft_set_pipelined_groups": (_st, [Handle, ctypes.c_int]),
    "fastfft_set_templates_per_block": (_st, [Handle, ctypes.c_int]),
    "fastfft_templates_per_block": (_st, [Handle, ctypes.POINTER(ctypes.c_int)]),
    "fastfft_pipelined_groups": (_st, [Handle, ctypes.POINTER(ctypes.c_int)]),
    "fastfft_set_image_reuse": (_st, [Handle, ctypes.c_int]),
    "fastfft_set_tensor_core_dft": (_st, [Handle, ctypes.c_int]),
    "fastfft_set_spectrum_output": (_st, [Handle, ctypes.c_int, ctypes.c_float]),
    "fastfft_radial_power": (_st, [Handle, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int]),
    "fastfft_apply_radial_filter": (_st, [Handle, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                          ctypes.c_int]),
    "fastfft_tensor_core_dft_active": (_st, [Handle, ctypes.POINTER(ctypes.c_int)]),
    "fastfft_fwd_image_inv_many_peaks": (_st, [Handle, ctypes.c_int, ctypes.POINTER(_vp), ctypes.POINTER(ctypes.c_int),
                                               ctypes.POINTER(_vp), ctypes.POINTER(_vp), _vp, _op, _op, _op]),
    "fastfft_fwd_image_inv_many_mip": (_st, [Handle, ctypes.c_int, ctypes.POINTER(_vp), ctypes.POINTER(ctypes.c_int),
                                             ctypes.POINTER(_vp), ctypes.POINTER(_vp), _vp, ctypes.c_int, _op, _op,
                                             _op]),
    "fastfft_decode_peak": (None, [ctypes.c_ulonglong, ctypes.POINTER(ctypes.c_float),
                                   ctypes.POINTER(ctypes.c_uint)]),
    "fastfft_templates_per_launch": (_st, [Handle, ctypes.POINTER(ctypes.c_int)]),
    "fastfft_fwd_image_inv_2d_noalloc": (_st, [_vp, ctypes.c_int, ctypes.c_int, _vp, ctypes.c_int, ctypes.c_int, _vp,
                                               ctypes.c_int, ctypes.c_int, _op, _op, _op, _vp]),
    "fastfft_set_full_size_correlation": (_st, [Handle, ctypes.c_int]),
    "fastfft_correlation_size": (_st, [Handle, _dims]),
    "fastfft_profile_start": (_st, [Handle, ctypes.c_int]),
    "fastfft_profile_stop": (_st, [Handle, ctypes.POINTER(ctypes.c_double), ctypes.c_int, _ll]),
    "fastfft_input_memory_size": (_st, [Handle, _ll]),
    "fastfft_fwd_output_memory_size": (_st, [Handle, _ll]),
    "fastfft_inv_output_memory_size": (_st, [Handle, _ll]),
    "fastfft_fwd_input_dims": (_st, [Handle, _dims]),
    "fastfft_fwd_output_dims": (_st, [Handle, _dims]),
    "fastfft_inv_input_dims": (_st, [Handle, _dims]),
    "fastfft_inv_output_dims": (_st, [Handle, _dims]),
    "fastfft_buffer_bytes": (_st, [Handle, _ll]),
    "fastfft_wait": (_st, [Handle]),
    "fastfft_last_error": (ctypes.c_char_p, [Handle]),
    "fastfft_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "fastfft_version": (ctypes.c_char_p, []),
}


def load(path: Path | str = LIB_PATH) -> ctypes.CDLL:
    path = Path(path)
    if not path.exists():
        raise ImportError(
            f"{path} is missing: the CUDA library is not built (python -m fastfft_b200.build). "
            "There is no CPU fallback.")
    lib = ctypes.CDLL(str(path))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


class FastFFTError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"[{status}] {message}")
        self.status = status


_lib: ctypes.CDLL | None = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        _lib = load()
    return _lib
