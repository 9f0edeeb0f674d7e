"""C ABI checks that need no GPU: exported symbols, plan validation, size queries.

The size queries must return the reference's numbers (ReturnPaddedMemorySize,
include/FastFFT.h:363-404) and the validation must reject what ValidateDimensions
rejects (src/fastfft/FastFFT.cu:803-930), with a status code instead of abort().
"""
import ctypes
import os
import re

import pytest

import fastfft_b200 as F
from fastfft_b200 import _capi as C
from oracle import fastfft_oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "fastfft_capi.h")).read()
    return sorted(set(re.findall(r"FASTFFT_API\s+[\w\s\*]+?\b(fastfft_\w+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(str(C.LIB_PATH))
    names = header_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(C.SIGNATURES), "binding and header disagree"


def test_version_and_status_strings():
    lib = C.lib()
    assert b"sm_100a" in lib.fastfft_version()
    assert lib.fastfft_status_string(C.ERR_INVALID_DIMS) == b"invalid dimensions"


def new(rank=2, input_dtype="float32"):
    return F.FourierTransformer(input_dtype=input_dtype, rank=rank)


@pytest.mark.parametrize("fin,fout,iout", [
    ((64, 64, 1), (512, 512, 1), (512, 512, 1)),
    ((384, 384, 1), (4096, 4096, 1), (1024, 1024, 1)),
    ((385, 200, 1), (4096, 2048, 1), (1000, 999, 1)),
    ((4096, 4096, 1), (4096, 4096, 1), (4096, 4096, 1)),
    ((64, 64, 64), (256, 256, 256), (128, 128, 128)),
])
def test_memory_sizes_match_reference(fin, fout, iout):
    ft = new(rank=3 if fout[2] > 1 else 2)
    ft.SetForwardFFTPlan(*fin, *fout)
    ft.SetInverseFFTPlan(*fout, *iout)
    assert ft.ReturnInputMemorySize() == O.padded_memory_size(fin)
    assert ft.ReturnFwdOutputMemorySize() == O.padded_memory_size(fout)
    assert ft.ReturnInvOutputMemorySize() == O.padded_memory_size(iout)
    assert ft.ReturnFwdInputDimensions() == (*fin, O.padded_x(fin[0])[0])
    assert ft.ReturnFwdOutputDimensions() == (*fout, O.padded_x(fout[0])[0])
    assert ft.ReturnInvOutputDimensions() == (*iout, O.padded_x(iout[0])[0])


@pytest.mark.parametrize("fin,fout,iin,iout,status", [
    ((64, 64, 1), (512, 512, 1), (256, 256, 1), (256, 256, 1), C.ERR_INVALID_DIMS),  # fwd out != inv in
    ((64, 128, 1), (128, 64, 1), (128, 64, 1), (128, 64, 1), C.ERR_INVALID_DIMS),    # mixed grow/shrink
    ((64, 64, 1), (10240, 64, 1), (10240, 64, 1), (10240, 64, 1), C.ERR_INVALID_DIMS),  # 5 * 2^k above 5120
    ((64, 64, 1), (7168, 64, 1), (7168, 64, 1), (7168, 64, 1), C.ERR_INVALID_DIMS),  # 7 * 2^k above 3584
    ((16, 16, 16), (384, 384, 384), (384, 384, 384), (384, 384, 384), C.ERR_INVALID_DIMS),  # 3 * 2^k in 3D
    ((64, 64, 1), (5000, 64, 1), (5000, 64, 1), (5000, 64, 1), C.ERR_INVALID_DIMS),  # other length above 4096
    ((64, 64, 1), (4097, 4097, 1), (4097, 4097, 1), (4097, 4097, 1), C.ERR_INVALID_DIMS),
    ((8, 8, 1), (12, 12, 1), (12, 12, 1), (12, 12, 1), C.ERR_INVALID_DIMS),  # other length below 17
    ((16, 16, 16), (600, 600, 600), (600, 600, 600), (600, 600, 600), C.ERR_INVALID_DIMS),  # 3D above 512
    ((64, 64, 1), (512, 512, 1), (512, 512, 1), (5000, 5000, 1), C.ERR_INVALID_DIMS),  # inverse grows, bad length
    ((64, 64, 64), (1024, 1024, 1024), (1024, 1024, 1024), (1024, 1024, 1024), C.ERR_INVALID_DIMS),  # 3D > 512
    ((64, 64, 1), (16384, 16384, 1), (16384, 16384, 1), (16384, 16384, 1), C.ERR_UNSUPPORTED),  # > 8192
    ((4, 4, 1), (8, 8, 1), (8, 8, 1), (8, 8, 1), C.ERR_UNSUPPORTED),  # < 16
])
def test_validation_rejects(fin, fout, iin, iout, status):
    ft = new(rank=3 if fout[2] > 1 else 2)
    ft.SetForwardFFTPlan(*fin, *fout)
    with pytest.raises(F.FastFFTError) as e:
        ft.SetInverseFFTPlan(*iin, *iout)
    assert e.value.status == status


@pytest.mark.parametrize("fin,fout,iout", [
    ((64, 64, 1), (384, 384, 1), (384, 384, 1)),
    ((1536, 1536, 1), (1536, 1536, 1), (700, 600, 1)),
    ((100, 200, 1), (768, 6144, 1), (768, 6144, 1)),
    ((1000, 10, 1), (3072, 32, 1), (3000, 20, 1)),
    ((64, 64, 1), (640, 640, 1), (640, 640, 1)),
    ((100, 200, 1), (1280, 5120, 1), (1280, 5120, 1)),
    ((1000, 10, 1), (2560, 32, 1), (2000, 20, 1)),
    ((64, 64, 1), (896, 896, 1), (896, 896, 1)),
    ((100, 200, 1), (1792, 3584, 1), (1792, 3584, 1)),
    # any other length in [17, 4096] (chirp-z transforms)
    ((100, 100, 1), (100, 100, 1), (100, 100, 1)),
    ((64, 64, 1), (320, 448, 1), (320, 448, 1)),
    ((64, 64, 1), (192, 192, 1), (192, 192, 1)),
    ((77, 53, 1), (999, 1001, 1), (700, 600, 1)),
    ((17, 4095, 1), (17, 4095, 1), (17, 4095, 1)),
])
def test_three_times_power_of_two_lengths_accepted_in_2d(fin, fout, iout):
    ft = new()
    ft.SetForwardFFTPlan(*fin, *fout)
    ft.SetInverseFFTPlan(*fout, *iout)
    assert ft.ReturnFwdOutputDimensions()[:3] == fout


def test_rank_mismatch_rejected():
    ft = new(rank=3)
    ft.SetForwardFFTPlan(64, 64, 1, 128, 128, 1)
    with pytest.raises(F.FastFFTError) as e:
        ft.SetInverseFFTPlan(128, 128, 1, 128, 128, 1)
    assert e.value.status == C.ERR_INVALID_DIMS


def test_transform_before_plan_is_an_error():
    ft = new()
    with pytest.raises(F.FastFFTError) as e:
        ft.FwdFFT(0x1000)
    assert e.value.status in (C.ERR_INVALID_ARGUMENT, C.ERR_NOT_PLANNED)


def test_bad_dtypes_and_zero_dims():
    h = C.Handle()
    assert C.lib().fastfft_create(ctypes.byref(h), 0, 9, C.DTYPE_C64, 2) == C.ERR_UNSUPPORTED      # no such dtype
    assert C.lib().fastfft_create(ctypes.byref(h), 0, C.DTYPE_F32, C.DTYPE_F32, 2) == C.ERR_UNSUPPORTED  # real image
    assert C.lib().fastfft_create(ctypes.byref(h), 1, C.DTYPE_F32, C.DTYPE_C64, 2) == C.ERR_UNSUPPORTED  # compute
    ft = new()
    with pytest.raises(F.FastFFTError) as e:
        ft.SetForwardFFTPlan(0, 64, 1, 64, 64, 1)
    assert e.value.status == C.ERR_INVALID_DIMS
    with pytest.raises(F.FastFFTError) as e:
        ft.SetForwardFFTPlan(64, 64, 1, 64, 64, 1, is_padded_output=False)
    assert e.value.status == C.ERR_UNSUPPORTED


def test_null_handle_calls_fail_cleanly():
    lib = C.lib()
    assert lib.fastfft_set_stream(None, None) == C.ERR_INVALID_ARGUMENT
    assert lib.fastfft_wait(None) == C.ERR_INVALID_ARGUMENT
    assert lib.fastfft_destroy(None) == C.OK
    assert lib.fastfft_last_error(None) != b""


def test_spectrum_output_setting_is_validated():
    ft = new()
    ft.SetSpectrumOutput("complex32", 1.0 / 4096)
    ft.SetSpectrumOutput("complex_bf16", 0.5)
    ft.SetSpectrumOutput("complex64")
    lib = C.lib()
    assert lib.fastfft_set_spectrum_output(ft._h, C.DTYPE_F32, 1.0) == C.ERR_INVALID_ARGUMENT   # real
    assert lib.fastfft_set_spectrum_output(ft._h, C.DTYPE_C32H, 0.0) == C.ERR_INVALID_ARGUMENT   # zero
    assert lib.fastfft_set_spectrum_output(ft._h, C.DTYPE_C32H, float("nan")) == C.ERR_INVALID_ARGUMENT
    assert lib.fastfft_set_spectrum_output(None, C.DTYPE_C64, 1.0) == C.ERR_INVALID_ARGUMENT


def test_radial_operations_validate_arguments():
    ft = new()
    lib = C.lib()
    assert lib.fastfft_radial_power(None, 0x1000, 64, 0x2000, 10) == C.ERR_INVALID_ARGUMENT
    assert lib.fastfft_radial_power(ft._h, None, 64, 0x2000, 10) == C.ERR_INVALID_ARGUMENT
    assert lib.fastfft_radial_power(ft._h, 0x1000, 63, 0x2000, 10) == C.ERR_INVALID_DIMS      # odd n
    assert lib.fastfft_radial_power(ft._h, 0x1000, 64, 0x2000, 0) == C.ERR_INVALID_ARGUMENT   # no bins
    assert lib.fastfft_apply_radial_filter(ft._h, 0x1000, None, 64, 0x2000, 10) == C.ERR_INVALID_ARGUMENT
    assert lib.fastfft_apply_radial_filter(ft._h, 0x1000, 0x3000, 16384, 0x2000, 10) == C.ERR_INVALID_DIMS
    ft.SetSpectrumOutput("complex32", 1.0)
    # in place needs complex64 storage
    assert lib.fastfft_apply_radial_filter(ft._h, 0x1000, 0x1000, 64, 0x2000, 10) == C.ERR_INVALID_ARGUMENT


@pytest.mark.parametrize("fin,fout,iout", [
    ((64, 64, 1), (512, 512, 1), (512, 512, 1)),
    ((384, 200, 1), (4096, 2048, 1), (1000, 999, 1)),
    ((64, 64, 64), (256, 256, 256), (128, 128, 128)),
])
def test_complex_input_memory_sizes(fin, fout, iout):
    """Complex InputType: 2 x y z scalar components, w = x (include/FastFFT.h:381-384)."""
    ft = new(rank=3 if fout[2] > 1 else 2, input_dtype="complex64")
    ft.SetForwardFFTPlan(*fin, *fout)
    ft.SetInverseFFTPlan(*fout, *iout)
    assert ft.ReturnInputMemorySize() == O.complex_memory_size(fin)
    assert ft.ReturnFwdOutputMemorySize() == O.complex_memory_size(fout)
    assert ft.ReturnInvOutputMemorySize() == O.complex_memory_size(iout)
    assert ft.ReturnFwdInputDimensions() == (*fin, fin[0])
    assert ft.ReturnFwdOutputDimensions() == (*fout, fout[0])


def test_complex_input_rules():
    ft = new(input_dtype="complex64")
    with pytest.raises(ValueError):
        ft.SetOutputDtype("float32")            # complex-input plans write complex output
    assert C.lib().fastfft_set_output_dtype(ft._h, C.DTYPE_F32) == C.ERR_INVALID_ARGUMENT
    ft.SetOutputDtype("complex_bf16")
    ft.SetForwardFFTPlan(64, 64, 1, 384, 384, 1)
    with pytest.raises(C.FastFFTError):           # 3 * 2^k lengths are real-input only
        ft.SetInverseFFTPlan(384, 384, 1, 384, 384, 1)
    real = new()
    with pytest.raises(ValueError):
        real.SetOutputDtype("complex64")
    assert C.lib().fastfft_set_output_dtype(real._h, C.DTYPE_C64) == C.ERR_INVALID_ARGUMENT


def test_chirp_z_lengths_complex_and_3d():
    """Complex-input and 3D plans take any length in [17, 4096] (chirp-z; 3D within 512)
    besides powers of two; 3 * 2^k stays rejected there."""
    for fin, fout, iout, rank, dt in (((77, 53, 1), (999, 1001, 1), (700, 600, 1), 2, "complex64"),
                                      ((16, 16, 16), (100, 60, 50), (100, 60, 50), 3, "float32"),
                                      ((16, 16, 16), (100, 60, 50), (30, 20, 10), 3, "complex64"),
                                      ((16, 16, 16), (320, 448, 64), (320, 448, 64), 3, "float32")):
        ft = new(rank=rank, input_dtype=dt)
        ft.SetForwardFFTPlan(*fin, *fout)
        ft.SetInverseFFTPlan(*fout, *iout)
        assert ft.ReturnFwdOutputDimensions()[:3] == fout
    for fout, rank in (((384, 384, 1), 2), ((384, 384, 384), 3)):
        ft = new(rank=rank, input_dtype="complex64")
        ft.SetForwardFFTPlan(16, 16, fout[2] if rank == 3 else 1, *fout)
        with pytest.raises(F.FastFFTError) as e:
            ft.SetInverseFFTPlan(*fout, *fout)
        assert e.value.status == C.ERR_INVALID_DIMS
