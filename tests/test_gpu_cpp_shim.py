"""The C++ drop-in header runs the reference's transforms on the GPU.

A small C++ caller (tests/cpp/shim_transforms.cpp), compiled against include/FastFFT.h as
INTEGRATION.md shows, runs FwdFFT / InvFFT (64^2 -> 512^2 -> 512^2, pre-op SCALE) and
FwdImageInvFFT (384^2 -> 4096^2 -> 1024^2 against the spectrum its own FwdFFT made of a
4096^2 image) on the default stream; the results are checked against the FP64 oracle.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

from oracle import fastfft_oracle as O
from tests._util import RTOL_L2_FP32, RTOL_MAX_FP32

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA_HOME = "/usr/local/cuda"


@pytest.mark.gpu
@pytest.mark.skipif(shutil.which("g++") is None or not os.path.isdir(CUDA_HOME + "/include"),
                    reason="needs g++ and the CUDA toolkit")
def test_cpp_shim_transforms(torch_cuda, tmp_path):
    exe = tmp_path / "shim_transforms"
    lib_dir = os.path.join(ROOT, "fastfft_b200")
    subprocess.run(["g++", "-std=c++17", "-O1", f"-I{ROOT}/include", f"-I{CUDA_HOME}/include",
                    os.path.join(ROOT, "tests", "cpp", "shim_transforms.cpp"), f"-L{lib_dir}", "-lfastfft_b200",
                    f"-L{CUDA_HOME}/lib64", "-lcudart", f"-Wl,-rpath,{lib_dir}", f"-Wl,-rpath,{CUDA_HOME}/lib64",
                    "-o", str(exe)], check=True, capture_output=True, text=True)

    rng = np.random.default_rng(O.SEED_BASE + 1)
    x1 = rng.standard_normal((64, 64))
    in1 = O.real_to_padded(x1, (64, 64, 1))
    in1.tofile(tmp_path / "cfg1_in.f32")
    img = O.gaussian_blob_image(4096)
    tpl = O.normal_template(384, O.SEED_BASE + 12)
    O.real_to_padded(img, (4096, 4096, 1)).tofile(tmp_path / "cfg2_image.f32")
    t_pad = O.real_to_padded(tpl, (384, 384, 1))
    t_pad.tofile(tmp_path / "cfg2_template.f32")

    r = subprocess.run([str(exe), str(tmp_path)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == "ok"

    # cfg1: spectrum [kx][ky] and the unnormalised round trip
    spec_ref = O.fwd(in1, (64, 64, 1), (512, 512, 1), pre_op=(O.OP_SCALE, 0.5))
    spec = np.fromfile(tmp_path / "cfg1_spec.f32", dtype=np.float32).view(np.complex64).reshape(spec_ref.shape)
    assert O.rel_l2(spec, spec_ref) < RTOL_L2_FP32
    assert O.rel_max(spec, spec_ref) < RTOL_MAX_FP32
    out_ref = O.real_from_padded(O.inv(spec_ref, (512, 512, 1), (512, 512, 1), out_dtype=np.float64), (512, 512, 1))
    out = O.real_from_padded(np.fromfile(tmp_path / "cfg1_out.f32", dtype=np.float32), (512, 512, 1))
    assert O.rel_l2(out, out_ref) < RTOL_L2_FP32
    assert O.rel_max(out, out_ref) < RTOL_MAX_FP32

    # cfg2: window against the FP64 correlation with the FP64 image spectrum; peak bit-exact
    img_spec = O.fwd(O.real_to_padded(img, (4096, 4096, 1), dtype=np.float64), (4096, 4096, 1), (4096, 4096, 1))
    plan = O.Plan((384, 384, 1), (4096, 4096, 1), (4096, 4096, 1), (1024, 1024, 1))
    ref = O.real_from_padded(O.fwd_image_inv(t_pad, img_spec, plan, out_dtype=np.float64), (1024, 1024, 1))
    got = O.real_from_padded(np.fromfile(tmp_path / "cfg2_window.f32", dtype=np.float32), (1024, 1024, 1))
    assert O.rel_l2(got, ref) < RTOL_L2_FP32
    assert O.rel_max(got, ref) < RTOL_MAX_FP32
    assert O.peak(got)[0] == O.peak(ref)[0]
