"""The C++ drop-in header compiles against the C ABI and its host logic works."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA_INC = "/usr/local/cuda/include"


@pytest.mark.skipif(shutil.which("g++") is None or not os.path.isdir(CUDA_INC), reason="needs g++ and CUDA headers")
def test_cpp_shim_plan_queries(tmp_path):
    exe = tmp_path / "shim_plan"
    lib_dir = os.path.join(ROOT, "fastfft_b200")
    cmd = ["g++", "-std=c++17", "-O1", f"-I{ROOT}/include", f"-I{CUDA_INC}",
           os.path.join(ROOT, "tests", "cpp", "shim_plan.cpp"), f"-L{lib_dir}", "-lfastfft_b200",
           f"-Wl,-rpath,{lib_dir}", "-o", str(exe)]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines()
    assert out[0].split() == ["148224", "16785408", "1050624", "4096", "4096", "1", "2049", "513"]
    assert out[1].startswith("rejected:") and "512" in out[1]
