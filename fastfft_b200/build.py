"""Build libfastfft_b200.so in-tree for sm_100a with nvcc (no torch dependency).

Usage: python -m fastfft_b200.build [--jobs N] [--ptxas-verbose]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
OBJ = PKG / "_build"
LIB = PKG / "libfastfft_b200.so"
SOURCES = ["launch_fft7.cu", "launch_fft5.cu", "launch_fft3.cu", "twiddles.cu", "launch_rows.cu", "launch_cols.cu", "launch_xcorr.cu",
           "capi.cu", "noalloc.cu", "spectrum_ops.cu", "launch_tc.cu", "launch_blue.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
         "--expt-relaxed-constexpr"]


def _compile(src: str, extra: list[str], obj_dir: Path = OBJ) -> tuple[str, str]:
    out = obj_dir / (Path(src).stem + ".o")
    cmd = [NVCC, *ARCH, *FLAGS, *extra, "-c", str(CSRC / src), "-o", str(out)]
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{' '.join(cmd)}\n{p.stdout}\n{p.stderr}")
    return str(out), p.stdout + p.stderr


def _needs_build(extra: list[str]) -> bool:
    if not LIB.exists():
        return True
    lib_t = LIB.stat().st_mtime
    deps = list(CSRC.glob("*")) + [PKG.parent / "include" / "fastfft_capi.h", Path(__file__)]
    return any(d.stat().st_mtime > lib_t for d in deps if d.exists())


def build(jobs: int | None = None, ptxas_verbose: bool = False, force: bool = False,
          defines: list[str] | None = None, out: Path | None = None) -> Path:
    """Compile and link the library; `defines` (NAME=VALUE) and `out` build a variant elsewhere."""
    extra = ["-Xptxas", "-v"] if ptxas_verbose else []
    extra += [f"-D{d}" for d in (defines or [])]
    lib = Path(out) if out else LIB
    if not force and not ptxas_verbose and not defines and out is None and not _needs_build(extra):
        return LIB
    obj_dir = OBJ if out is None else Path(out).parent / "_obj"
    obj_dir.mkdir(parents=True, exist_ok=True)
    jobs = jobs or min(len(SOURCES), os.cpu_count() or 1)
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        results = list(ex.map(lambda s: _compile(s, extra, obj_dir), SOURCES))
    if ptxas_verbose:
        for _, log in results:
            sys.stderr.write(log)
    objs = [r[0] for r in results]
    tmp = lib.with_suffix(".so.tmp")
    cmd = [NVCC, *ARCH, "-shared", "-Xcompiler", "-fPIC", *objs, "-o", str(tmp), "-lcudart"]
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        raise RuntimeError(f"link failed:\n{' '.join(cmd)}\n{p.stdout}\n{p.stderr}")
    os.replace(tmp, lib)
    return lib


COMPARATOR = CSRC / "comparator"
BIN = PKG / "bin"


def build_comparator(force: bool = False) -> Path | None:
    """The cuFFT comparator of bench.py (not part of the library): a standalone program running
    the reference's cuFFT recipe with a load callback, which needs the static cuFFT library (the
    program is about 290 MB, so it is built where it runs, in a few seconds, and kept out of the
    repository).  Returns its path, or None when the toolkit has no static cuFFT."""
    cuda = Path(NVCC).resolve().parent.parent
    if not (cuda / "lib64" / "libcufft_static.a").exists():
        return None
    BIN.mkdir(exist_ok=True)
    exe = BIN / "cufft_recipe_bench"
    src = COMPARATOR / "cufft_recipe_bench.cu"
    if not force and exe.exists() and src.stat().st_mtime < exe.stat().st_mtime:
        return exe
    cmd = [NVCC, *ARCH, "-O3", "-std=c++17", "-rdc=true", str(src), "-o", str(exe), "-lcufft_static", "-lculibos"]
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        raise RuntimeError(f"nvcc failed:\n{' '.join(cmd)}\n{p.stdout}\n{p.stderr}")
    return exe


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("--ptxas-verbose", action="store_true")
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--define", action="append", default=[], help="NAME=VALUE preprocessor define")
    ap.add_argument("--out", default=None, help="write the library here instead of in-tree")
    a = ap.parse_args()
    print(build(a.jobs, a.ptxas_verbose, a.force, a.define, a.out))
