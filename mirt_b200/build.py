"""Build libmirt_b200.so in-tree with nvcc for sm_100a.

    python -m mirt_b200.build [-v]

Each source under mirt_b200/csrc is compiled to an object in
mirt_b200/_build (skipped when up to date), then linked into
mirt_b200/libmirt_b200.so against cuFFT.  The CUDA runtime is linked
statically, so the library only needs libcufft.so.11 at run time.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libmirt_b200.so")
ROOT = os.path.dirname(PKG)

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler",
           "-fPIC,-O3,-Wall,-Wextra,-Wshadow,-Wpointer-arith",
           "--expt-relaxed-constexpr", "-I" + os.path.join(ROOT, "include")]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _cuda_lib() -> str:
    nv = os.path.realpath(_nvcc())
    return os.path.join(os.path.dirname(os.path.dirname(nv)), "lib64")


def sources() -> list[str]:
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC)
                  if f.endswith((".cu", ".cpp")))


def _deps() -> list[str]:
    hdr = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    return hdr + [os.path.join(ROOT, "include", "mirt_b200.h")]


def _compile(src: str, verbose: bool) -> str:
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    newest_dep = max(os.path.getmtime(p) for p in _deps() + [src])
    if os.path.exists(obj) and os.path.getmtime(obj) >= newest_dep:
        return obj
    cmd = [_nvcc(), *ARCH, *NVFLAGS, "-c", src, "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    out = subprocess.run(cmd, capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{out.stderr}")
    if verbose and out.stderr:
        sys.stderr.write(out.stderr)
    return obj


def build(verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    srcs = sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(o) for o in objs):
        return LIB
    libdir = _cuda_lib()
    cmd = [_nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-L" + libdir, "-lcufft",
           "-Xlinker", "-rpath=" + libdir, "-cudart", "static"]
    out = subprocess.run(cmd, capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("link failed:\n" + out.stderr)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
