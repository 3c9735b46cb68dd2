"""In-tree build of the CUDA library libmsgpu.so for sm_100a (B200)."""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
CSRC = os.path.join(PKG, "csrc")
OUT = os.path.join(HERE, "libmsgpu.so")
SOURCES = [os.path.join(CSRC, "msgpu.cu"), os.path.join(CSRC, "msgpu_io.cpp")]
DEPS = SOURCES + sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cuh")) + [
    os.path.join(os.path.dirname(PKG), "include", "msgpu.h")]

# -fmad=false: no contraction of a*b+c into FMA, so that every FP64 operation
# rounds like the reference build (which has no FMA contraction).
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17", "-fmad=false",
              "-Xcompiler", "-fPIC", "-shared"]
# bzip2 (the image has the shared library without its development symlink)
# and zlib for the compressed array files of msgpu_io.cpp
LIBS = ["-l:libbz2.so.1.0", "-lz"]


def nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def up_to_date() -> bool:
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    return all(os.path.getmtime(d) <= t for d in DEPS if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return OUT
    cmd = [nvcc(), *NVCC_FLAGS, "-o", OUT, *SOURCES, *LIBS]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    build(force=True, verbose=True)
