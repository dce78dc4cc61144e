"""Builds the CUDA library in-tree:

  cudacompress_b200/_lib/libcudacompress_b200.so   product library (C ABI + C++ API)
  cudacompress_b200/_lib/libcc_selftest.so         host build of the table builder (tests)

Usage: python -m cudacompress_b200.build [--force]
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "_lib")
OBJ = os.path.join(HERE, "_build")

CUDA_SOURCES = ["instance.cu", "encode.cu", "decode.cu", "dwt.cu", "quantize.cu", "image.cu", "pipeline.cu", "batch.cu",
                "cuda_timer.cu",
                "container.cu", "cxx_api.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", 
              "--expt-relaxed-constexpr", "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]

LIB_NAME = "libcudacompress_b200.so"


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def host_cxx() -> str:
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else (shutil.which("g++") or "g++")


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps)


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    inc = os.path.join(ROOT, "include")
    for dp, _, fs in os.walk(inc):
        hs += [os.path.join(dp, f) for f in fs if f.endswith(".h")]
    return hs


def _compile(src: str, force: bool) -> str:
    obj = os.path.join(OBJ, os.path.splitext(src)[0] + ".o")
    srcp = os.path.join(CSRC, src)
    if not force and _newer(obj, [srcp] + _headers()):
        return obj
    cmd = [nvcc()] + ARCH + NVCC_FLAGS + ["-x", "cu", "-c", srcp, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj


def build(force: bool = False, verbose: bool = True) -> str:
    os.makedirs(LIB, exist_ok=True)
    os.makedirs(OBJ, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: _compile(s, force), CUDA_SOURCES))
    out = os.path.join(LIB, LIB_NAME)
    if force or not _newer(out, objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-Xcompiler", "-fPIC", "-o", out] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    st = os.path.join(LIB, "libcc_selftest.so")
    st_src = os.path.join(CSRC, "selftest_host.cpp")
    if force or not _newer(st, [st_src] + _headers()):
        cmd = [host_cxx(), "-O2", "-std=c++17", "-fPIC", "-shared", "-I/usr/local/cuda/include", "-x", "c++",
               st_src, "-o", st]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"self-test build failed:\n{r.stderr}")
    if verbose:
        print(f"built {out}")
    return out


if __name__ == "__main__":
    build(force="--force" in sys.argv)
