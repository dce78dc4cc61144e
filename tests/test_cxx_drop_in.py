"""A C++ program written against the reference's API headers only
(tests/cxx/drop_in.cpp) compiles against include/cudaCompress/ and links
against the library with no other symbol (CPU); on a GPU it runs and every
check in it holds."""
import os
import shutil
import subprocess

import pytest

from helpers import ROOT

SRC = os.path.join(ROOT, "tests", "cxx", "drop_in.cpp")
LIB_DIR = os.path.join(ROOT, "cudacompress_b200", "_lib")
CUDA = "/usr/local/cuda"


def build(out_dir):
    if not os.path.exists(os.path.join(LIB_DIR, "libcudacompress_b200.so")):
        from cudacompress_b200 import build as b
        b.build(verbose=False)
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else shutil.which("g++")
    exe = os.path.join(out_dir, "drop_in")
    cmd = [cxx, "-std=c++17", "-O1", "-I" + os.path.join(ROOT, "include"), "-I" + CUDA + "/include", SRC, "-o", exe,
           "-L" + LIB_DIR, "-lcudacompress_b200", "-Wl,-rpath," + LIB_DIR, "-L" + CUDA + "/lib64", "-lcudart",
           "-Wl,--no-undefined"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]
    return exe


def test_drop_in_program_builds(tmp_path):
    assert os.path.exists(build(str(tmp_path)))


@pytest.mark.gpu
def test_drop_in_program_runs(tmp_path):
    exe = build(str(tmp_path))
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "DROPIN OK" in r.stdout, r.stdout + r.stderr
