"""The C-ABI library loads and exports every entry point include/*.h declares
(no compute calls: runs without a GPU)."""
import ctypes
import os
import re

import pytest

from helpers import ROOT


def declared_functions():
    names = set()
    for dp, _, fs in os.walk(os.path.join(ROOT, "include")):
        for f in fs:
            if f == "cudacompress_b200.h":
                text = open(os.path.join(dp, f)).read()
                names |= set(re.findall(r"\b(cc_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    from cudacompress_b200 import _ffi
    if not os.path.exists(_ffi.LIB_PATH):
        from cudacompress_b200 import build
        build.build(verbose=False)
    lib = ctypes.CDLL(_ffi.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    assert set(declared_functions()) == set(_ffi.exported_names())


def test_cxx_api_symbols_exported():
    """The C++ drop-in layer (namespace cudaCompress) is in the same library."""
    from cudacompress_b200 import _ffi
    import subprocess
    out = subprocess.run(["nm", "-DC", _ffi.LIB_PATH], capture_output=True, text=True).stdout
    for sym in ["cudaCompress::createInstance(int, unsigned int, unsigned int, unsigned int, unsigned int)",
                "cudaCompress::destroyInstance(cudaCompress::Instance*)",
                "cudaCompress::setInstanceCudaStream(cudaCompress::Instance*, CUstream_st*)",
                "cudaCompress::setInstanceStream(cudaCompress::Instance*, CUstream_st*)",
                "cudaCompress::encodeRLHuff(cudaCompress::Instance*, cudaCompress::BitStream&, unsigned short const* const*, unsigned int, unsigned int)",
                "cudaCompress::decodeHuff(cudaCompress::Instance*, cudaCompress::BitStreamReadOnly**, unsigned int**, unsigned int, unsigned int)",
                "cudaCompress::util::dwtFloat3DForward(float*, float*, float*, float const*, int, int, int, int, int, int, int, int, CUstream_st*)",
                "cudaCompress::util::quantizeToSymbols(unsigned short*, float const*, unsigned int, unsigned int, unsigned int, float, unsigned int, unsigned int, cudaCompress::util::EQuantizeType)"]:
        assert sym in out, sym


def test_product_fails_loudly_without_extension(monkeypatch):
    from cudacompress_b200 import _ffi
    monkeypatch.setattr(_ffi, "LIB_PATH", "/nonexistent/libcudacompress_b200.so")
    monkeypatch.setattr(_ffi, "_lib", None)
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        _ffi.lib()
