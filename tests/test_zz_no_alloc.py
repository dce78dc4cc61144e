"""cc_dwt_float_forward_static (forward float DWT with the library's fixed
device scratch, for callers that cannot allocate device memory) against
cc_dwt_float_forward with caller buffers, through the C ABI, on two calls in
a row.  Collected last so it also runs after every other test."""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from cudacompress_b200 import _ffi  # noqa: E402


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def _reference(lib, src, sx, sy, sz):
    dst = torch.empty(sz * sy * sx, dtype=torch.float32, device="cuda")
    b1 = torch.empty_like(dst)
    b2 = torch.empty_like(dst)
    _ffi.check(lib.cc_dwt_float_forward(_p(dst), _p(b2), _p(b1), _p(src), sx, sy, sz, 1, 0, 0, 0, 0, None),
               "cc_dwt_float_forward")
    return dst


@pytest.mark.parametrize("shape", [(64, 48, 32), (128, 128, 64), (256, 128, 1)])
def test_static_scratch_matches_buffered_forward(shape):
    lib = _ffi.lib()
    sx, sy, sz = shape
    g = torch.Generator().manual_seed(1234 + sx + sy + sz)
    # two different inputs in a row: the second call must not see the first's scratch
    for k in range(2):
        src = (torch.randn(sz * sy * sx, generator=g) * (10.0 ** k)).cuda()
        want = _reference(lib, src, sx, sy, sz)
        got = torch.full_like(want, float("nan"))
        _ffi.check(lib.cc_dwt_float_forward_static(_p(got), _p(src), sx, sy, sz, 1, 0, 0, 0, 0, None),
                   "cc_dwt_float_forward_static")
        torch.cuda.synchronize()
        # same kernels, same arithmetic: bit-identical (tolerance 0)
        assert torch.equal(got.view(torch.int32), want.view(torch.int32)), (shape, k)


def test_static_scratch_rejects_oversize():
    lib = _ffi.lib()
    src = torch.zeros(8, dtype=torch.float32, device="cuda")
    rc = lib.cc_dwt_float_forward_static(_p(src), _p(src), 256, 256, 32, 1, 0, 0, 0, 0, None)
    assert rc != 0
    assert b"fixed scratch" in lib.cc_last_error()
