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


def _pair(lib, src, sx, sy, sz, ch, dst_row, dst_slice, src_row, src_slice):
    """(static result, buffered result) of one call with explicit pitches."""
    n = (sz - 1) * dst_slice + (sy - 1) * dst_row + sx if sz > 1 else (sy - 1) * dst_row + sx
    want = torch.full((n,), float("nan"), dtype=torch.float32, device="cuda")
    b1 = torch.empty_like(want)
    b2 = torch.empty_like(want)
    _ffi.check(lib.cc_dwt_float_forward(_p(want), _p(b2), _p(b1), _p(src), sx, sy, sz, ch, dst_row, dst_slice,
                                        src_row, src_slice, None), "cc_dwt_float_forward")
    got = torch.full_like(want, float("nan"))
    _ffi.check(lib.cc_dwt_float_forward_static(_p(got), _p(src), sx, sy, sz, ch, dst_row, dst_slice, src_row,
                                               src_slice, None), "cc_dwt_float_forward_static")
    torch.cuda.synchronize()
    return got, want


def _same_on(got, want, sx, sy, sz, dst_row, dst_slice):
    """Bit-identical on every element of the volume (padding is not written)."""
    idx = (torch.arange(sz, device="cuda")[:, None, None] * dst_slice
           + torch.arange(sy, device="cuda")[None, :, None] * dst_row
           + torch.arange(sx, device="cuda")[None, None, :]).reshape(-1)
    return torch.equal(got[idx].view(torch.int32), want[idx].view(torch.int32))


def test_static_scratch_interleaved_channels_and_padded_pitches():
    """A 3-channel interleaved source (channel 1) and a padded destination:
    bit-identical to the buffered transform with the same pitches."""
    lib = _ffi.lib()
    sx, sy, sz, ch = 64, 48, 32, 3
    g = torch.Generator().manual_seed(99)
    img = torch.randn(sz * sy * sx * ch, generator=g).cuda()
    src = img[1:]                                   # channel 1
    got, want = _pair(lib, src, sx, sy, sz, ch, 80, 80 * 56, sx * ch, sx * ch * sy)
    assert _same_on(got, want, sx, sy, sz, 80, 80 * 56)


def test_static_scratch_capacity_boundary():
    """An intermediate extent of exactly 2^20 floats is accepted (and equal
    to the buffered transform); 2^20 + 1 is rejected."""
    lib = _ffi.lib()
    sx, sy, row = 18, 8, 149794                     # (sy - 1) * row + sx = 2^20
    assert (sy - 1) * row + sx == 1 << 20
    src = torch.randn(sy * sx, generator=torch.Generator().manual_seed(5)).cuda()
    for _ in range(2):
        got, want = _pair(lib, src, sx, sy, 1, 1, row, 0, 0, 0)
        assert _same_on(got, want, sx, sy, 1, row, 0)
    sx, row = 12, 149795                            # (sy - 1) * row + sx = 2^20 + 1
    assert (sy - 1) * row + sx == (1 << 20) + 1
    out = torch.empty((sy - 1) * row + sx, dtype=torch.float32, device="cuda")
    rc = lib.cc_dwt_float_forward_static(_p(out), _p(src), sx, sy, 1, 1, row, 0, 0, 0, None)
    assert rc != 0 and b"fixed scratch" in lib.cc_last_error()


def test_static_scratch_rejects_oversize():
    lib = _ffi.lib()
    src = torch.zeros(8, dtype=torch.float32, device="cuda")
    rc = lib.cc_dwt_float_forward_static(_p(src), _p(src), 256, 256, 32, 1, 0, 0, 0, 0, None)
    assert rc != 0
    assert b"fixed scratch" in lib.cc_last_error()
