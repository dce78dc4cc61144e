"""Failure handling, with no GPU fault: allocation failures injected on the
host (cc_inject_allocation_failures makes chosen device / page-locked
allocations report out-of-memory without allocating), a real out-of-memory
at instance creation, and calls beyond an instance's capacity.  Every entry
point returns a status, releases what it holds, and the next call works."""
import ctypes

import numpy as np
import pytest

from helpers import Oracle, symbol_streams

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

import cudacompress_b200 as cc  # noqa: E402
from cudacompress_b200 import _ffi, fields  # noqa: E402

CC_ERR_OUT_OF_MEMORY = -3
CC_ERR_CAPACITY = -7


@pytest.fixture(autouse=True)
def injection_off():
    yield
    _ffi.lib().cc_inject_allocation_failures(0, 0)


def create(streams=7, elems=4096):
    h = ctypes.c_void_p()
    rc = _ffi.lib().cc_create_instance(ctypes.byref(h), 0, streams, elems, 128, 14)
    return rc, h


def test_instance_creation_survives_every_failed_allocation():
    """Instance creation makes one device and several page-locked
    allocations; failing each in turn returns out-of-memory with no handle."""
    lib = _ffi.lib()
    failures = 0
    for skip in range(16):
        lib.cc_inject_allocation_failures(skip, 1)
        rc, h = create()
        if rc == 0:              # fewer allocations than `skip`: nothing failed
            lib.cc_destroy_instance(h)
            lib.cc_inject_allocation_failures(0, 0)
            break
        failures += 1
        assert rc == CC_ERR_OUT_OF_MEMORY and not h.value, (skip, rc)
        assert b"cudaMalloc" in lib.cc_last_error() or b"cudaHostAlloc" in lib.cc_last_error()
    assert failures >= 2
    rc, h = create()
    assert rc == 0 and h.value
    lib.cc_destroy_instance(h)


def test_real_out_of_memory_at_creation():
    """An arena larger than the device: cudaMalloc itself fails."""
    rc, h = create(streams=64, elems=1 << 30)
    assert rc == CC_ERR_OUT_OF_MEMORY and not h.value
    rc, h = create()
    assert rc == 0
    _ffi.lib().cc_destroy_instance(h)


def test_volume_batch_creation_survives_every_failed_allocation():
    """A batch creates two instances of its own, a work area and page-locked
    tables; failing each allocation in turn returns an error, and a batch
    made afterwards still codes exactly like the oracle."""
    lib = _ffi.lib()
    vol = fields.turbulence_field(32, 128, 8, seed=71)
    with cc.Instance(0, 7, 16 ** 3, 128, 14) as inst:
        failures = 0
        for skip in range(40):
            lib.cc_inject_allocation_failures(skip, 1)
            try:
                b = cc.VolumeBatch(inst, [vol.shape, (16, 24, 32)], 2, [0.01, 0.02], graph=True)
            except cc.CudaCompressError as e:
                failures += 1
                assert "memory" in str(e).lower() or "cudaMalloc" in str(e) or "cudaHostAlloc" in str(e)
                continue
            b.close()
            lib.cc_inject_allocation_failures(0, 0)
            break
        assert failures >= 4
        with cc.VolumeBatch(inst, [vol.shape], 2, [0.01], graph=True) as b:
            d = torch.from_numpy(vol).cuda()
            b.compress([d])
            words, bits = b.read_stream(0)
        ref_words, ref_bits = Oracle().compress_volume(vol, 2, 0.01)
        assert bits == ref_bits and np.array_equal(words, ref_words)


def test_pipeline_workspace_failure_then_recovery():
    """The plain volume codec allocates its work memory on first use: a
    failed allocation there raises, and the next call allocates and codes
    correctly."""
    lib = _ffi.lib()
    vol = fields.turbulence_field(32, 128, 8, seed=72)
    d = torch.from_numpy(vol).cuda()
    with cc.Instance(0, 7, 16 ** 3, 128, 14) as inst:
        lib.cc_inject_allocation_failures(0, 1)
        with pytest.raises(cc.CudaCompressError):
            cc.compress_volume_float(inst, d, 2, 0.01)
        lib.cc_inject_allocation_failures(0, 0)
        words, bits = cc.compress_volume_float(inst, d, 2, 0.01)
        torch.cuda.synchronize()
        ref_words, ref_bits = Oracle().compress_volume(vol, 2, 0.01)
        assert bits == ref_bits
        assert np.array_equal(words[: (bits + 31) // 32].cpu().numpy().view(np.uint32), ref_words)


def test_calls_beyond_instance_capacity_fail_cleanly():
    """More streams or longer streams than the instance was made for: the
    call returns false (CC_ERR_CAPACITY); a call within capacity still
    matches the oracle."""
    lib = _ffi.lib()
    oracle = Oracle()
    with cc.Instance(0, 2, 1000, 128, 14) as inst:
        three = [torch.from_numpy(s).cuda() for s in symbol_streams("laplace", 3, 1000, seed=5)]
        assert not cc.encode_rlhuff(inst, cc.BitStream(), three, 1000)
        assert b"capacity" in lib.cc_last_error().lower() or b"exceeds" in lib.cc_last_error().lower()
        long_ = [torch.from_numpy(s).cuda() for s in symbol_streams("laplace", 2, 3000, seed=6)]
        assert not cc.encode_rlhuff(inst, cc.BitStream(), long_, 3000)
        ok_streams = symbol_streams("laplace", 2, 1000, seed=7)
        bs = cc.BitStream()
        assert cc.encode_rlhuff(inst, bs, [torch.from_numpy(s).cuda() for s in ok_streams], 1000), cc.last_error()
        ref_words, ref_bits, _ = oracle.encode(0, ok_streams)
        assert bs.bit_size == ref_bits and np.array_equal(bs.raw(), ref_words)
        # decoding more streams than the instance holds fails the same way
        outs = [torch.zeros(1000, dtype=torch.int16, device="cuda") for _ in range(3)]
        assert not cc.decode_rlhuff(inst, cc.BitStream(ref_words, ref_bits), outs, 1000)
