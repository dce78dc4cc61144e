"""Stream container (cc_container_*): round trips, the documented header
fields, and rejection of truncated or foreign data.  Host code only."""
import struct

import numpy as np
import pytest

from cudacompress_b200 import container as ct


def streams(seed, n):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        bits = int(rng.integers(0, 5000))
        w = rng.integers(0, 2 ** 32, (bits + 31) // 32, dtype=np.uint64).astype(np.uint32)
        shape = tuple(int(v) for v in rng.choice([16, 24, 32, 64], 3))
        out.append(ct.Stream(shape, float(rng.uniform(0.001, 0.1)), bits, w))
    return out


def test_round_trip(tmp_path):
    info = ct.ContainerInfo(ct.QUANT_FIRST, 1, 2, 64, 16)
    ss = streams(1, 9)
    p = tmp_path / "a.ccb"
    ct.save(str(p), info, ss)
    info2, ss2 = ct.load(str(p))
    assert info2 == info
    assert len(ss2) == len(ss)
    for a, b in zip(ss, ss2):
        assert a.shape == b.shape and a.bit_size == b.bit_size and np.float32(a.quant_step) == np.float32(b.quant_step)
        assert np.array_equal(a.words, b.words)


def test_header_layout():
    data = ct.pack(ct.ContainerInfo(ct.FLOAT, 0, 3, 128, 14), streams(2, 3))
    magic, version, codec, flags, levels, cb, l2, n, total = struct.unpack_from("<8IQ", data, 0)
    assert (magic, version, codec, flags, levels, cb, l2, n, total) == (0x32424343, 1, 0, 0, 3, 128, 14, 3, len(data))
    x, y, z, q, bits, off = struct.unpack_from("<3IfQQ", data, 48)
    assert off % 8 == 0 and off >= 48 + 3 * 32


def test_empty_and_rejects():
    data = ct.pack(ct.ContainerInfo(), [])
    info, ss = ct.unpack(data)
    assert ss == []
    full = ct.pack(ct.ContainerInfo(), streams(3, 4))
    with pytest.raises(Exception):
        ct.unpack(full[:-8])                 # truncated
    with pytest.raises(Exception):
        ct.unpack(b"RAWWORDS" + full[8:])    # foreign data
