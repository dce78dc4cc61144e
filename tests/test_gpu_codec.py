"""GPU parity tests: every CUDA stage against the CPU oracle, bit exact.

Run on a B200 with `pytest -m gpu`.  Sizes are small enough for the oracle to
finish in seconds; full-size checks use round-trip properties
(test_gpu_pipeline.py)."""
import ctypes

import numpy as np
import pytest

from helpers import Oracle, symbol_streams

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

import cudacompress_b200 as cc  # noqa: E402


@pytest.fixture(scope="module")
def oracle():
    return Oracle()


@pytest.fixture(scope="module")
def inst():
    with cc.Instance(0, 8, 1 << 18, 128, 14) as i:
        yield i


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def bits_equal(a, b):
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    return a.shape == b.shape and np.array_equal(a.view(np.uint32), b.view(np.uint32))


# ------------------------------------------------------------------ quantize
@pytest.mark.parametrize("step", [0.01, 0.0025, 0.37])
def test_quantize_matches_oracle(oracle, step):
    rng = np.random.default_rng(3)
    a = (rng.standard_normal((8, 16, 24)) * 2).astype(np.float32)
    a[0, 0, :4] = [0.0, -0.0, step, -step]
    sym = torch.empty(a.shape, dtype=torch.int16, device="cuda")
    cc.quantize_to_symbols(sym, dev(a), 24, 16, 8, step)
    got = host(sym).view(np.uint16)
    assert np.array_equal(got, oracle.quantize(a, step))
    back = torch.empty(a.shape, dtype=torch.float32, device="cuda")
    cc.unquantize_from_symbols(back, sym, 24, 16, 8, step)
    assert bits_equal(host(back), oracle.unquantize(got, step))


@pytest.mark.parametrize("n", [1, 7, 1000, 1 << 20, (1 << 24) + 3])
def test_get_max_abs_matches_oracle(oracle, inst, n):
    """getMaxAbs (util/Quantize.cu:355-361): the largest magnitude, exact."""
    rng = np.random.default_rng(n)
    a = (rng.standard_normal(n) * 3).astype(np.float32)
    if n > 8:
        a[:4] = [np.float32(1e-40), -0.0, 0.0, -np.float32(1e-39)]
        a[n // 3] = -50.0          # the largest magnitude is negative
        a[n - 1] = 49.5
    out = torch.full((1,), -1.0, dtype=torch.float32, device="cuda")
    cc.get_max_abs(inst, dev(a), n, out)
    assert bits_equal(host(out), np.array([oracle.max_abs(a)], np.float32))
    # a second call on other data overwrites the result
    b = np.full(n, -0.25, np.float32)
    cc.get_max_abs(inst, dev(b), n, out)
    assert host(out)[0] == np.float32(0.25)


def test_symbolize_roundtrip():
    rng = np.random.default_rng(4)
    a = rng.integers(-3000, 3000, (4, 16, 32)).astype(np.int16)
    s = torch.empty(a.shape, dtype=torch.int16, device="cuda")
    cc.symbolize(s, dev(a), 32, 16, 4)
    su = host(s).view(np.uint16).astype(np.int64)
    v = a.astype(np.int64)
    assert np.array_equal(su, np.where(v >= 0, 2 * v, 2 * np.abs(v) - 1))
    back = torch.empty_like(s)
    cc.unsymbolize(back, s, 32, 16, 4)
    assert np.array_equal(host(back), a)


# ---------------------------------------------------------------------- DWT
@pytest.mark.parametrize("shape", [(16, 16, 16), (8, 24, 32), (32, 16, 8), (1, 40, 64), (1, 16, 520)])
def test_dwt_float_matches_oracle(oracle, shape):
    rng = np.random.default_rng(sum(shape))
    a = rng.standard_normal(shape).astype(np.float32)
    nz, ny, nx = shape
    src = dev(a)
    dst = torch.empty_like(src)
    b1 = torch.empty_like(src)
    b2 = torch.empty_like(src)
    cc.dwt_float_forward(dst, b2, b1, src, nx, ny, nz)
    fwd = host(dst)
    assert bits_equal(fwd, oracle.dwt_float(a))
    inv = torch.empty_like(src)
    cc.dwt_float_inverse(inv, b2, b1, dst, nx, ny, nz)
    assert bits_equal(host(inv), oracle.dwt_float(fwd, inverse=True))


def test_dwt_float_pitched_lowpass_level(oracle):
    """Second level of a multi-level transform: source = LLL corner of a
    larger array (pitches), as CompressVolume.cpp:341-347 calls it."""
    rng = np.random.default_rng(9)
    big = rng.standard_normal((32, 32, 32)).astype(np.float32)
    src = dev(big)
    dst = torch.empty((16, 16, 16), dtype=torch.float32, device="cuda")
    b1 = torch.empty_like(dst)
    b2 = torch.empty_like(dst)
    cc.dwt_float_forward(dst, b2, b1, src, 16, 16, 16, 1, 0, 0, 32, 32 * 32)
    assert bits_equal(host(dst), oracle.dwt_float(np.ascontiguousarray(big[:16, :16, :16])))


@pytest.mark.parametrize("shape", [(1, 64, 64), (1, 24, 40), (16, 16, 16), (8, 32, 24)])
def test_dwt_int_matches_oracle_and_is_lossless(oracle, shape):
    rng = np.random.default_rng(sum(shape) + 1)
    a = rng.integers(-2000, 8000, shape).astype(np.int16)
    nz, ny, nx = shape
    src = dev(a)
    dst = torch.empty_like(src)
    buf = torch.empty_like(src)
    cc.dwt_int_forward(dst, buf, src, nx, ny, nz)
    fwd = host(dst)
    assert np.array_equal(fwd, oracle.dwt_int(a))
    back = torch.empty_like(src)
    cc.dwt_int_inverse(back, buf, dst, nx, ny, nz)
    assert np.array_equal(host(back), a)


def test_dwt_int_narrowing_matches_oracle(oracle):
    """Values near the int16 limits exercise the reference's 16-bit wrap."""
    rng = np.random.default_rng(12)
    a = rng.integers(-32768, 32767, (1, 32, 32)).astype(np.int16)
    src = dev(a)
    dst = torch.empty_like(src)
    buf = torch.empty_like(src)
    cc.dwt_int_forward(dst, buf, src, 32, 32, 1)
    assert np.array_equal(host(dst), oracle.dwt_int(a))


# ------------------------------------------------------------ entropy coder
KINDS = ["sparse", "dense", "laplace", "runs", "zeros", "single"]


def encode_gpu(inst, kind, streams):
    S, n = streams.shape
    t = dev(streams.view(np.int16) if streams.dtype == np.uint16 else streams.view(np.int32))
    bs = cc.BitStream()
    fn = cc.encode_rlhuff if kind == 0 else cc.encode_huff
    ok = fn(inst, bs, [t[i] for i in range(S)], n)
    assert ok, cc.last_error()
    return bs


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("n", [1, 37, 4096, 100003])
def test_encode_rlhuff_byte_identical(oracle, inst, kind, n):
    streams = symbol_streams(kind, 5, n, seed=n)
    bs = encode_gpu(inst, 0, streams)
    ref = oracle.encode(0, streams)
    assert bs.bit_size == ref[1]
    assert np.array_equal(bs.raw(), ref[0])


@pytest.mark.parametrize("kind", ["dense", "laplace", "single", "sparse"])
@pytest.mark.parametrize("n", [1, 100, 65536 + 17])
def test_encode_huff_byte_identical(oracle, inst, kind, n):
    streams = symbol_streams(kind, 3, n, seed=n + 5)
    bs = encode_gpu(inst, 1, streams)
    ref = oracle.encode(1, streams)
    assert bs.bit_size == ref[1]
    assert np.array_equal(bs.raw(), ref[0])


def test_all_zero_call_matches_oracle(oracle):
    """Every stream empty after run-length coding: the reference's zero-count
    tables come from its arena layout (1 symbol for tables 0..2 of 7)."""
    with cc.Instance(0, 7, 4096, 128, 14) as inst7:
        streams = np.zeros((7, 4096), np.uint16)
        bs = encode_gpu(inst7, 0, streams)
        ref = oracle.encode(0, streams)
        assert np.array_equal(bs.raw(), ref[0])


@pytest.mark.parametrize("start_bits", [0, 5, 31, 64, 77])
def test_encode_huff_unaligned_start(oracle, inst, start_bits):
    """encodeHuff appends at the current bit position; earlier bits are kept."""
    streams = symbol_streams("laplace", 2, 3000, seed=start_bits)
    rng = np.random.default_rng(start_bits)
    prefix = rng.integers(0, 2 ** 32, (start_bits + 31) // 32 + 1, dtype=np.uint64).astype(np.uint32)
    bs = cc.BitStream(prefix, start_bits)
    bs.pos = start_bits
    t = dev(streams.view(np.int16))
    assert cc.encode_huff(inst, bs, [t[0], t[1]], 3000), cc.last_error()
    ref = oracle.encode(1, streams, start_words=prefix[: (start_bits + 31) // 32], start_bit_size=start_bits,
                        start_pos=start_bits)
    assert bs.bit_size == ref[1] and bs.pos == ref[2]
    assert np.array_equal(bs.raw(), ref[0])


@pytest.mark.parametrize("kind", KINDS)
def test_decode_rlhuff_roundtrip(oracle, inst, kind):
    n = 50000
    streams = symbol_streams(kind, 4, n, seed=77)
    ref_words, ref_bits, _ = oracle.encode(0, streams)
    bs = cc.BitStream(ref_words, ref_bits)
    # outputs hold garbage: the decoder writes every symbol (zeros included)
    outs = [torch.full((n,), -1, dtype=torch.int16, device="cuda") for _ in range(4)]
    assert cc.decode_rlhuff(inst, bs, outs, n), cc.last_error()
    assert cc.decode_status(inst) == 0, cc.last_error()
    for i in range(4):
        assert np.array_equal(host(outs[i]).view(np.uint16), streams[i])
    assert bs.pos == ref_bits


def test_decode_rlhuff_long_runs_into_garbage(oracle, inst):
    """Zero runs far longer than a coding block's shared-memory stage (the
    in-place fill path), an all-zero stream and trailing zeros, decoded into
    outputs full of garbage."""
    n = 1 << 18
    streams = np.zeros((3, n), np.uint16)
    streams[0, [5, 70000, 70001, 200000]] = [3, 9, 1, 4]      # runs of ~70k and ~130k zeros
    streams[2, ::4099] = 7                                      # runs of 4098 zeros
    ref_words, ref_bits, _ = oracle.encode(0, streams)
    bs = cc.BitStream(ref_words, ref_bits)
    outs = [torch.full((n,), -1, dtype=torch.int16, device="cuda") for _ in range(3)]
    assert cc.decode_rlhuff(inst, bs, outs, n), cc.last_error()
    assert cc.decode_status(inst) == 0, cc.last_error()
    for i in range(3):
        assert np.array_equal(host(outs[i]).view(np.uint16), streams[i]), i


@pytest.mark.parametrize("kind", ["dense", "laplace", "single"])
def test_decode_huff_roundtrip(oracle, inst, kind):
    n = 70001
    streams = symbol_streams(kind, 3, n, seed=78)
    ref_words, ref_bits, _ = oracle.encode(1, streams)
    bs = cc.BitStream(ref_words, ref_bits)
    outs = [torch.zeros(n, dtype=torch.int16, device="cuda") for _ in range(3)]
    assert cc.decode_huff(inst, bs, outs, n), cc.last_error()
    assert cc.decode_status(inst) == 0
    for i in range(3):
        assert np.array_equal(host(outs[i]).view(np.uint16), streams[i])


def fibonacci_stream(count, seed):
    """Symbols 1..count with Fibonacci counts (code lengths up to count - 1
    bits), shuffled."""
    fib = [1, 1]
    while len(fib) < count:
        fib.append(fib[-1] + fib[-2])
    s = np.repeat(np.arange(1, count + 1, dtype=np.uint16), fib)
    np.random.default_rng(seed).shuffle(s)
    return s


@pytest.mark.parametrize("kind", [0, 1])
def test_codes_longer_than_27_bits(oracle, kind):
    """Codewords of 28-29 bits (the packer keeps codes of up to 27 bits
    packed with their lengths and looks longer ones up again): streams,
    tables and the decode identical to the oracle's."""
    s = fibonacci_stream(30, seed=31 + kind)
    n = len(s)
    streams = np.stack([s, np.roll(s, 1000)])
    with cc.Instance(0, 2, n, 128, 14) as big:
        bs = encode_gpu(big, kind, streams)
        ref_words, ref_bits, _ = oracle.encode(kind, streams)
        assert bs.bit_size == ref_bits
        assert np.array_equal(bs.raw(), ref_words)
        outs = [torch.full((n,), -1, dtype=torch.int16, device="cuda") for _ in range(2)]
        dec = cc.decode_rlhuff if kind == 0 else cc.decode_huff
        assert dec(big, cc.BitStream(ref_words, ref_bits), outs, n), cc.last_error()
        assert cc.decode_status(big) == 0
        for i in range(2):
            assert np.array_equal(host(outs[i]).view(np.uint16), streams[i])


def test_tables_of_every_builder_tier(oracle):
    """One call of 40 streams (80 tables, so the tables are built by the
    leaf-count tiers) whose symbol tables have from a few to ~5800 leaves:
    warp builders (<= 256 leaves), 64-thread builders (<= 1024), 256-thread
    builders (<= 2048) and full-heap builders (more) in the same call.  Both
    encoders' streams identical to the oracle's; the decode round trips."""
    rng = np.random.default_rng(91)
    n, S = 20000, 40
    distinct = [8, 60, 200, 250, 400, 700, 1000, 1300, 1700, 2000, 3000, 6000]
    streams = np.zeros((S, n), np.uint16)
    for k in range(S):
        d = distinct[k % len(distinct)]
        v = rng.integers(1, d + 1, n)
        streams[k] = np.where(rng.random(n) < 0.2, 0, v)   # zero runs for the run-length tables
    with cc.Instance(0, S, n, 128, 14) as big:
        for kind in (0, 1):
            bs = encode_gpu(big, kind, streams)
            ref_words, ref_bits, _ = oracle.encode(kind, streams)
            assert bs.bit_size == ref_bits, kind
            assert np.array_equal(bs.raw(), ref_words), kind
            outs = [torch.full((n,), -1, dtype=torch.int16, device="cuda") for _ in range(S)]
            dec = cc.decode_rlhuff if kind == 0 else cc.decode_huff
            assert dec(big, cc.BitStream(ref_words, ref_bits), outs, n), cc.last_error()
            assert cc.decode_status(big) == 0
            for i in range(S):
                assert np.array_equal(host(outs[i]).view(np.uint16), streams[i]), (kind, i)


@pytest.mark.parametrize("cb", [32, 64, 256])
def test_coding_block_sizes(oracle, cb):
    with cc.Instance(0, 4, 40000, cb, 14) as inst_cb:
        streams = symbol_streams("laplace", 3, 40000, seed=cb)
        t = dev(streams.view(np.int16))
        bs = cc.BitStream()
        assert cc.encode_rlhuff(inst_cb, bs, [t[i] for i in range(3)], 40000)
        ref = oracle.encode(0, streams, cb=cb)
        assert np.array_equal(bs.raw(), ref[0])
        bs.pos = 0
        outs = [torch.zeros(40000, dtype=torch.int16, device="cuda") for _ in range(3)]
        assert cc.decode_rlhuff(inst_cb, bs, outs, 40000)
        for i in range(3):
            assert np.array_equal(host(outs[i]).view(np.uint16), streams[i])


def test_symbol32_streams(oracle):
    """Symbol32 coding with a 20-bit alphabet (longSymbols: 5-bit symbolBits)."""
    with cc.Instance(0, 3, 20000, 128, 20) as inst32:
        rng = np.random.default_rng(5)
        streams = (rng.integers(0, 1 << 19, (2, 20000)) * (rng.random((2, 20000)) < 0.3)).astype(np.uint32)
        t = dev(streams.view(np.int32))
        bs = cc.BitStream()
        assert cc.encode_rlhuff(inst32, bs, [t[0], t[1]], 20000), cc.last_error()
        ref = oracle.encode(0, streams, log2max=20)
        assert np.array_equal(bs.raw(), ref[0])
        bs.pos = 0
        outs = [torch.zeros(20000, dtype=torch.int32, device="cuda") for _ in range(2)]
        assert cc.decode_rlhuff(inst32, bs, outs, 20000)
        for i in range(2):
            assert np.array_equal(host(outs[i]).view(np.uint32), streams[i])


def test_symbol_out_of_range_fails(inst):
    """A symbol >= 2^log2Max makes the call fail (HuffmanTable.cu:411-419)."""
    a = np.zeros((1, 1000), np.uint16)
    a[0, 10] = 20000
    t = dev(a.view(np.int16))
    assert not cc.encode_huff(inst, cc.BitStream(), [t[0]], 1000)
    assert "range" in cc.last_error()


def test_corrupt_stream_is_rejected(oracle, inst):
    streams = symbol_streams("laplace", 1, 5000, seed=1)
    words, bits, _ = oracle.encode(0, streams)
    bad = words.copy()
    bad[0] = 0xFFFFFFFF          # compact count far beyond the symbol count
    bs = cc.BitStream(bad, bits)
    out = torch.zeros(5000, dtype=torch.int16, device="cuda")
    assert not cc.decode_rlhuff(inst, bs, [out], 5000)
    truncated = cc.BitStream(words[:3], 96)
    assert not cc.decode_rlhuff(inst, truncated, [out], 5000)
