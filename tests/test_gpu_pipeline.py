"""Whole-codec GPU tests: byte-identical streams against the oracle pipeline,
bit-exact reconstructions, lossless integer round trips."""
import numpy as np
import pytest

from helpers import Oracle

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

import cudacompress_b200 as cc  # noqa: E402
from cudacompress_b200 import fields  # noqa: E402


@pytest.fixture(scope="module")
def oracle():
    return Oracle()


def stream_of(words_t, bits):
    torch.cuda.synchronize()
    return words_t[: (bits + 31) // 32].cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("n,levels,q0", [(32, 2, 0.01), (64, 3, 0.01), (64, 2, 0.05), (48, 2, 0.002)])
def test_volume_codec_matches_oracle(oracle, n, levels, q0):
    vol = fields.turbulence_field(n, 256, n // 4, seed=2000 + n)
    with cc.Instance(0, 7, (n // 2) ** 3, 128, 14) as inst:
        words, bits = cc.compress_volume_float(inst, torch.from_numpy(vol).cuda(), levels, q0)
        got = stream_of(words, bits)
        ref_words, ref_bits = oracle.compress_volume(vol, levels, q0)
        assert bits == ref_bits
        assert np.array_equal(got, ref_words)
        out = torch.empty_like(torch.from_numpy(vol)).cuda()
        cc.decompress_volume_float(inst, out, levels, q0, words, bits)
        rec = out.cpu().numpy()
        ref_rec = oracle.decompress_volume(ref_words, ref_bits, vol.shape, levels, q0)
        assert np.array_equal(rec.view(np.uint32), ref_rec.view(np.uint32))
        assert fields.psnr(vol, rec) > 30


def test_plain_decode_reuses_its_batch_across_steps_and_sizes(oracle):
    """decompressVolumeFloat takes the level-by-level path for a shape's
    first four consecutive calls and a volume batch kept on the instance from
    the fifth (two kept, least recently used replaced): calls with other
    quantization steps (the batch's steps patched), a second shape, the first
    again, a third shape (evicting one), each bit-identical to the oracle's
    reconstruction of the oracle's stream."""
    a, b, c = ((32, 32, 32), 2), ((32, 48, 64), 2), ((32, 48, 64), 3)
    cases = ([a + (0.01,)] * 5 + [a + (0.05,), a + (0.002,)] + [b + (0.01,)] * 5 + [a + (0.01,)] +
             [c + (0.01,)] * 5 + [b + (0.05,), a + (0.05,)])
    with cc.Instance(0, 7, 32 ** 3, 128, 14) as inst:
        for shape, levels, q0 in cases:
            vol = np.ascontiguousarray(fields.turbulence_field(64, 256, 16, seed=2100)[: shape[0], : shape[1], : shape[2]])
            ref_words, ref_bits = oracle.compress_volume(vol, levels, q0)
            words = torch.from_numpy(ref_words.view(np.int32).copy()).cuda()
            out = torch.full(shape, float("nan"), dtype=torch.float32, device="cuda")
            cc.decompress_volume_float(inst, out, levels, q0, words, ref_bits)
            ref_rec = oracle.decompress_volume(ref_words, ref_bits, vol.shape, levels, q0)
            assert np.array_equal(out.cpu().numpy().view(np.uint32), ref_rec.view(np.uint32)), (shape, levels, q0)


def test_plain_calls_through_the_batch_report_their_sections(oracle):
    """With timing on, compress / decompress calls that run through the
    instance's volume batch fold the batch's sections into the instance's
    (cc_timing_*), and still match the oracle."""
    import ctypes
    from cudacompress_b200 import _ffi
    lib = _ffi.lib()
    vol = fields.turbulence_field(32, 128, 8, seed=2102)
    d = torch.from_numpy(vol).cuda()
    ref_words, ref_bits = oracle.compress_volume(vol, 2, 0.01)
    ref_rec = oracle.decompress_volume(ref_words, ref_bits, vol.shape, 2, 0.01)
    with cc.Instance(0, 7, 16 ** 3, 128, 14) as inst:
        for _ in range(3):   # the shape's batch comes on its fifth consecutive call
            w, b = cc.compress_volume_float(inst, d, 2, 0.01)
            out = torch.empty_like(d)
            cc.decompress_volume_float(inst, out, 2, 0.01, w, b)
        lib.cc_reset_timings(inst.handle)
        lib.cc_set_timing(inst.handle, 1)
        w, b = cc.compress_volume_float(inst, d, 2, 0.01)
        out = torch.full_like(d, float("nan"))
        cc.decompress_volume_float(inst, out, 2, 0.01, w, b)
        lib.cc_set_timing(inst.handle, 0)
        names = set()
        for i in range(lib.cc_timing_count(inst.handle)):
            name, ms, cnt = ctypes.c_char_p(), ctypes.c_double(), ctypes.c_uint32()
            lib.cc_timing_entry(inst.handle, i, ctypes.byref(name), ctypes.byref(ms), ctypes.byref(cnt))
            names.add(name.value.decode())
        assert "batch.dwt_forward" in names and "batch.dwt_inverse" in names, sorted(names)
        assert b == ref_bits and np.array_equal(stream_of(w, b), ref_words)
        assert np.array_equal(out.cpu().numpy().view(np.uint32), ref_rec.view(np.uint32))


def test_plain_decode_beyond_instance_capacity_fails_cleanly(oracle):
    """The instance's declared stream length bounds decompressVolumeFloat as
    it bounds the encoder: a volume whose level-0 bands exceed it fails with
    a capacity error and nothing is decoded."""
    vol = fields.turbulence_field(32, 128, 8, seed=2101)
    ref_words, ref_bits = oracle.compress_volume(vol, 2, 0.01)
    words = torch.from_numpy(ref_words.view(np.int32).copy()).cuda()
    with cc.Instance(0, 7, 15 ** 3, 128, 14) as inst:
        out = torch.zeros((32, 32, 32), dtype=torch.float32, device="cuda")
        with pytest.raises(cc.CudaCompressError):
            cc.decompress_volume_float(inst, out, 2, 0.01, words, ref_bits)


def test_volume_codec_c0_full_size(oracle):
    """128^3, 3 levels, q0 = 0.01 (the small lossy volume config)."""
    vol = fields.turbulence_field(128, 512, 32, fields.SEED_C0)
    with cc.Instance(0, 7, 64 ** 3, 128, 14) as inst:
        words, bits = cc.compress_volume_float(inst, torch.from_numpy(vol).cuda(), 3, 0.01)
        ref_words, ref_bits = oracle.compress_volume(vol, 3, 0.01)
        assert bits == ref_bits and np.array_equal(stream_of(words, bits), ref_words)
        out = torch.empty((128, 128, 128), dtype=torch.float32, device="cuda")
        cc.decompress_volume_float(inst, out, 3, 0.01, words, bits)
        rec = out.cpu().numpy()
        assert fields.psnr(vol, rec) > 40


def test_vector_field_256_full_size(oracle):
    """The bench workload at full size: 3 x 256^3 fields (the bench's seeds),
    3 levels, q0 = 0.01, one batch replayed as CUDA graphs.  Component 0's
    stream is word-identical to the oracle's and its reconstruction
    bit-identical; the other components' streams equal the plain codec's."""
    n, levels, q0 = 256, 3, 0.01
    vols = [fields.turbulence_field(n, 1024, 64, seed) for seed in (1002, 1003, 1004)]
    dev = [torch.from_numpy(v).cuda() for v in vols]
    outs = [torch.empty_like(d) for d in dev]
    with cc.Instance(0, 7, (n // 2) ** 3, 128, 14) as inst:
        with cc.VolumeBatch(inst, [v.shape for v in vols], levels, [q0] * 3, graph=True) as batch:
            for _ in range(2):   # the second pass replays the captured graphs
                batch.compress(dev)
                batch.decompress(outs)
            torch.cuda.synchronize()
            batch.status()
            streams = [batch.read_stream(c) for c in range(3)]
        ref_words, ref_bits = oracle.compress_volume(vols[0], levels, q0)
        assert streams[0][1] == ref_bits and np.array_equal(streams[0][0], ref_words)
        want = oracle.decompress_volume(ref_words, ref_bits, vols[0].shape, levels, q0)
        assert np.array_equal(outs[0].cpu().numpy().view(np.uint32), want.view(np.uint32))
        cap = cc.volume_stream_capacity_words(n, n, n)
        plain = torch.empty(cap, dtype=torch.int32, device="cuda")
        for c in (1, 2):
            _, bits = cc.compress_volume_float(inst, dev[c], levels, q0, plain)
            assert bits == streams[c][1] and np.array_equal(stream_of(plain, bits), streams[c][0])
            assert fields.psnr(vols[c], outs[c].cpu().numpy()) > 50


@pytest.mark.parametrize("n,levels,streams", [(64, 2, 3), (256, 4, 3), (256, 4, 5), (512, 3, 5), (2048, 4, 5)])
def test_heightfield_codec_matches_oracle_and_is_lossless(oracle, n, levels, streams):
    """3 streams: the decoder walks the stream one level at a time; 5: every
    level's streams in one device-walked decode."""
    img = fields.fbm_heightfield(n, seed=3000 + n)
    with cc.Instance(0, streams, (n // 2) ** 2, 128, 14) as inst:
        words, bits = cc.compress_heightfield(inst, torch.from_numpy(img).cuda(), levels)
        ref_words, ref_bits = oracle.compress_heightfield(img, levels)
        assert bits == ref_bits
        assert np.array_equal(stream_of(words, bits), ref_words)
        out = torch.empty((n, n), dtype=torch.int16, device="cuda")
        cc.decompress_heightfield(inst, out, levels, words, bits)
        assert np.array_equal(out.cpu().numpy(), img)
