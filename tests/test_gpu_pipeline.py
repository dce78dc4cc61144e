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


@pytest.mark.parametrize("n,levels,streams", [(64, 2, 3), (256, 4, 3), (256, 4, 5), (512, 3, 5)])
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
