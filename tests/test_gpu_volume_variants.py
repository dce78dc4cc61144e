"""The volume codec variants on the GPU (cc_compress_volume_float_ex with
CC_VOLUME_RLE_ONLY_LEVEL0, the quant-first codec and both multi-channel
decoders) against the reference's own example codec (tests/golden/
ref_volume.npz: streams word-identical, reconstructions bit-identical) and
against the oracle on larger volumes."""
import hashlib
import os

import numpy as np
import pytest

from helpers import Oracle

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

import cudacompress_b200 as cc  # noqa: E402
from cudacompress_b200 import fields  # noqa: E402

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_volume.npz")
SHAPES = {"f2": (16, 16, 32), "f2r": (16, 16, 32), "f3r": (32, 32, 32), "q2": (16, 16, 32), "q2r": (16, 16, 32),
          "q3": (32, 32, 32), "mf": (16, 16, 32), "mfr": (16, 16, 32), "mq": (16, 16, 32)}


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


@pytest.fixture(scope="module")
def oracle():
    return Oracle()


@pytest.fixture(scope="module")
def inst():
    i = cc.Instance(0, 7 * 3, 64 ** 3 // 8, 128, 14)
    yield i
    i.close()


def regen(shape, seed, sha):
    nz, ny, nx = shape
    v = fields.turbulence_field(max(shape), 64, 8, seed=int(seed))[:nz, :ny, :nx].copy()
    assert hashlib.sha256(v.tobytes()).digest() == bytes(sha)
    return v


def compress(inst, v, levels, q, rle, qf):
    f = cc.compress_volume_float_quant_first if qf else cc.compress_volume_float
    w, bits = f(inst, torch.from_numpy(v).cuda(), levels, q, rle_only_level0=bool(rle))
    return w[: (bits + 31) // 32].cpu().numpy().view(np.uint32).copy(), bits


def decompress(inst, words, shape, levels, q, rle, qf):
    out = torch.full(shape, float("nan"), dtype=torch.float32, device="cuda")
    d = torch.from_numpy(words.view(np.int32).copy()).cuda()
    f = cc.decompress_volume_float_quant_first if qf else cc.decompress_volume_float
    f(inst, out, levels, q, d, words.size * 32, rle_only_level0=bool(rle))
    return out.cpu().numpy()


@pytest.mark.parametrize("name", ["f2", "f2r", "f3r", "q2", "q2r", "q3"])
def test_volume_variant_matches_reference(gold, oracle, inst, name):
    levels, rle, qf = (int(x) for x in gold[f"{name}_meta"])
    q = float(gold[f"{name}_q"][0])
    v = regen(SHAPES[name], gold[f"{name}_seed"][0], gold[f"{name}_insha"])
    words, bits = compress(inst, v, levels, q, rle, qf)
    ref = gold[f"{name}_words"]
    assert bits == ref.size * 32 and np.array_equal(words, ref)
    rec = decompress(inst, ref, v.shape, levels, q, rle, qf)
    if f"{name}_rec" in gold.files:
        assert np.array_equal(rec.view(np.uint32), gold[f"{name}_rec"].view(np.uint32))
    else:
        # odd level count of the quant-first codec: the oracle's (correct) inverse
        want = oracle.decompress_volume(ref, ref.size * 32, v.shape, levels, q, rle_only_level0=rle, quant_first=qf)
        assert np.array_equal(rec.view(np.uint32), want.view(np.uint32))


@pytest.mark.parametrize("name", ["mf", "mfr", "mq"])
def test_multichannel_matches_reference(gold, inst, name):
    levels, rle, qf, count = (int(x) for x in gold[f"{name}_meta"])
    qs = [float(x) for x in gold[f"{name}_q"]]
    shape = SHAPES[name]
    outs = [torch.full(shape, float("nan"), dtype=torch.float32, device="cuda") for _ in range(count)]
    ws = [gold[f"{name}_words{k}"] for k in range(count)]
    dws = [torch.from_numpy(w.view(np.int32).copy()).cuda() for w in ws]
    cc.decompress_volume_float_multichannel(inst, outs, dws, [w.size * 32 for w in ws], qs, levels,
                                            rle_only_level0=bool(rle), quant_first=bool(qf))
    for k in range(count):
        got = outs[k].cpu().numpy()
        assert np.array_equal(got.view(np.uint32), gold[f"{name}_rec{k}"].view(np.uint32)), k
        single = decompress(inst, ws[k], shape, levels, qs[k], rle, qf)
        assert np.array_equal(got.view(np.uint32), single.view(np.uint32)), k


@pytest.mark.parametrize("qf,rle,levels", [(0, 1, 3), (1, 0, 3), (1, 1, 2), (1, 0, 1)])
def test_larger_volumes_against_oracle(oracle, qf, rle, levels):
    """64 x 64 x 128 field: streams word-identical to the oracle's and
    reconstructions bit-identical; quant-first within step / 2."""
    v = fields.turbulence_field(128, 256, 16, seed=9000 + levels)[:64, :64, :128].copy()
    q = 0.05 if qf else 0.01
    inst = cc.Instance(0, 7, 64 * 64 * 128 // 8, 128, 14)
    try:
        words, bits = compress(inst, v, levels, q, rle, qf)
        ow, ob = oracle.compress_volume(v, levels, q, rle_only_level0=rle, quant_first=qf)
        assert bits == ob and np.array_equal(words, ow)
        rec = decompress(inst, words, v.shape, levels, q, rle, qf)
        want = oracle.decompress_volume(ow, ob, v.shape, levels, q, rle_only_level0=rle, quant_first=qf)
        assert np.array_equal(rec.view(np.uint32), want.view(np.uint32))
        if qf:
            assert np.abs(rec - v).max() <= q / 2 * (1 + 1e-5)
    finally:
        inst.close()


def test_unknown_flags_rejected(inst):
    v = torch.zeros((16, 16, 32), dtype=torch.float32, device="cuda")
    w = torch.empty(1 << 16, dtype=torch.int32, device="cuda")
    bits = cc.lib().cc_compress_volume_float_ex(inst.handle, v.data_ptr(), 32, 16, 16, 2, 0.1, 4, w.data_ptr(),
                                                w.numel(), None)
    assert bits != 0
    assert "flags" in cc.last_error()


def test_container_round_trip_decodes(oracle, inst):
    """Streams written to a container with their sizes and steps decode from
    the container alone to the same reconstruction."""
    from cudacompress_b200 import container as ct
    vols = [fields.turbulence_field(32, 64, 8, seed=s)[:16, :16, :32].copy() for s in (71, 72)]
    steps = [0.05, 0.03]
    ss = []
    for v, q in zip(vols, steps):
        w, bits = compress(inst, v, 2, q, 1, 1)
        ss.append(ct.Stream(v.shape, q, bits, w))
    info, back = ct.unpack(ct.pack(ct.ContainerInfo(ct.QUANT_FIRST, cc.RLE_ONLY_LEVEL0, 2, 128, 14), ss))
    assert info.codec == ct.QUANT_FIRST and info.flags == cc.RLE_ONLY_LEVEL0 and info.levels == 2
    for v, s in zip(vols, back):
        rec = decompress(inst, s.words, s.shape, info.levels, s.quant_step, info.flags & 1, 1)
        want = oracle.decompress_volume(s.words, s.bit_size, v.shape, 2, s.quant_step, rle_only_level0=True,
                                        quant_first=True)
        assert np.array_equal(rec.view(np.uint32), want.view(np.uint32))
