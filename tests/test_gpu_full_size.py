"""The CUDA path against the reference's own output at the scope's full
sizes (SHA-256 digests of the reference library's streams and
reconstructions, tests/golden/ref_digests.json): the 3 x 256^3 vector field
at every q0 of its sweep through the batched codec (CUDA graphs) and through
the plain per-volume codec, the 128^3 volume, a sample of the uneven bricks in
one batch, and the 2048^2 lossless heightfield."""
import json
import os
import sys

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

import cudacompress_b200 as cc  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import digest_cases as dc  # noqa: E402

DIGESTS = os.path.join(HERE, "golden", "ref_digests.json")
if not os.path.exists(DIGESTS):
    pytest.skip("ref_digests.json not generated", allow_module_level=True)
with open(DIGESTS) as f:
    REF = json.load(f)


def by_q0(q0):
    return [c for c in REF["volumes"] if c["n"] == 256 and c["q0"] == q0]


@pytest.mark.parametrize("q0", dc.C2_Q0)
def test_vector_field_256_matches_reference(q0):
    cases = by_q0(q0)
    assert len(cases) == 3
    vols = [dc.volume_input(c) for c in cases]
    dev = [torch.from_numpy(v).cuda() for v in vols]
    outs = [torch.full_like(d, float("nan")) for d in dev]
    n, levels = 256, cases[0]["levels"]
    with cc.Instance(0, 7, (n // 2) ** 3, 128, 14) as inst:
        with cc.VolumeBatch(inst, [v.shape for v in vols], levels, [q0] * 3, graph=True) as batch:
            for _ in range(2):      # the second pass replays the captured graphs
                batch.compress(dev)
                batch.decompress(outs)
            torch.cuda.synchronize()
            batch.status()
            for k, c in enumerate(cases):
                words, bits = batch.read_stream(k)
                assert len(words) == c["words"] and bits == 32 * c["words"], c["name"]
                assert dc.sha256(words) == c["stream_sha256"], c["name"]
                assert dc.sha256(outs[k].cpu().numpy()) == c["recon_sha256"], c["name"]
        # the plain per-volume codec on component 0
        cap = cc.volume_stream_capacity_words(n, n, n)
        words_t = torch.empty(cap, dtype=torch.int32, device="cuda")
        _, bits = cc.compress_volume_float(inst, dev[0], levels, q0, words_t)
        torch.cuda.synchronize()
        got = words_t[: (bits + 31) // 32].cpu().numpy().view(np.uint32)
        assert dc.sha256(got) == cases[0]["stream_sha256"]
        out = torch.full_like(dev[0], float("nan"))
        cc.decompress_volume_float(inst, out, levels, q0, words_t, bits)
        assert dc.sha256(out.cpu().numpy()) == cases[0]["recon_sha256"]


def test_volume_128_matches_reference():
    c = REF["volumes"][0]
    assert c["n"] == 128
    vol = dc.volume_input(c)
    with cc.Instance(0, 7, 64 ** 3, 128, 14) as inst:
        words_t, bits = cc.compress_volume_float(inst, torch.from_numpy(vol).cuda(), c["levels"], c["q0"])
        torch.cuda.synchronize()
        got = words_t[: (bits + 31) // 32].cpu().numpy().view(np.uint32)
        assert len(got) == c["words"] and dc.sha256(got) == c["stream_sha256"]
        out = torch.full((128, 128, 128), float("nan"), dtype=torch.float32, device="cuda")
        cc.decompress_volume_float(inst, out, c["levels"], c["q0"], words_t, bits)
        assert dc.sha256(out.cpu().numpy()) == c["recon_sha256"]


def test_brick_sample_matches_reference():
    bricks, qs = dc.brick_inputs()
    items = REF["bricks"]["items"]
    dev = [torch.from_numpy(b).cuda() for b in bricks]
    outs = [torch.full_like(d, float("nan")) for d in dev]
    with cc.Instance(0, 7, 32 ** 3, 128, 14) as inst:
        with cc.VolumeBatch(inst, [b.shape for b in bricks], dc.BRICK_LEVELS, qs, graph=True) as batch:
            for _ in range(2):
                batch.compress(dev)
                batch.decompress(outs)
            torch.cuda.synchronize()
            batch.status()
            for k, it in enumerate(items):
                words, _ = batch.read_stream(k)
                assert len(words) == it["words"] and dc.sha256(words) == it["stream_sha256"], k
                assert dc.sha256(outs[k].cpu().numpy()) == it["recon_sha256"], k


def test_heightfield_2048_matches_reference():
    h = REF["heightfield"]
    img = dc.heightfield_input()
    n = h["n"]
    with cc.Instance(0, 5, (n // 2) ** 2, 128, 14) as inst:
        words_t, bits = cc.compress_heightfield(inst, torch.from_numpy(img).cuda(), h["levels"])
        torch.cuda.synchronize()
        got = words_t[: (bits + 31) // 32].cpu().numpy().view(np.uint32)
        assert len(got) == h["words"] and dc.sha256(got) == h["stream_sha256"]
        out = torch.empty((n, n), dtype=torch.int16, device="cuda")
        cc.decompress_heightfield(inst, out, h["levels"], words_t, bits)
        assert np.array_equal(out.cpu().numpy(), img)


def test_fp32_error_against_fp64():
    """The FP32 transform and codec against the FP64 transform with the same
    taps (cudacompress_b200/accuracy.py) on component 0 of the vector field:
    coefficients within 2e-6 of the largest coefficient, reconstructions
    within 2e-5 of the FP64 inverse of the same symbols, and the codec's PSNR
    within 0.01 dB of the FP64 pipeline's at every q0 of the sweep."""
    from cudacompress_b200 import accuracy
    c = by_q0(dc.C2_Q0[0])[0]
    vol = torch.from_numpy(dc.volume_input(c)).cuda()
    with cc.Instance(0, 7, 128 ** 3, 128, 14) as inst:
        rep = accuracy.error_report(inst, vol, c["levels"], dc.C2_Q0)
    co = rep["coefficients"]
    assert co["max_abs"] < 2e-6 * co["max_abs_coefficient"], co
    for q0, r in rep["reconstruction"].items():
        assert r["max_abs"] < 2e-5 and r["rms"] < 2e-6, (q0, r)
        assert abs(r["psnr_fp32"] - r["psnr_fp64"]) < 0.01, (q0, r)
