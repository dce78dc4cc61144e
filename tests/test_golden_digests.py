"""The oracle against the reference's own output at the scope's full sizes:
SHA-256 digests of the streams and reconstructions the reference library
produced on a B200 (tests/golden/ref_digests.json, made by
tests/golden/make_golden.py --only digests) for the 128^3 volume, the three
256^3 components at q0 in {0.002, 0.01, 0.05}, a sample of the uneven bricks
and the 2048^2 lossless heightfield."""
import json
import os
import sys

import numpy as np
import pytest

from helpers import Oracle

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import digest_cases as dc  # noqa: E402

DIGESTS = os.path.join(HERE, "golden", "ref_digests.json")
if not os.path.exists(DIGESTS):
    pytest.skip("ref_digests.json not generated", allow_module_level=True)
with open(DIGESTS) as f:
    REF = json.load(f)


@pytest.fixture(scope="module")
def oracle():
    return Oracle()


@pytest.mark.parametrize("case", REF["volumes"], ids=[c["name"] for c in REF["volumes"]])
def test_oracle_volume_streams_match_reference(oracle, case):
    vol = dc.volume_input(case)
    assert dc.sha256(vol) == case["input_sha256"], "field generator changed"
    words, bits = oracle.compress_volume(vol, case["levels"], case["q0"])
    assert len(words) == case["words"] and bits == 32 * case["words"]
    assert dc.sha256(words) == case["stream_sha256"]
    rec = oracle.decompress_volume(words, bits, vol.shape, case["levels"], case["q0"])
    assert dc.sha256(rec) == case["recon_sha256"]


def test_oracle_brick_streams_match_reference(oracle):
    bricks, qs = dc.brick_inputs()
    items = REF["bricks"]["items"]
    assert len(items) == len(bricks)
    for b, q, it in zip(bricks, qs, items):
        assert list(b.shape) == it["shape"] and dc.sha256(b) == it["input_sha256"]
        assert np.float32(q) == np.float32(it["q0"])
        words, bits = oracle.compress_volume(b, dc.BRICK_LEVELS, q)
        assert len(words) == it["words"] and dc.sha256(words) == it["stream_sha256"], it["index"]
        rec = oracle.decompress_volume(words, bits, b.shape, dc.BRICK_LEVELS, q)
        assert dc.sha256(rec) == it["recon_sha256"], it["index"]


def test_oracle_heightfield_stream_matches_reference(oracle):
    h = REF["heightfield"]
    img = dc.heightfield_input()
    assert dc.sha256(img) == h["input_sha256"]
    words, bits = oracle.compress_heightfield(img, h["levels"])
    assert len(words) == h["words"] and dc.sha256(words) == h["stream_sha256"]
    rec = oracle.decompress_heightfield(words, bits, img.shape, h["levels"])
    assert np.array_equal(rec, img)
