"""The oracle and the product's host table builder against the golden
fixtures made from the reference's own code (tests/golden/make_golden.py):
Huffman tables and serialized headers (reference HuffmanEncodeTable built on
the CPU), and - where the fixtures from the reference's GPU run are present -
encodeRLHuff / encodeHuff bit streams, DWT and quantizer outputs."""
import ctypes
import os

import numpy as np
import pytest

from helpers import ROOT, Oracle, bind_build, load_oracle, load_selftest, run_build

GOLDEN = os.path.join(ROOT, "tests", "golden")


def _load(name):
    path = os.path.join(GOLDEN, name)
    if not os.path.exists(path):
        pytest.skip(f"{name} not generated")
    return np.load(path, allow_pickle=False)


def golden_tables():
    z = _load("ref_tables.npz")
    ho, to = z["hist_off"], z["table_off"]
    for k, (smax, log2max, r, tb) in enumerate(z["meta"]):
        yield (z["hist"][ho[k]:ho[k + 1]], int(smax), int(log2max), int(r), int(tb),
               z["lengths"][ho[k]:ho[k + 1]], z["codewords"][ho[k]:ho[k + 1]], z["table_words"][to[k]:to[k + 1]])


def _check_builder(f):
    count = 0
    for hist, smax, log2max, r, tb, lens, cws, tws in golden_tables():
        a = run_build(f, hist, smax, log2max)
        assert a[0] == r and a[4] == tb, (count, a[0], r, a[4], tb)
        assert np.array_equal(a[3], tws), count
        if hist.any():
            assert np.array_equal(a[2].astype(np.uint8), lens), count
            assert np.array_equal(a[1], cws), count
        count += 1
    assert count > 100


def test_oracle_tables_match_reference_golden():
    _check_builder(bind_build(load_oracle(), "orc_huffman_build"))


def test_product_host_builder_matches_reference_golden():
    lib = load_selftest()
    if lib is None:
        pytest.skip("self-test library not built")
    _check_builder(bind_build(lib, "ccst_huffman_build"))


def golden_streams():
    z = _load("ref_streams.npz")
    for i in range(int(z["count"][0])):
        kind, sym_bytes, log2max, cb, S, n, start, rc, size, pos = (int(v) for v in z[f"c{i}_meta"])
        yield dict(i=i, kind=kind, sym_bytes=sym_bytes, log2max=log2max, cb=cb, S=S, n=n, start=start, rc=rc,
                   size=size, pos=pos, syms=z[f"c{i}_in"], words=z[f"c{i}_out"], prefix=z[f"c{i}_prefix"])


def test_oracle_streams_match_reference_gpu_golden():
    orc = Oracle()
    seen = 0
    for c in golden_streams():
        pre = c["prefix"] if c["start"] else None
        res = orc.encode(c["kind"], c["syms"], cb=c["cb"], log2max=c["log2max"], start_words=pre,
                         start_bit_size=c["start"], start_pos=c["start"])
        if c["rc"] != 0:
            assert res is None, c["i"]
            continue
        words, size, pos = res
        assert size == c["size"] and pos == c["pos"], (c["i"], size, c["size"])
        assert np.array_equal(words, c["words"]), c["i"]
        seen += 1
    assert seen >= 15


def test_oracle_dwt_and_quantizer_match_reference_gpu_golden():
    z = _load("ref_dwt.npz")
    orc = Oracle()
    for i in range(3):
        vol = z[f"f{i}_in"]
        fwd = orc.dwt_float(vol)
        assert np.array_equal(fwd.view(np.uint32), z[f"f{i}_fwd"].view(np.uint32)), i
        inv = orc.dwt_float(z[f"f{i}_fwd"], inverse=True)
        assert np.array_equal(inv.view(np.uint32), z[f"f{i}_inv"].view(np.uint32)), i
        sym = orc.quantize(z[f"f{i}_fwd"], float(z[f"q{i}_step"][0]))
        assert np.array_equal(sym, z[f"q{i}_sym"]), i
        img = z[f"i{i}_in"]
        img = img if img.shape[0] > 1 else img[0]
        fwd_i = orc.dwt_int(img)
        assert np.array_equal(fwd_i.reshape(-1), z[f"i{i}_fwd"].reshape(-1)), i
        inv_i = orc.dwt_int(z[f"i{i}_fwd"] if z[f"i{i}_fwd"].shape[0] > 1 else z[f"i{i}_fwd"][0], inverse=True)
        assert np.array_equal(inv_i.reshape(-1), z[f"i{i}_inv"].reshape(-1)), i
