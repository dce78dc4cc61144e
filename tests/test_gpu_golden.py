"""The CUDA path against the golden fixtures made by running the reference's
own GPU code (tests/golden/make_golden.py --gpu): encodeRLHuff / encodeHuff
bit streams byte-identical, decode of the reference's streams, DWT and
quantizer outputs bit-identical."""
import os

import numpy as np
import pytest

from helpers import ROOT

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

import cudacompress_b200 as cc  # noqa: E402

GOLDEN = os.path.join(ROOT, "tests", "golden")


def _load(name):
    path = os.path.join(GOLDEN, name)
    if not os.path.exists(path):
        pytest.skip(f"{name} not generated")
    return np.load(path, allow_pickle=False)


def _cases():
    z = _load("ref_streams.npz")
    out = []
    for i in range(int(z["count"][0])):
        kind, sym_bytes, log2max, cb, S, n, start, rc, size, pos = (int(v) for v in z[f"c{i}_meta"])
        out.append(dict(i=i, kind=kind, log2max=log2max, cb=cb, S=S, n=n, start=start, rc=rc, size=size, pos=pos,
                        syms=z[f"c{i}_in"], words=z[f"c{i}_out"], prefix=z[f"c{i}_prefix"]))
    return out


def _dev_streams(syms):
    dt = torch.int16 if syms.dtype == np.uint16 else torch.int32
    view = np.int16 if syms.dtype == np.uint16 else np.int32
    return [torch.from_numpy(np.ascontiguousarray(r).view(view)).cuda().view(dt) for r in syms]


def test_encode_matches_reference_gpu_streams():
    for c in _cases():
        with cc.Instance(0, c["S"], c["n"], c["cb"], c["log2max"]) as inst:
            bs = cc.BitStream(c["prefix"], c["start"]) if c["start"] else cc.BitStream()
            bs.set_bit_position(c["start"])
            streams = _dev_streams(c["syms"])
            enc = cc.encode_rlhuff if c["kind"] == 0 else cc.encode_huff
            ok = enc(inst, bs, streams, c["n"])
            if c["rc"] != 0:
                assert not ok, c["i"]
                continue
            assert ok, (c["i"], cc.last_error())
            assert bs.bit_size == c["size"] and bs.pos == c["pos"], (c["i"], bs.bit_size, c["size"])
            assert np.array_equal(bs.raw(), c["words"]), c["i"]


def test_decode_of_reference_gpu_streams():
    for c in _cases():
        if c["rc"] != 0:
            continue
        with cc.Instance(0, c["S"], c["n"], c["cb"], c["log2max"]) as inst:
            bs = cc.BitStream(c["words"], c["size"])
            bs.set_bit_position(c["start"])
            dt = torch.int16 if c["syms"].dtype == np.uint16 else torch.int32
            outs = [torch.zeros(c["n"] + 32 * c["cb"], dtype=dt, device="cuda") for _ in range(c["S"])]
            dec = cc.decode_rlhuff if c["kind"] == 0 else cc.decode_huff
            assert dec(inst, bs, outs, c["n"]), (c["i"], cc.last_error())
            assert cc.decode_status(inst) == 0, c["i"]
            assert bs.pos == c["pos"], c["i"]
            got = np.stack([o[: c["n"]].cpu().numpy() for o in outs]).view(c["syms"].dtype)
            assert np.array_equal(got, c["syms"]), c["i"]


def test_dwt_and_quantizer_match_reference_gpu():
    z = _load("ref_dwt.npz")
    for i in range(3):
        vol = z[f"f{i}_in"]
        nz, ny, nx = vol.shape
        src = torch.from_numpy(vol).cuda()
        dst, b1, b2 = (torch.empty_like(src) for _ in range(3))
        cc.dwt_float_forward(dst, b2, b1, src, nx, ny, nz)
        assert np.array_equal(dst.cpu().numpy().view(np.uint32), z[f"f{i}_fwd"].view(np.uint32)), i
        src2 = torch.from_numpy(z[f"f{i}_fwd"]).cuda()
        inv = torch.empty_like(src2)
        cc.dwt_float_inverse(inv, b2, b1, src2, nx, ny, nz)
        assert np.array_equal(inv.cpu().numpy().view(np.uint32), z[f"f{i}_inv"].view(np.uint32)), i
        sym = torch.zeros(vol.size, dtype=torch.int16, device="cuda")
        cc.quantize_to_symbols(sym, src2, nx, ny, nz, float(z[f"q{i}_step"][0]))
        assert np.array_equal(sym.cpu().numpy().view(np.uint16).reshape(vol.shape), z[f"q{i}_sym"]), i
        img = z[f"i{i}_in"]
        nz, ny, nx = img.shape
        s = torch.from_numpy(img).cuda()
        d, buf = torch.empty_like(s), torch.empty_like(s)
        cc.dwt_int_forward(d, buf, s, nx, ny, nz)
        assert np.array_equal(d.cpu().numpy(), z[f"i{i}_fwd"]), i
        s2 = torch.from_numpy(z[f"i{i}_fwd"]).cuda()
        d2 = torch.empty_like(s2)
        cc.dwt_int_inverse(d2, buf, s2, nx, ny, nz)
        assert np.array_equal(d2.cpu().numpy(), z[f"i{i}_inv"]), i
