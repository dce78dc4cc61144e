"""Pins the oracle's 2D image side (byte DWTs, lowpass-only transforms,
byte-image quantizers, YCoCg, Bits, one-level image and heightfield codecs)
against fixtures recorded from the reference's own code on a GPU
(tests/golden/ref_image.npz, made by tests/golden/make_golden.py), plus
properties of the oracle that need no fixture.  CPU only."""
import os

import numpy as np
import pytest

from helpers import ROOT, ImageOracle

FIX = os.path.join(ROOT, "tests", "golden", "ref_image.npz")


@pytest.fixture(scope="module")
def orc():
    return ImageOracle()


@pytest.fixture(scope="module")
def g():
    if not os.path.exists(FIX):
        pytest.skip("ref_image.npz not generated")
    return dict(np.load(FIX))


def test_byte_dwt_forward(orc, g):
    for name in ("b2", "b3"):
        img = g[f"{name}_in"]
        dims = img.shape[:-1]
        for c in range(img.shape[-1]):
            got = orc.dwt_fwd_from_byte(img[0] if dims[0] == 1 else img, c)
            assert np.array_equal(got.reshape(dims), g[f"{name}_fwd{c}"]), (name, c)


def test_byte_dwt_inverse(orc, g):
    for name in ("b2", "b3"):
        ref = g[f"{name}_inv"]
        tgt = np.full(ref.shape, 77, np.uint8)
        orc.dwt_inv_to_byte(g[f"{name}_invcoef"], tgt, 1)
        assert np.array_equal(tgt, ref), name


def test_byte_dwt_inverse_from_symbols(orc, g):
    for name in ("b2", "b3"):
        ref = g[f"{name}_symout"]
        bands = g[f"{name}_symbands"]
        lpfull = g[f"{name}_symlp"]
        nz, ny, nx = lpfull.shape
        lp = lpfull[: max(nz // 2, 1), : ny // 2, : nx // 2]
        tgt = np.full(ref.shape, 55, np.uint8)
        orc.dwt_inv_from_symbols_to_byte(lp, [bands[k] for k in range(len(bands))], 0.75, tgt, ref.shape[-1] - 1)
        assert np.array_equal(tgt, ref), name


def lowpass_columns_defined(nx):
    """LL columns the reference's dwtFloat2DForwardLowpassOnly writes: past the
    whole 256-sample blocks its rest kernel covers ceil(rest / 32) blocks of
    32 samples but stores only blockCount / 2 (rounded down) blocks of 32
    outputs (DWTFloat2DLowpassKernels.cui:140-155), so with an odd block count
    the last outputs come from whatever the buffer held."""
    done = nx // 256 * 256
    rest = nx - done
    return min(nx // 2, done // 2 + (-(-rest // 32) // 2) * 32)


def test_lowpass_only(orc, g):
    for name in ("lf", "lfr"):
        got = orc.lowpass_from_byte(g[f"{name}_in"], int(g[f"{name}_meta"][0]))
        k = lowpass_columns_defined(g[f"{name}_in"].shape[1])
        assert np.array_equal(got[:, :k], g[f"{name}_out"][:, :k]), name
    assert lowpass_columns_defined(200) == 96 and lowpass_columns_defined(64) == 32
    for name in ("li", "li2"):
        assert np.array_equal(orc.int_lowpass(g[f"{name}_in"]), g[f"{name}_out"]), name


def test_byte_quantizers(orc, g):
    data, ref = g["q_data"], g["q_ref"]
    ny, pitch = data.shape
    nx = ref.shape[1]
    qb = np.zeros(ref.shape, np.uint8)
    orc.float_to_byte_2d(qb, 1, (data * 3).astype(np.float32), nx, ny, pitch)
    assert np.array_equal(qb, g["q_f2b"])
    fb = np.zeros((ny, pitch), np.float32)
    orc.byte_to_float_2d(fb, ref, 1, nx, ny, pitch)
    assert np.array_equal(fb, g["q_b2f"])
    for t in (0, 1):
        for rt in (0, 1):
            d = data.copy()
            sym = orc.quantize_difference(d, 3.0, ref, 1, nx, ny, pitch, t, bool(rt))
            assert np.array_equal(sym, g[f"q_sym{t}{rt}"]), (t, rt)
            assert np.array_equal(d, g[f"q_data{t}{rt}"]), (t, rt)
        back = np.full((ny, pitch), -1.0, np.float32)
        orc.unquantize_difference(back, g[f"q_sym{t}0"], 3.0, ref, 1, nx, ny, pitch, t)
        assert np.array_equal(back, g[f"q_unq{t}"]), t


def test_ycocg(orc, g):
    for ch in (3, 4):
        px = g[f"y{ch}_in"]
        assert np.array_equal(orc.ycocg(px, True), g[f"y{ch}_1"])
        assert np.array_equal(orc.ycocg(px, False), g[f"y{ch}_0"])


def test_bits(orc, g):
    vals, bits0 = g["l_in"], g["l_bits_in"]
    for mode, shift in [(0, 0), (1, 0), (1, 3), (2, 0), (2, -5)]:
        d, b = orc.lsb(mode, vals, bits0 if mode == 2 else (np.zeros(len(bits0), np.uint32)), shift)
        assert np.array_equal(d, g[f"l{mode}_{shift}_data"]), (mode, shift)
        assert np.array_equal(b, g[f"l{mode}_{shift}_bits"]), (mode, shift)
    assert np.array_equal(orc.shift_elems(vals, 7), g["l3_7_data"])
    d, _ = orc.lsb(1, vals, None, 2)
    assert np.array_equal(d, g["l1n_2_data"])


def test_image_codec(orc, g):
    for name in ("c3", "c4", "m3"):
        proc, count = (int(v) for v in g[f"{name}_meta"])
        steps, offs, words = g[f"{name}_steps"], g[f"{name}_offsets"], g[f"{name}_words"]
        for k in range(count):
            img = g[f"{name}_in{k}"]
            lp = g[f"{name}_lp{k}"]   # the reference's getLowpassImage output is the codec's input
            kx = lowpass_columns_defined(img.shape[1])
            assert np.array_equal(orc.lowpass_image(img, proc)[:, :kx], lp[:, :kx]), (name, k)
            w, bits, rec = orc.compress_image(img, proc, lp, float(steps[k]))
            ref_w = words[offs[k]: offs[k + 1]]
            assert np.array_equal(w, ref_w), (name, k)
            assert np.array_equal(rec, g[f"{name}_rec{k}"]), (name, k)
            out = np.full(img.shape, 201, np.uint8)
            orc.decompress_image(ref_w, len(ref_w) * 32, out, proc, lp, float(steps[k]))
            assert np.array_equal(out, g[f"{name}_dec{k}"]), (name, k)


def test_heightfield_one_level(orc, g):
    for name in ("h0", "h3"):
        img, shift = g[f"{name}_in"], int(g[f"{name}_shift"][0])
        w, bits, lp = orc.compress_heightfield_one_level(img, shift)
        assert np.array_equal(w, g[f"{name}_words"]), name
        assert np.array_equal(lp, g[f"{name}_lp"]), name
        out, lpd = orc.decompress_heightfield_one_level(g[f"{name}_words"], len(g[f"{name}_words"]) * 32, img.shape,
                                                        g[f"{name}_lp"], shift)
        assert np.array_equal(out, g[f"{name}_dec"]), name
        # the decoder adds the shift again after appending the bit: lossless for shift 0
        assert shift != 0 or np.array_equal(out, img), name
        assert np.array_equal(lpd, g[f"{name}_lpdec"]), name
        assert np.array_equal(orc.lowpass_heightfield(img, shift + 2), g[f"{name}_getlp"]), name


# ---- properties that need no fixture ----
def test_lsb_remove_append_identity(orc):
    rng = np.random.default_rng(1)
    v = rng.integers(-32768, 32768, 5000).astype(np.int16)
    for shift in (0, 1, -7, 100):
        d, b = orc.lsb(1, v, np.zeros((v.size + 31) // 32, np.uint32), shift)
        back, _ = orc.lsb(2, d, b, -shift)
        assert np.array_equal(back, v), shift
        # removing the bit is a floor division of (v + shift) by two (16-bit wrap)
        assert np.array_equal(d, ((v.astype(np.int32) + shift).astype(np.int16).astype(np.int32) >> 1).astype(np.int16))


def test_heightfield_one_level_lossless(orc):
    rng = np.random.default_rng(2)
    img = np.cumsum(rng.integers(-9, 10, (40, 72)), axis=1).astype(np.int16)
    for shift in (0, 5):
        w, bits, lp = orc.compress_heightfield_one_level(img, shift)
        # appendLSB adds its shift after the bit: -shift restores the lowpass exactly
        out, lpd = orc.decompress_heightfield_one_level(w, bits, img.shape, lp, -shift)
        assert np.array_equal(out, img), shift


def test_ycocg_ranges(orc):
    px = np.array(np.meshgrid(np.arange(0, 256, 15), np.arange(0, 256, 15), np.arange(0, 256, 15))).reshape(3, -1).T
    px = np.ascontiguousarray(px.astype(np.uint8))
    y = orc.ycocg(px, True)
    back = orc.ycocg(y, False).astype(int)
    # one bit of chroma is lost: the round trip is within 2 of the input
    assert np.abs(back - px.astype(int)).max() <= 2
