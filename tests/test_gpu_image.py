"""The 2D image side on the GPU: byte-input / byte-output float DWTs, the
lowpass-only transforms, the byte-image quantizers, YCoCg, the Bits helpers,
and the one-level image and heightfield codecs - against the reference's own
outputs (tests/golden/ref_image.npz: bit-identical arrays, word-identical
streams) and against the oracle on larger and ragged cases."""
import os

import numpy as np
import pytest

from helpers import ImageOracle
from test_golden_image import lowpass_columns_defined

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

import cudacompress_b200 as cc  # noqa: E402
from cudacompress_b200 import image as ci  # noqa: E402
from cudacompress_b200._ffi import CudaCompressError  # noqa: E402

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_image.npz")


@pytest.fixture(scope="module")
def gold():
    if not os.path.exists(GOLD):
        pytest.skip("ref_image.npz not generated")
    return dict(np.load(GOLD))


@pytest.fixture(scope="module")
def orc():
    return ImageOracle()


@pytest.fixture(scope="module")
def inst():
    i = cc.Instance(0, 4 * 3 * 4, 256 * 256, 128, 14)
    yield i
    i.close()


def cu(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t, dtype=None):
    a = t.cpu().numpy()
    return a.view(dtype) if dtype is not None else a


def image(shape, seed):
    ny, nx, ch = shape
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:ny, 0:nx].astype(np.float64)
    out = np.empty(shape, np.uint8)
    for c in range(ch):
        k = rng.uniform(0.02, 0.3, 4)
        v = 128 + 80 * np.sin(k[0] * x + k[1] * y) + 40 * np.cos(k[2] * x - k[3] * y) + rng.uniform(-20, 20, (ny, nx))
        out[..., c] = np.clip(np.rint(v), 0, 255).astype(np.uint8)
    return out


def terrain(shape, seed):
    rng = np.random.default_rng(seed)
    return np.clip(np.cumsum(np.cumsum(rng.integers(-6, 7, shape), axis=0), axis=1), -30000, 30000).astype(np.int16)


def fwd_from_byte(img, channel):
    """Product forward DWT of one channel of img (..., ch) uint8."""
    dims = img.shape[:-1]
    nz, ny, nx = (1,) + dims if len(dims) == 2 else dims
    src = cu(img)
    dst, b1, b2 = (torch.empty(dims, dtype=torch.float32, device="cuda") for _ in range(3))
    view = src.view(-1)[channel:]
    cc.dwt_float_forward_from_byte(dst, b2, b1, view, nx, ny, nz, img.shape[-1])
    return host(dst)


def inv_to_byte(coef, target, channel):
    dims = coef.shape
    nz, ny, nx = (1,) + dims if len(dims) == 2 else dims
    t = cu(target)
    b1, b2 = (torch.empty(dims, dtype=torch.float32, device="cuda") for _ in range(2))
    cc.dwt_float_inverse_to_byte(t.view(-1)[channel:], b2, b1, cu(coef.astype(np.float32)), nx, ny, nz,
                                 target.shape[-1])
    return host(t)


# ------------------------------------------------------------- fixtures
def test_byte_dwt_vs_reference(gold):
    for name in ("b2", "b3"):
        img = gold[f"{name}_in"]
        dims = img.shape[:-1]
        for c in range(img.shape[-1]):
            got = fwd_from_byte(img[0] if dims[0] == 1 else img, c)
            assert np.array_equal(got.reshape(dims), gold[f"{name}_fwd{c}"]), (name, c)
        ref = gold[f"{name}_inv"]
        coef = gold[f"{name}_invcoef"]
        got = inv_to_byte(coef[0] if dims[0] == 1 else coef, np.full(ref.shape, 77, np.uint8).reshape(
            ref.shape[1:] if dims[0] == 1 else ref.shape), 1)
        assert np.array_equal(got.reshape(ref.shape), ref), name


def test_byte_dwt_from_symbols_vs_reference(gold):
    for name in ("b2", "b3"):
        ref = gold[f"{name}_symout"]
        bands = gold[f"{name}_symbands"]
        lpfull = gold[f"{name}_symlp"]
        nz, ny, nx = lpfull.shape
        ch = ref.shape[-1]
        dband = [cu(bands[k]) for k in range(len(bands))]
        ptrs = torch.tensor([t.data_ptr() for t in dband], dtype=torch.int64, device="cuda")
        t = cu(np.full(ref.shape, 55, np.uint8))
        b1, b2 = (torch.empty((nz, ny, nx), dtype=torch.float32, device="cuda") for _ in range(2))
        cc.dwt_float_inverse_from_symbols_to_byte(t.view(-1)[ch - 1:], b2, b1, cu(lpfull), ptrs, 2, 0.75, nx, ny, nz,
                                                  ch)
        assert np.array_equal(host(t), ref), name


def test_lowpass_only_vs_reference(gold):
    for name in ("lf", "lfr"):
        img = gold[f"{name}_in"]
        ny, nx, ch = img.shape
        c = int(gold[f"{name}_meta"][0])
        dst = torch.full((ny // 2, nx // 2), float("nan"), dtype=torch.float32, device="cuda")
        cc.dwt_float2d_forward_lowpass_only_from_byte(dst, None, cu(img).view(-1)[c:], nx, ny, ch)
        k = lowpass_columns_defined(nx)   # the reference leaves the rest to its buffer's contents
        assert np.array_equal(host(dst)[:, :k], gold[f"{name}_out"][:, :k]), name
    for name in ("li", "li2"):
        hf = gold[f"{name}_in"]
        ny, nx = hf.shape
        dst = torch.zeros((ny // 2, nx // 2), dtype=torch.int16, device="cuda")
        cc.dwt_int_forward_lowpass_only(dst, None, cu(hf), nx, ny)
        assert np.array_equal(host(dst), gold[f"{name}_out"]), name


def test_byte_quantizers_vs_reference(gold):
    data, ref = gold["q_data"], gold["q_ref"]
    ny, pitch = data.shape
    nx, chc = ref.shape[1], ref.shape[2]
    qb = torch.zeros(ref.shape, dtype=torch.uint8, device="cuda")
    ci.float_to_byte_2d(qb, chc, 1, cu(data * 3), nx, ny, pitch)
    assert np.array_equal(host(qb), gold["q_f2b"])
    fb = torch.zeros((ny, pitch), dtype=torch.float32, device="cuda")
    ci.byte_to_float_2d(fb, cu(ref), chc, 1, nx, ny, pitch)
    assert np.array_equal(host(fb), gold["q_b2f"])
    dref = cu(ref)
    for t in (0, 1):
        for rt in (0, 1):
            d = cu(data)
            sym = torch.zeros((ny, nx), dtype=torch.int16, device="cuda")
            f = ci.quantize_difference_to_symbols_roundtrip_2d if rt else ci.quantize_difference_to_symbols_2d
            f(sym, d, 3.0, dref, chc, 1, nx, ny, pitch, t)
            assert np.array_equal(host(sym, np.uint16), gold[f"q_sym{t}{rt}"]), (t, rt)
            assert np.array_equal(host(d), gold[f"q_data{t}{rt}"]), (t, rt)
        back = cu(np.full((ny, pitch), -1.0, np.float32))
        ci.unquantize_difference_from_symbols_2d(back, cu(gold[f"q_sym{t}0"].view(np.int16)), 3.0, dref, chc, 1, nx,
                                                 ny, pitch, t)
        assert np.array_equal(host(back), gold[f"q_unq{t}"]), t


def test_ycocg_vs_reference(gold):
    for ch in (3, 4):
        px = cu(gold[f"y{ch}_in"])
        for d, f in ((1, ci.convert_rgb_to_ycocg), (0, ci.convert_ycocg_to_rgb)):
            out = torch.zeros_like(px)
            f(out, px)
            assert np.array_equal(host(out), gold[f"y{ch}_{d}"]), (ch, d)
        inplace = px.clone()
        ci.convert_rgb_to_ycocg(inplace, inplace)   # target and source may be the same memory
        assert np.array_equal(host(inplace), gold[f"y{ch}_1"]), ch


def test_bits_vs_reference(gold):
    vals, bits0 = gold["l_in"], gold["l_bits_in"]
    n = vals.size
    for mode, shift in [(0, 0), (1, 0), (1, 3), (2, 0), (2, -5)]:
        d = cu(vals)
        b = cu(bits0.view(np.int32)) if mode == 2 else torch.zeros(n // 32, dtype=torch.int32, device="cuda")
        if mode == 0:
            ci.get_lsb(d, b, n)
        elif mode == 1:
            ci.remove_lsb(d, b, n, shift)
        else:
            ci.append_lsb(d, b, n, shift)
        assert np.array_equal(host(d), gold[f"l{mode}_{shift}_data"]), (mode, shift)
        assert np.array_equal(host(b, np.uint32), gold[f"l{mode}_{shift}_bits"]), (mode, shift)
    d = cu(vals)
    ci.shift_elems(d, n, 7)
    assert np.array_equal(host(d), gold["l3_7_data"])
    d = cu(vals)
    ci.remove_lsb(d, None, n, 2)
    assert np.array_equal(host(d), gold["l1n_2_data"])


def test_image_codec_vs_reference(gold, inst):
    for name in ("c3", "c4", "m3"):
        proc, count = (int(v) for v in gold[f"{name}_meta"])
        steps, offs, words = gold[f"{name}_steps"], gold[f"{name}_offsets"], gold[f"{name}_words"]
        imgs = [cu(gold[f"{name}_in{k}"]) for k in range(count)]
        kx = lowpass_columns_defined(gold[f"{name}_in0"].shape[1])
        for k in range(count):
            got = host(ci.get_lowpass_image(imgs[k], proc))
            assert np.array_equal(got[:, :kx], gold[f"{name}_lp{k}"][:, :kx]), (name, k)
        lps = [cu(gold[f"{name}_lp{k}"]) for k in range(count)]   # the reference's lowpass is the codec input
        if count == 1:
            w, bits = ci.compress_image_one_level(inst, imgs[0], proc, lps[0], float(steps[0]))
            res = [(w, bits)]
        else:
            res = ci.compress_images_one_level(inst, imgs, proc, lps, [float(s) for s in steps])
        for k in range(count):
            w, bits = res[k]
            got = host(w[: bits // 32], np.uint32)
            assert np.array_equal(got, words[offs[k]: offs[k + 1]]), (name, k)
            assert np.array_equal(host(imgs[k]), gold[f"{name}_rec{k}"]), (name, k)
        outs = [cu(np.full(gold[f"{name}_in0"].shape, 201, np.uint8)) for _ in range(count)]
        dw = [cu(words[offs[k]: offs[k + 1]].view(np.int32)) for k in range(count)]
        bit_sizes = [int(offs[k + 1] - offs[k]) * 32 for k in range(count)]
        if count == 1:
            ci.decompress_image_one_level(inst, outs[0], proc, lps[0], float(steps[0]), dw[0], bit_sizes[0])
        else:
            ci.decompress_images_one_level(inst, outs, proc, lps, [float(s) for s in steps], dw, bit_sizes)
        for k in range(count):
            assert np.array_equal(host(outs[k]), gold[f"{name}_dec{k}"]), (name, k)


def test_heightfield_one_level_vs_reference(gold, inst):
    for name in ("h0", "h3"):
        hf, shift = gold[f"{name}_in"], int(gold[f"{name}_shift"][0])
        ny, nx = hf.shape
        lp = torch.zeros((ny // 2, nx // 2), dtype=torch.int16, device="cuda")
        w, bits = ci.compress_heightfield_one_level(inst, cu(hf), lp, shift)
        assert np.array_equal(host(w[: bits // 32], np.uint32), gold[f"{name}_words"]), name
        assert np.array_equal(host(lp), gold[f"{name}_lp"]), name
        rec = torch.zeros((ny, nx), dtype=torch.int16, device="cuda")
        ci.decompress_heightfield_one_level(inst, rec, lp, shift, w, bits)
        assert np.array_equal(host(rec), gold[f"{name}_dec"]), name
        assert np.array_equal(host(lp), gold[f"{name}_lpdec"]), name
        got = ci.get_lowpass_heightfield(cu(hf), shift + 2)
        assert np.array_equal(host(got), gold[f"{name}_getlp"]), name


# ---------------------------------------------------------- vs the oracle
def test_byte_dwt_vs_oracle(orc):
    img = image((80, 96, 4), 11)
    for c in (0, 3):
        want = orc.dwt_fwd_from_byte(img, c)
        assert np.array_equal(fwd_from_byte(img, c), want), c
        tgt = np.full(img.shape, 9, np.uint8)
        want_t = tgt.copy()
        orc.dwt_inv_to_byte(want * 1.3, want_t, c)
        assert np.array_equal(inv_to_byte(want * 1.3, tgt, c), want_t), c
    vol = np.stack([image((24, 32, 2), 20 + z)[..., :2] for z in range(16)])   # (16, 24, 32, 2)
    want = orc.dwt_fwd_from_byte(vol, 1)
    assert np.array_equal(fwd_from_byte(vol, 1), want)


@pytest.mark.parametrize("shape", [(66, 130, 3), (96, 512, 1), (256, 256, 4), (18, 20, 2)])
def test_lowpass_only_vs_oracle(orc, shape):
    img = image(shape, shape[0])
    ny, nx, ch = shape
    c = ch - 1
    dst = torch.full((ny // 2, nx // 2), float("nan"), dtype=torch.float32, device="cuda")
    cc.dwt_float2d_forward_lowpass_only_from_byte(dst, None, cu(img).view(-1)[c:], nx, ny, ch)
    assert np.array_equal(host(dst), orc.lowpass_from_byte(img, c))
    hf = terrain((ny, nx), nx)
    di = torch.zeros((ny // 2, nx // 2), dtype=torch.int16, device="cuda")
    cc.dwt_int_forward_lowpass_only(di, None, cu(hf), nx, ny)
    assert np.array_equal(host(di), orc.int_lowpass(hf))
    # the image lowpass of all processed channels in one launch
    lp = ci.get_lowpass_image(cu(img), ch)
    assert np.array_equal(host(lp), orc.lowpass_image(img, ch))


def test_lowpass_equals_full_transform_ll():
    img = image((64, 96, 1), 5)
    full = fwd_from_byte(img, 0)
    dst = torch.zeros((32, 48), dtype=torch.float32, device="cuda")
    cc.dwt_float2d_forward_lowpass_only_from_byte(dst, None, cu(img), 96, 64, 1)
    assert np.array_equal(host(dst), full[:32, :48])


def test_bits_ragged_vs_oracle(orc):
    rng = np.random.default_rng(3)
    for n in (1, 31, 33, 1000, 70001):
        v = rng.integers(-32768, 32768, n).astype(np.int16)
        words = (n + 31) // 32
        d, b = cu(v), torch.full((words,), -1, dtype=torch.int32, device="cuda")
        ci.remove_lsb(d, b, n, 3)
        wd, wb = orc.lsb(1, v, np.zeros(words, np.uint32), 3)
        assert np.array_equal(host(d), wd) and np.array_equal(host(b, np.uint32), wb), n
        ci.append_lsb(d, b, n, -3)
        assert np.array_equal(host(d), v), n
        g = torch.zeros((words,), dtype=torch.int32, device="cuda")
        ci.get_lsb(cu(v), g, n)
        assert np.array_equal(host(g, np.uint32), orc.lsb(0, v)[1]), n


@pytest.mark.parametrize("shape,proc,step", [((192, 256, 3), 3, 3.0), ((128, 160, 4), 3, 1.0), ((64, 48, 1), 1, 6.0)])
def test_image_codec_vs_oracle(orc, inst, shape, proc, step):
    img = image(shape, sum(shape))
    lp = orc.lowpass_image(img, proc)
    w_o, bits_o, rec_o = orc.compress_image(img, proc, lp, step)
    d = cu(img)
    w, bits = ci.compress_image_one_level(inst, d, proc, cu(lp), step)
    assert bits == len(w_o) * 32
    assert np.array_equal(host(w[: bits // 32], np.uint32), w_o)
    assert np.array_equal(host(d), rec_o)
    out = cu(np.full(shape, 3, np.uint8))
    ci.decompress_image_one_level(inst, out, proc, cu(lp), step, w, bits)
    want = np.full(shape, 3, np.uint8)
    orc.decompress_image(w_o, bits_o, want, proc, lp, step)
    assert np.array_equal(host(out), want)
    # the encoder's reconstruction is what the decoder produces
    assert np.array_equal(host(out)[..., :proc], rec_o[..., :proc])


def test_images_batch_equals_single(orc, inst):
    shape, proc = (96, 128, 4), 3
    imgs = [image(shape, 40 + k) for k in range(4)]
    steps = [1.0, 2.5, 4.0, 8.0]
    lps = [orc.lowpass_image(im, proc) for im in imgs]
    dimgs = [cu(im) for im in imgs]
    res = ci.compress_images_one_level(inst, dimgs, proc, [cu(lp) for lp in lps], steps)
    for k in range(4):
        w_o, bits_o, rec_o = orc.compress_image(imgs[k], proc, lps[k], steps[k])
        w, bits = res[k]
        assert np.array_equal(host(w[: bits // 32], np.uint32), w_o), k
        assert np.array_equal(host(dimgs[k]), rec_o), k
    outs = [cu(np.zeros(shape, np.uint8)) for _ in range(4)]
    ci.decompress_images_one_level(inst, outs, proc, [cu(lp) for lp in lps], steps, [r[0] for r in res],
                                   [r[1] for r in res])
    for k in range(4):
        assert np.array_equal(host(outs[k])[..., :proc], host(dimgs[k])[..., :proc]), k


@pytest.mark.parametrize("shape,shift", [((256, 256), 0), ((200, 136), 3), ((64, 1024), -2)])
def test_heightfield_one_level_vs_oracle(orc, inst, shape, shift):
    hf = terrain(shape, shape[1] + shift)
    ny, nx = shape
    w_o, bits_o, lp_o = orc.compress_heightfield_one_level(hf, shift)
    lp = torch.zeros((ny // 2, nx // 2), dtype=torch.int16, device="cuda")
    w, bits = ci.compress_heightfield_one_level(inst, cu(hf), lp, shift)
    assert bits == len(w_o) * 32
    assert np.array_equal(host(w[: bits // 32], np.uint32), w_o)
    assert np.array_equal(host(lp), lp_o)
    rec = torch.zeros(shape, dtype=torch.int16, device="cuda")
    ci.decompress_heightfield_one_level(inst, rec, lp, -shift, w, bits)   # -shift restores the lowpass exactly
    assert np.array_equal(host(rec), hf)
    got = ci.get_lowpass_heightfield(cu(hf), shift)
    assert np.array_equal(host(got), orc.lowpass_heightfield(hf, shift))


def test_ycocg_inplace_vs_oracle(orc):
    rng = np.random.default_rng(8)
    for ch in (3, 4):
        px = rng.integers(0, 256, (100001, ch)).astype(np.uint8)
        d = cu(px)
        ci.convert_rgb_to_ycocg(d, d)
        assert np.array_equal(host(d), orc.ycocg(px, True)), ch
        ci.convert_ycocg_to_rgb(d, d)
        assert np.array_equal(host(d), orc.ycocg(orc.ycocg(px, True), False)), ch


def test_image_argument_errors(inst):
    img = cu(np.zeros((33, 64, 3), np.uint8))
    lp = cu(np.zeros((16, 32, 3), np.uint8))
    with pytest.raises(CudaCompressError):
        ci.compress_image_one_level(inst, img, 3, lp, 1.0)            # odd height
    img = cu(np.zeros((32, 64, 3), np.uint8))
    with pytest.raises(CudaCompressError):
        ci.compress_image_one_level(inst, img, 4, lp, 1.0)            # more channels coded than present
    with pytest.raises(CudaCompressError):
        ci.get_lowpass_image(cu(np.zeros((32, 64, 5), np.uint8)), 3)  # 5 channels
    with pytest.raises(CudaCompressError):
        ci.convert_rgb_to_ycocg(cu(np.zeros((10, 2), np.uint8)), cu(np.zeros((10, 2), np.uint8)))
    small = cc.Instance(0, 2, 1024, 128, 14)
    try:
        hf = cu(np.zeros((64, 64), np.int16))
        with pytest.raises(CudaCompressError):                        # 3 band streams needed
            ci.compress_heightfield_one_level(small, hf, torch.zeros((32, 32), dtype=torch.int16, device="cuda"), 0)
    finally:
        small.close()
