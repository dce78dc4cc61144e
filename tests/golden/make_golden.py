"""Generates the golden fixtures in tests/golden/ from the reference's own
code: the reference cudaCompress sources compiled by oracle/ref/Makefile into
oracle/_ref/libref_gpu.so (test infrastructure; never shipped).

    python tests/golden/make_golden.py          # ref_tables.npz (CPU only)
    python tests/golden/make_golden.py --gpu    # + ref_streams.npz, ref_dwt.npz (runs the reference on a GPU)

ref_tables.npz   Huffman tables of the reference's HuffmanEncodeTable::build
                 and writeToBitStream (HuffmanTable.cu:470-596) for seeded
                 histograms and edge cases.
ref_streams.npz  encodeRLHuff / encodeHuff bit streams (Encode.cpp:207-471,
                 648-790) of seeded symbol streams, with their inputs.
ref_dwt.npz      util::dwtFloat3DForward/Inverse, dwtIntForward/Inverse and
                 quantizeToSymbols outputs with their inputs.
ref_volume.npz   the reference's example volume codec (examples/CompressVolume.cpp):
                 compressVolumeFloat / compressVolumeFloatQuantFirst streams with and
                 without doRLEOnlyOnLvl0, their reconstructions, and the multi-channel
                 decoders' outputs (python tests/golden/make_golden.py --gpu --only volume).
                 Inputs are seeded fields (cudacompress_b200.fields), stored as seed +
                 SHA-256 of the generated array.
ref_digests.json SHA-256 digests and word counts of the reference's streams (and
                 reconstructions) at the scope's full sizes: the 128^3 volume, the
                 3 x 256^3 vector field at q0 in {0.002, 0.01, 0.05}, a sample of the
                 uneven bricks and the 2048^2 lossless heightfield
                 (python tests/golden/make_golden.py --gpu --only digests).  The
                 streams themselves are megabytes, so only their digests are kept;
                 inputs are regenerated from the recorded generator parameters.
ref_image.npz    the 2D image side: util byte-DWT, lowpass-only, byte-image quantizer,
                 YCoCg and Bits outputs, and the examples' one-level image and
                 heightfield codecs (CompressImage.cpp, CompressHeightfield.cpp):
                 streams, reconstructions and lowpass bands, with their inputs
                 (python tests/golden/make_golden.py --gpu --only image).
"""
import argparse
import hashlib
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
TESTS = os.path.dirname(HERE)
sys.path.insert(0, TESTS)
sys.path.insert(0, os.path.dirname(TESTS))

from helpers import bind_build, load_ref_gpu_lib, random_histograms, run_build, symbol_streams  # noqa: E402

c = ctypes


def edge_histograms():
    """Degenerate and boundary histograms (bins, symbolMax, log2Max)."""
    out = []
    h = np.zeros(1, np.uint32); out.append((h, 0, 14))                     # empty
    h = np.array([5], np.uint32); out.append((h, 0, 14))                   # one symbol 0
    h = np.zeros(100, np.uint32); h[99] = 3; out.append((h, 99, 14))       # one symbol
    h = np.zeros(10, np.uint32); h[[2, 9]] = [1, 1]; out.append((h, 9, 14))
    h = np.ones(16384, np.uint32); out.append((h, 16383, 14))             # full range, all ties
    h = np.zeros(65536, np.uint32); h[[0, 7, 65535]] = [3, 2, 9]; out.append((h, 65535, 16))
    fib = [1, 1]
    while len(fib) < 31:
        fib.append(fib[-1] + fib[-2])
    h = np.array(fib, np.uint32); out.append((h, 30, 14))                 # 30-bit codes
    h = np.zeros(300, np.uint32); h[::3] = np.arange(100) % 4 + 1; out.append((h, int(np.nonzero(h)[0][-1]), 14))
    return out


def make_tables(ref):
    f = bind_build(ref, "ref_huffman_build")
    cases = [(h, smax, 14 if smax < (1 << 14) else 16) for h, smax in random_histograms(120, seed=2024)]
    cases += edge_histograms()
    hists, hoff, meta, lens, cws, tws, twoff = [], [0], [], [], [], [], [0]
    for h, smax, log2max in cases:
        r, cw, ln, tw, tb = run_build(f, h, smax, log2max)
        hists.append(h.astype(np.uint32)); hoff.append(hoff[-1] + len(h))
        meta.append([smax, log2max, r, tb])
        lens.append(ln.astype(np.uint8)); cws.append(cw.astype(np.uint32))
        tws.append(tw.astype(np.uint32)); twoff.append(twoff[-1] + len(tw))
    np.savez_compressed(os.path.join(HERE, "ref_tables.npz"),
                        hist=np.concatenate(hists), hist_off=np.array(hoff, np.int64),
                        meta=np.array(meta, np.int64), lengths=np.concatenate(lens), codewords=np.concatenate(cws),
                        table_words=np.concatenate(tws), table_off=np.array(twoff, np.int64))
    print(f"ref_tables.npz: {len(cases)} tables")


# kind (0 RLHuff, 1 Huff), symbol dtype, log2Max, cb, S, n, generator, seed, start bit position
STREAM_CASES = [
    (0, np.uint16, 14, 128, 7, 4096, "sparse", 1),
    (0, np.uint16, 14, 128, 7, 4999, "laplace", 2),
    (0, np.uint16, 14, 32, 3, 3001, "sparse", 3),
    (0, np.uint16, 14, 64, 3, 3001, "dense", 4),
    (0, np.uint16, 14, 256, 3, 3001, "laplace", 5),
    (0, np.uint16, 14, 128, 4, 20000, "runs", 6),
    (0, np.uint16, 14, 128, 2, 70001, "laplace", 7),
    (0, np.uint16, 14, 128, 1, 1000, "zeros", 8),
    (0, np.uint16, 14, 128, 3, 1000, "zeros", 9),
    (0, np.uint16, 14, 128, 6, 1000, "zeros", 10),
    (0, np.uint16, 14, 128, 3, 1000, "single", 11),
    (0, np.uint16, 16, 128, 2, 5000, "dense", 12),
    (0, np.uint32, 20, 128, 3, 4000, "laplace", 13),
    (1, np.uint16, 14, 128, 1, 4096, "laplace", 14),
    (1, np.uint16, 14, 128, 3, 4099, "dense", 15),
    (1, np.uint16, 14, 64, 2, 777, "laplace", 16),
    (1, np.uint16, 14, 128, 1, 1000, "single", 17),
    (1, np.uint16, 14, 128, 1, 1000, "zeros", 18),
    (1, np.uint32, 20, 128, 2, 3000, "dense", 19),
    (1, np.uint16, 14, 128, 1, 500, "dense", 20),
]
START_BITS = {14: 13, 16: 0, 17: 7}   # Huff cases written after a prefix ending at this bit (mod 32)


def case_input(kind, dt, log2max, cb, S, n, gen, seed):
    a = symbol_streams(gen, S, n, seed, dtype=np.uint32, max_symbol=min(1 << log2max, 5000))
    if seed == 12:                      # 2^16 bins with symbol 65535 present (odd and even counts)
        a[0, :3] = 65535
        a[1, :4] = 65535
    if seed == 19:
        a[:, 0] = (1 << 20) - 1
    if seed == 20:                      # symbol >= 2^log2Max: the reference's encode fails
        a[0, 5] = 1 << log2max
    mixed = seed == 9                    # one empty stream among nonempty ones
    if mixed:
        a[1] = symbol_streams("sparse", 1, n, 99, dtype=np.uint32)[0]
    return np.ascontiguousarray(a.astype(dt))


def make_streams(ref):
    import torch
    f = ref.ref_encode_strided
    f.restype = c.c_int
    f.argtypes = [c.c_void_p, c.c_int, c.c_int, c.c_void_p, c.c_uint32, c.c_uint32, c.c_uint32,
                  np.ctypeslib.ndpointer(np.uint32, flags="C"), c.c_uint32, c.POINTER(c.c_uint32),
                  c.POINTER(c.c_uint32)]
    ref.ref_create.restype = c.c_void_p
    ref.ref_create.argtypes = [c.c_int, c.c_uint32, c.c_uint32, c.c_uint32, c.c_uint32]
    ref.ref_destroy.argtypes = [c.c_void_p]
    out = {}
    for i, (kind, dt, log2max, cb, S, n, gen, seed) in enumerate(STREAM_CASES):
        a = case_input(kind, dt, log2max, cb, S, n, gen, seed)
        stride = (n + 7) // 8 * 8 + 8
        # slack between streams (padding writes) and 64 Ki elements after the last one
        flat = np.zeros(S * stride + 65536, dt)
        flat[: S * stride].reshape(S, stride)[:, :n] = a
        tt = torch.from_numpy(flat.view(np.int16 if dt == np.uint16 else np.int32)).cuda()
        inst = ref.ref_create(0, S, n, cb, log2max)
        assert inst, "reference createInstance failed"
        r0 = START_BITS.get(seed, 0)
        prefix = np.array([0x9E3779B9, 0x7F4A7C15], np.uint32)
        cap = S * n * 4 + 8192
        words = np.zeros(cap, np.uint32)
        size = c.c_uint32(0)
        pos = c.c_uint32(0)
        if r0:
            words[:2] = prefix
            size.value = 32 + r0
            pos.value = 32 + r0
        rc = f(inst, kind, np.dtype(dt).itemsize, c.c_void_p(tt.data_ptr()), S, n, stride, words, cap,
               c.byref(size), c.byref(pos))
        torch.cuda.synchronize()
        ref.ref_destroy(inst)
        out[f"c{i}_meta"] = np.array([kind, np.dtype(dt).itemsize, log2max, cb, S, n, 32 + r0 if r0 else 0,
                                      rc, size.value, pos.value], np.int64)
        out[f"c{i}_in"] = a
        out[f"c{i}_out"] = words[: (size.value + 31) // 32].copy() if rc == 0 else np.zeros(0, np.uint32)
        out[f"c{i}_prefix"] = prefix
        print(f"case {i}: kind {kind} S {S} n {n} rc {rc} bits {size.value}")
    out["count"] = np.array([len(STREAM_CASES)], np.int64)
    np.savez_compressed(os.path.join(HERE, "ref_streams.npz"), **out)


def make_dwt(ref):
    import torch
    from cudacompress_b200 import fields
    for name in ["ref_dwt_float3d_fwd", "ref_dwt_float3d_inv"]:
        getattr(ref, name).argtypes = [c.c_void_p] * 4 + [c.c_int] * 3
    for name in ["ref_dwt_int_fwd", "ref_dwt_int_inv"]:
        getattr(ref, name).argtypes = [c.c_void_p] * 3 + [c.c_int] * 3
    ref.ref_quantize_to_symbols.argtypes = [c.c_void_p, c.c_void_p, c.c_uint32, c.c_uint32, c.c_uint32, c.c_float,
                                            c.c_uint32, c.c_uint32]
    P = lambda t: c.c_void_p(t.data_ptr())  # noqa: E731
    out = {}
    shapes = [(16, 24, 32), (32, 32, 32), (8, 16, 64)]
    for i, (nz, ny, nx) in enumerate(shapes):
        vol = fields.turbulence_field(max(nx, ny, nz), 64, 8, seed=300 + i)[:nz, :ny, :nx].copy()
        src = torch.from_numpy(vol).cuda()
        dst, b1, b2 = (torch.empty_like(src) for _ in range(3))
        ref.ref_dwt_float3d_fwd(P(dst), P(b2), P(b1), P(src), nx, ny, nz)
        fwd = dst.cpu().numpy()
        inv_t = torch.empty_like(src)
        ref.ref_dwt_float3d_inv(P(inv_t), P(b2), P(b1), P(dst), nx, ny, nz)
        out[f"f{i}_in"], out[f"f{i}_fwd"], out[f"f{i}_inv"] = vol, fwd, inv_t.cpu().numpy()
        step = 0.01
        sym = torch.zeros(vol.size + 64, dtype=torch.int16, device="cuda")
        ref.ref_quantize_to_symbols(P(sym), P(dst), nx, ny, nz, step, nx, nx * ny)
        out[f"q{i}_sym"] = sym[: vol.size].cpu().numpy().view(np.uint16).reshape(vol.shape)
        out[f"q{i}_step"] = np.array([step], np.float32)
    ishapes = [(1, 64, 48), (16, 16, 16), (1, 40, 96)]
    for i, (nz, ny, nx) in enumerate(ishapes):
        rng = np.random.default_rng(400 + i)
        img = np.cumsum(np.cumsum(rng.integers(-40, 41, (nz, ny, nx)), axis=1), axis=2).astype(np.int16)
        src = torch.from_numpy(img).cuda()
        dst, buf = torch.empty_like(src), torch.empty_like(src)
        ref.ref_dwt_int_fwd(P(dst), P(buf), P(src), nx, ny, nz)
        fwd = dst.cpu().numpy()
        inv_t = torch.empty_like(src)
        ref.ref_dwt_int_inv(P(inv_t), P(buf), P(dst), nx, ny, nz)
        out[f"i{i}_in"], out[f"i{i}_fwd"], out[f"i{i}_inv"] = img, fwd, inv_t.cpu().numpy()
    np.savez_compressed(os.path.join(HERE, "ref_dwt.npz"), **out)
    print("ref_dwt.npz written")


# Whole-volume cases of the reference's example codec (examples/CompressVolume.cpp):
# (name, (nz, ny, nx), levels, step, rleOnlyLevel0, quantFirst, keep the reconstruction)
VOLUME_CASES = [
    ("f2", (16, 16, 32), 2, 0.01, 0, 0, True),
    ("f2r", (16, 16, 32), 2, 0.01, 1, 0, True),
    ("f3r", (32, 32, 32), 3, 0.01, 1, 0, True),
    ("q2", (16, 16, 32), 2, 0.05, 0, 1, True),
    ("q2r", (16, 16, 32), 2, 0.05, 1, 1, True),
    ("q3", (32, 32, 32), 3, 0.05, 0, 1, False),   # odd levels: the reference's decompress reads the other buffer
]
# multi-channel decodes: (name, (nz, ny, nx), levels, steps per channel, rleOnlyLevel0, quantFirst)
MULTI_CASES = [
    ("mf", (16, 16, 32), 2, (0.01, 0.02, 0.005), 0, 0),
    ("mfr", (16, 16, 32), 2, (0.01, 0.02, 0.005), 1, 0),
    ("mq", (16, 16, 32), 2, (0.05, 0.1, 0.03), 0, 1),
]


def make_volume(ref, out_dir):
    import torch
    from cudacompress_b200 import fields
    u32p = c.POINTER(c.c_uint32)
    ref.ref_volume_compress.argtypes = [c.c_void_p, c.c_uint32, c.c_uint32, c.c_uint32, c.c_uint32, c.c_float,
                                        c.c_int, c.c_int, u32p, c.c_uint32, u32p]
    ref.ref_volume_decompress.argtypes = [c.c_void_p, c.c_uint32, c.c_uint32, c.c_uint32, c.c_uint32, c.c_float,
                                          c.c_int, c.c_int, u32p, c.c_uint32]
    ref.ref_volume_decompress_multichannel.argtypes = [c.c_void_p, c.c_void_p, u32p, c.POINTER(c.c_float), c.c_uint32,
                                                       c.c_uint32, c.c_uint32, c.c_uint32, c.c_uint32, c.c_int, c.c_int]
    P = lambda t: c.c_void_p(t.data_ptr())  # noqa: E731

    def vol_for(shape, seed):
        nz, ny, nx = shape
        return fields.turbulence_field(max(shape), 64, 8, seed=seed)[:nz, :ny, :nx].copy()

    def compress(v, levels, q, rle, qf):
        nz, ny, nx = v.shape
        cap = v.size * 4 + 65536
        words = np.zeros(cap, np.uint32)
        nw = c.c_uint32()
        r = ref.ref_volume_compress(P(torch.from_numpy(v).cuda()), nx, ny, nz, levels, q, rle, qf,
                                    words.ctypes.data_as(u32p), cap, c.byref(nw))
        assert r == 0, r
        return words[: nw.value].copy()

    def sha(v):
        return np.frombuffer(hashlib.sha256(v.tobytes()).digest(), np.uint8)

    # inputs are not stored: they are regenerated from their seeds (the hash guards the generator)
    out = {}
    for i, (name, shape, levels, q, rle, qf, keep) in enumerate(VOLUME_CASES):
        v = vol_for(shape, 500 + i)
        w = compress(v, levels, q, rle, qf)
        out[f"{name}_seed"], out[f"{name}_insha"], out[f"{name}_words"] = np.array([500 + i], np.int64), sha(v), w
        out[f"{name}_meta"] = np.array([levels, rle, qf], np.int32)
        out[f"{name}_q"] = np.array([q], np.float32)
        if keep:
            nz, ny, nx = shape
            rec = torch.full(shape, float("nan"), dtype=torch.float32, device="cuda")
            r = ref.ref_volume_decompress(P(rec), nx, ny, nz, levels, q, rle, qf, w.ctypes.data_as(u32p), len(w))
            assert r == 0, r
            out[f"{name}_rec"] = rec.cpu().numpy()
    for i, (name, shape, levels, qs, rle, qf) in enumerate(MULTI_CASES):
        nz, ny, nx = shape
        seeds = [600 + 10 * i + k for k in range(len(qs))]
        vols = [vol_for(shape, sd) for sd in seeds]
        ws = [compress(v, levels, q, rle, qf) for v, q in zip(vols, qs)]
        recs = [torch.full(shape, float("nan"), dtype=torch.float32, device="cuda") for _ in qs]
        ptrs = (c.c_void_p * len(qs))(*[r.data_ptr() for r in recs])
        wp = (u32p * len(qs))(*[w.ctypes.data_as(u32p) for w in ws])
        nws = (c.c_uint32 * len(qs))(*[len(w) for w in ws])
        qa = (c.c_float * len(qs))(*qs)
        r = ref.ref_volume_decompress_multichannel(ptrs, wp, nws, qa, len(qs), nx, ny, nz, levels, rle, qf)
        assert r == 0, r
        out[f"{name}_meta"] = np.array([levels, rle, qf, len(qs)], np.int32)
        out[f"{name}_q"] = np.array(qs, np.float32)
        for k in range(len(qs)):
            out[f"{name}_seed{k}"], out[f"{name}_insha{k}"] = np.array([seeds[k]], np.int64), sha(vols[k])
            out[f"{name}_words{k}"] = ws[k]
            out[f"{name}_rec{k}"] = recs[k].cpu().numpy()
    np.savez_compressed(os.path.join(out_dir, "ref_volume.npz"), **out)
    print("ref_volume.npz written")


def make_digests(ref, out_dir):
    """Digests of the reference's streams and reconstructions at the full
    sizes of the scope (cases in digest_cases.py)."""
    import json
    import torch
    import digest_cases as dc
    u32p = c.POINTER(c.c_uint32)
    ref.ref_volume_compress.argtypes = [c.c_void_p, c.c_uint32, c.c_uint32, c.c_uint32, c.c_uint32, c.c_float,
                                        c.c_int, c.c_int, u32p, c.c_uint32, u32p]
    ref.ref_volume_decompress.argtypes = [c.c_void_p, c.c_uint32, c.c_uint32, c.c_uint32, c.c_uint32, c.c_float,
                                          c.c_int, c.c_int, u32p, c.c_uint32]
    ref.ref_heightfield_compress.argtypes = [c.c_void_p, c.c_uint32, c.c_uint32, c.c_uint32, u32p, c.c_uint32, u32p]
    P = lambda t: c.c_void_p(t.data_ptr())  # noqa: E731

    def volume(v, levels, q):
        nz, ny, nx = v.shape
        cap = v.size * 2 + 65536
        words = np.zeros(cap, np.uint32)
        nw = c.c_uint32()
        d = torch.from_numpy(v).cuda()
        r = ref.ref_volume_compress(P(d), nx, ny, nz, levels, q, 0, 0, words.ctypes.data_as(u32p), cap, c.byref(nw))
        assert r == 0, r
        w = words[: nw.value].copy()
        rec = torch.full(v.shape, float("nan"), dtype=torch.float32, device="cuda")
        r = ref.ref_volume_decompress(P(rec), nx, ny, nz, levels, q, 0, 0, w.ctypes.data_as(u32p), len(w))
        assert r == 0, r
        return w, rec.cpu().numpy()

    out = {"volumes": [], "bricks": None, "heightfield": None}
    for case in dc.volume_cases():
        v = dc.volume_input(case)
        w, rec = volume(v, case["levels"], case["q0"])
        out["volumes"].append(dict(case, input_sha256=dc.sha256(v), words=int(len(w)), stream_sha256=dc.sha256(w),
                                   recon_sha256=dc.sha256(rec)))
        print(case["name"], len(w), "words")
    bricks, qs = dc.brick_inputs()
    items = []
    for i, (b, q) in enumerate(zip(bricks, qs)):
        w, rec = volume(b, dc.BRICK_LEVELS, q)
        items.append(dict(index=i, shape=list(b.shape), q0=q, input_sha256=dc.sha256(b), words=int(len(w)),
                          stream_sha256=dc.sha256(w), recon_sha256=dc.sha256(rec)))
    out["bricks"] = dict(count=dc.BRICK_COUNT, seed=dc.BRICK_SEED, levels=dc.BRICK_LEVELS, items=items)
    img = dc.heightfield_input()
    n = dc.HEIGHTFIELD["n"]
    cap = img.size + 65536
    words = np.zeros(cap, np.uint32)
    nw = c.c_uint32()
    r = ref.ref_heightfield_compress(P(torch.from_numpy(img).cuda()), n, n, dc.HEIGHTFIELD["levels"],
                                     words.ctypes.data_as(u32p), cap, c.byref(nw))
    assert r == 0, r
    w = words[: nw.value]
    out["heightfield"] = dict(dc.HEIGHTFIELD, input_sha256=dc.sha256(img), words=int(len(w)),
                              stream_sha256=dc.sha256(w))
    with open(os.path.join(out_dir, "ref_digests.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("ref_digests.json written")


def test_image(shape, seed):
    """Seeded smooth 8-bit test image (y, x, channels): two plane waves per
    channel plus uniform noise, clipped to [0, 255]."""
    ny, nx, ch = shape
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:ny, 0:nx].astype(np.float64)
    out = np.empty(shape, np.uint8)
    for c in range(ch):
        k = rng.uniform(0.02, 0.2, 4)
        v = 128 + 70 * np.sin(k[0] * x + k[1] * y) + 40 * np.cos(k[2] * x - k[3] * y) + rng.uniform(-12, 12, (ny, nx))
        out[..., c] = np.clip(np.rint(v), 0, 255).astype(np.uint8)
    return out


def test_heightfield(shape, seed):
    """Seeded int16 terrain-like field: cumulative sums of small steps."""
    rng = np.random.default_rng(seed)
    v = np.cumsum(np.cumsum(rng.integers(-6, 7, shape), axis=0), axis=1)
    return np.clip(v, -30000, 30000).astype(np.int16)


IMAGE_CODEC_CASES = [
    # name, (ny, nx, channels), channels coded, steps per image
    ("c3", (48, 64, 3), 3, (4.0,)),
    ("c4", (64, 96, 4), 3, (2.0,)),
    ("m3", (64, 64, 4), 3, (2.0, 4.0, 8.0)),
]
HEIGHTFIELD_CASES = [("h0", (128, 512), 0), ("h3", (64, 1024), 3)]


def make_image(ref, out_dir):
    import torch
    i32, u32, f32 = c.c_int, c.c_uint32, c.c_float
    vp = c.c_void_p
    u32p = c.POINTER(c.c_uint32)
    ref.ref_dwt_float_fwd_from_byte.argtypes = [vp] * 4 + [i32] * 4
    ref.ref_dwt_float_inv_to_byte.argtypes = [vp] * 4 + [i32] * 4
    ref.ref_dwt_float_inv_from_symbols_to_byte.argtypes = [vp] * 5 + [f32] + [i32] * 4
    ref.ref_dwt_float2d_lowpass_from_byte.argtypes = [vp] * 3 + [i32] * 3
    ref.ref_dwt_int_lowpass.argtypes = [vp] * 3 + [i32] * 2
    ref.ref_float_to_byte_2d.argtypes = [vp, u32, u32, vp, u32, u32, u32]
    ref.ref_byte_to_float_2d.argtypes = [vp, vp, u32, u32, u32, u32, u32]
    ref.ref_quantize_difference_2d.argtypes = [vp, vp, f32, vp, u32, u32, u32, u32, u32, i32, i32]
    ref.ref_unquantize_difference_2d.argtypes = [vp, vp, f32, vp, u32, u32, u32, u32, u32, i32]
    ref.ref_ycocg.argtypes = [vp, vp, i32, i32, i32]
    ref.ref_lsb.argtypes = [i32, vp, vp, u32, c.c_int16]
    ref.ref_images_compress.argtypes = [vp, vp, vp, u32, u32, u32, u32, u32, u32p, u32, u32p]
    ref.ref_images_decompress.argtypes = [vp, vp, vp, u32, u32, u32, u32, u32, u32p, u32p]
    ref.ref_get_lowpass_image.argtypes = [vp, u32, u32, u32, u32, vp]
    ref.ref_heightfield_compress_one_level.argtypes = [vp, u32, u32, vp, c.c_int16, u32p, u32, u32p]
    ref.ref_heightfield_decompress_one_level.argtypes = [vp, u32, u32, vp, c.c_int16, u32p, u32]
    ref.ref_get_lowpass_heightfield.argtypes = [vp, u32, u32, vp, c.c_int16]
    P = lambda t: c.c_void_p(t.data_ptr())  # noqa: E731
    cu = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    out = {}

    # byte DWT forward / inverse, 2D (3 channels) and 3D (2 channels)
    for name, shape, ch in [("b2", (48, 64), 3), ("b3", (16, 16, 32), 2)]:
        dims = shape if len(shape) == 3 else (1,) + shape
        nz, ny, nx = dims
        img = test_image((nz * ny, nx, ch), 700 + len(shape)).reshape(dims + (ch,))
        src = cu(img)
        out[f"{name}_in"] = img
        for cc in range(ch):
            dst, b1, b2 = (torch.empty(dims, dtype=torch.float32, device="cuda") for _ in range(3))
            ref.ref_dwt_float_fwd_from_byte(P(dst), P(b2), P(b1), c.c_void_p(src.data_ptr() + cc), nx, ny, nz, ch)
            out[f"{name}_fwd{cc}"] = dst.cpu().numpy()
        # inverse of channel 0's coefficients, scaled to reach the clamp, into channel 1 of a patterned image
        coef = torch.from_numpy(out[f"{name}_fwd0"] * 1.7).cuda()
        tgt = cu(np.full(dims + (ch,), 77, np.uint8))
        b1, b2 = (torch.empty(dims, dtype=torch.float32, device="cuda") for _ in range(2))
        ref.ref_dwt_float_inv_to_byte(c.c_void_p(tgt.data_ptr() + 1), P(b2), P(b1), P(coef), nx, ny, nz, ch)
        out[f"{name}_invcoef"] = out[f"{name}_fwd0"] * np.float32(1.7)
        out[f"{name}_inv"] = tgt.cpu().numpy()
        # inverse from symbols to bytes: lowpass in a full-size array (default pitches), random bands
        rng = np.random.default_rng(710 + len(shape))
        nb = 7 if nz > 1 else 3
        hz = max(nz // 2, 1)
        bands = rng.integers(0, 40, (nb, hz, ny // 2, nx // 2)).astype(np.uint16)
        lpfull = (out[f"{name}_fwd0"]).copy()
        dband = [cu(bands[k]) for k in range(nb)]
        ptrs = torch.tensor([t.data_ptr() for t in dband], dtype=torch.int64, device="cuda")
        tgt = cu(np.full(dims + (ch,), 55, np.uint8))
        dlp = cu(lpfull)
        ref.ref_dwt_float_inv_from_symbols_to_byte(c.c_void_p(tgt.data_ptr() + ch - 1), P(b2), P(b1), P(dlp),
                                                   P(ptrs), 0.75, nx, ny, nz, ch)
        out[f"{name}_symbands"], out[f"{name}_symlp"], out[f"{name}_symout"] = bands, lpfull, tgt.cpu().numpy()

    # lowpass-only transforms
    for name, (ny, nx, ch, cc) in [("lf", (48, 64, 3, 1)), ("lfr", (72, 200, 1, 0))]:
        img = test_image((ny, nx, ch), 720 + nx)
        dst = torch.full((ny // 2, nx // 2), float("nan"), dtype=torch.float32, device="cuda")
        buf = torch.empty((ny, nx), dtype=torch.float32, device="cuda")
        src = cu(img)
        ref.ref_dwt_float2d_lowpass_from_byte(P(dst), P(buf), c.c_void_p(src.data_ptr() + cc), nx, ny, ch)
        out[f"{name}_in"], out[f"{name}_meta"], out[f"{name}_out"] = img, np.array([cc], np.int32), dst.cpu().numpy()
    for name, (ny, nx) in [("li", (128, 512)), ("li2", (64, 1024))]:
        hf = test_heightfield((ny, nx), 730 + nx)
        dst = torch.zeros((ny // 2, nx // 2), dtype=torch.int16, device="cuda")
        buf = torch.empty((ny, nx), dtype=torch.int16, device="cuda")
        dhf = cu(hf)
        ref.ref_dwt_int_lowpass(P(dst), P(buf), P(dhf), nx, ny)
        out[f"{name}_in"], out[f"{name}_out"] = hf, dst.cpu().numpy()

    # byte-image quantizers (40 x 24 region, row pitch 48, 3 channels, channel 1)
    nx, ny, pitch, chc, ch = 40, 24, 48, 3, 1
    rng = np.random.default_rng(740)
    data = rng.normal(0, 40, (ny, pitch)).astype(np.float32)
    refimg = rng.integers(0, 256, (ny, nx, chc)).astype(np.uint8)
    qb = torch.zeros((ny, nx, chc), dtype=torch.uint8, device="cuda")
    d3, dref = cu(data * 3), cu(refimg)
    ref.ref_float_to_byte_2d(P(qb), chc, ch, P(d3), nx, ny, pitch)
    fb = torch.zeros((ny, pitch), dtype=torch.float32, device="cuda")
    ref.ref_byte_to_float_2d(P(fb), P(dref), chc, ch, nx, ny, pitch)
    out["q_data"], out["q_ref"], out["q_f2b"], out["q_b2f"] = data, refimg, qb.cpu().numpy(), fb.cpu().numpy()
    for t in (0, 1):
        for rt in (0, 1):
            d = cu(data)
            sym = torch.zeros((ny, nx), dtype=torch.int16, device="cuda")
            ref.ref_quantize_difference_2d(P(sym), P(d), 3.0, P(dref), chc, ch, nx, ny, pitch, t, rt)
            out[f"q_sym{t}{rt}"] = sym.cpu().numpy().view(np.uint16)
            out[f"q_data{t}{rt}"] = d.cpu().numpy()
        back = cu(np.full((ny, pitch), -1.0, np.float32))
        dsym = cu(out[f"q_sym{t}0"].view(np.int16))
        ref.ref_unquantize_difference_2d(P(back), P(dsym), 3.0, P(dref), chc, ch, nx, ny, pitch, t)
        out[f"q_unq{t}"] = back.cpu().numpy()

    # YCoCg, every byte value, both pixel sizes and directions
    rng = np.random.default_rng(750)
    for chn in (3, 4):
        px = rng.integers(0, 256, (1000, chn)).astype(np.uint8)
        dpx = cu(px)
        for d in (1, 0):
            dst = torch.zeros_like(dpx)
            ref.ref_ycocg(P(dst), P(dpx), 1000, chn, d)
            out[f"y{chn}_{d}"] = dst.cpu().numpy()
        out[f"y{chn}_in"] = px

    # Bits on 8192 elements (whole blocks of 4096, as the reference requires)
    n = 8192
    vals = rng.integers(-3000, 3000, n).astype(np.int16)
    bits0 = rng.integers(0, 2 ** 32, n // 32, dtype=np.uint64).astype(np.uint32)
    out["l_in"], out["l_bits_in"] = vals, bits0
    for mode, shift in [(0, 0), (1, 0), (1, 3), (2, 0), (2, -5), (3, 7)]:
        d = cu(vals)
        b = cu(bits0.view(np.int32)) if mode == 2 else torch.zeros(n // 32, dtype=torch.int32, device="cuda")
        ref.ref_lsb(mode, P(d), P(b), n, shift)
        out[f"l{mode}_{shift}_data"] = d.cpu().numpy()
        out[f"l{mode}_{shift}_bits"] = b.cpu().numpy().view(np.uint32)
    d = cu(vals)
    ref.ref_lsb(1, P(d), None, n, 2)
    out["l1n_2_data"] = d.cpu().numpy()

    # one image level: single images and a batch of three
    for name, shape, proc, steps in IMAGE_CODEC_CASES:
        ny, nx, ch = shape
        count = len(steps)
        imgs = [test_image(shape, 760 + 10 * IMAGE_CODEC_CASES.index((name, shape, proc, steps)) + k)
                for k in range(count)]
        dimg = [cu(im) for im in imgs]
        drefs = []
        for k in range(count):
            lp = torch.zeros((ny // 2, nx // 2, ch), dtype=torch.uint8, device="cuda")
            r = ref.ref_get_lowpass_image(P(dimg[k]), nx, ny, ch, proc, P(lp))
            assert r == 0, r
            drefs.append(lp)
        cap = nx * ny * ch * 4 * count + 65536
        words = np.zeros(cap, np.uint32)
        offs = np.zeros(count + 1, np.uint32)
        ip = (c.c_void_p * count)(*[t.data_ptr() for t in dimg])
        rp = (c.c_void_p * count)(*[t.data_ptr() for t in drefs])
        qs = (c.c_float * count)(*steps)
        r = ref.ref_images_compress(ip, rp, qs, count, nx, ny, ch, proc, words.ctypes.data_as(u32p), cap,
                                    offs.ctypes.data_as(u32p))
        assert r == 0, r
        recon = [t.cpu().numpy() for t in dimg]
        outs = [cu(np.full(shape, 201, np.uint8)) for _ in range(count)]
        op = (c.c_void_p * count)(*[t.data_ptr() for t in outs])
        r = ref.ref_images_decompress(op, rp, qs, count, nx, ny, ch, proc, words.ctypes.data_as(u32p),
                                      offs.ctypes.data_as(u32p))
        assert r == 0, r
        out[f"{name}_meta"] = np.array([proc, count], np.int32)
        out[f"{name}_steps"] = np.array(steps, np.float32)
        out[f"{name}_offsets"] = offs
        out[f"{name}_words"] = words[: offs[-1]].copy()
        for k in range(count):
            out[f"{name}_in{k}"], out[f"{name}_lp{k}"] = imgs[k], drefs[k].cpu().numpy()
            out[f"{name}_rec{k}"], out[f"{name}_dec{k}"] = recon[k], outs[k].cpu().numpy()

    # one heightfield level and its lowpass
    for name, (ny, nx), shift in HEIGHTFIELD_CASES:
        hf = test_heightfield((ny, nx), 780 + shift)
        dimg = cu(hf)
        lp = torch.zeros((ny // 2, nx // 2), dtype=torch.int16, device="cuda")
        cap = nx * ny + 65536
        words = np.zeros(cap, np.uint32)
        nw = c.c_uint32()
        r = ref.ref_heightfield_compress_one_level(P(dimg), nx, ny, P(lp), shift, words.ctypes.data_as(u32p), cap,
                                                   c.byref(nw))
        assert r == 0, r
        out[f"{name}_in"], out[f"{name}_lp"] = hf, lp.cpu().numpy()
        out[f"{name}_words"] = words[: nw.value].copy()
        rec = torch.zeros_like(dimg)
        r = ref.ref_heightfield_decompress_one_level(P(rec), nx, ny, P(lp), shift, words.ctypes.data_as(u32p),
                                                     nw.value)
        assert r == 0, r
        out[f"{name}_dec"], out[f"{name}_lpdec"] = rec.cpu().numpy(), lp.cpu().numpy()
        lp2 = torch.zeros_like(lp)
        r = ref.ref_get_lowpass_heightfield(P(dimg), nx, ny, P(lp2), shift + 2)
        assert r == 0, r
        out[f"{name}_getlp"] = lp2.cpu().numpy()
        out[f"{name}_shift"] = np.array([shift], np.int32)
    np.savez_compressed(os.path.join(out_dir, "ref_image.npz"), **out)
    print("ref_image.npz written")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpu", action="store_true", help="also run the reference's GPU code")
    ap.add_argument("--only", choices=["volume", "image", "digests"], help="only the whole-volume or image fixtures (GPU)")
    ap.add_argument("--out", default=HERE, help="output directory")
    args = ap.parse_args()
    ref = load_ref_gpu_lib()
    if ref is None:
        sys.exit("oracle/_ref/libref_gpu.so missing: run `make -C oracle/ref` first")
    if args.only == "volume":
        make_volume(ref, args.out)
        return
    if args.only == "image":
        make_image(ref, args.out)
        return
    if args.only == "digests":
        make_digests(ref, args.out)
        return
    make_tables(ref)
    if args.gpu:
        make_streams(ref)
        make_dwt(ref)
        make_volume(ref, args.out)
        make_image(ref, args.out)
        make_digests(ref, args.out)


if __name__ == "__main__":
    main()
