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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpu", action="store_true", help="also run the reference's GPU code")
    ap.add_argument("--only", choices=["volume"], help="only the whole-volume fixtures (GPU)")
    ap.add_argument("--out", default=HERE, help="output directory")
    args = ap.parse_args()
    ref = load_ref_gpu_lib()
    if ref is None:
        sys.exit("oracle/_ref/libref_gpu.so missing: run `make -C oracle/ref` first")
    if args.only == "volume":
        make_volume(ref, args.out)
        return
    make_tables(ref)
    if args.gpu:
        make_streams(ref)
        make_dwt(ref)
        make_volume(ref, args.out)


if __name__ == "__main__":
    main()
