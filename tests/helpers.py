"""Shared test helpers: ctypes loaders for the oracle, the reference build and
the self-test library, plus histogram generators."""
import ctypes
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
U32P = np.ctypeslib.ndpointer(np.uint32, flags="C")
U16P = np.ctypeslib.ndpointer(np.uint16, flags="C")
F32P = np.ctypeslib.ndpointer(np.float32, flags="C")
F64P = np.ctypeslib.ndpointer(np.float64, flags="C")
I16P = np.ctypeslib.ndpointer(np.int16, flags="C")


def _load(path):
    full = os.path.join(ROOT, path)
    if not os.path.exists(full):
        return None
    return ctypes.CDLL(full)


def load_oracle():
    lib = _load("oracle/liboracle.so")
    if lib is None:
        import subprocess
        subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle")])
        lib = _load("oracle/liboracle.so")
    return lib


def load_ref_gpu_lib():
    """The reference library built from the reference sources (may be absent)."""
    return _load("oracle/_ref/libref_gpu.so")


def load_selftest():
    return _load("cudacompress_b200/_lib/libcc_selftest.so")


def bind_build(lib, name):
    f = getattr(lib, name)
    f.restype = ctypes.c_int
    f.argtypes = [U32P, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, U32P, U32P, U32P,
                  ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint32)]
    return f


def run_build(f, hist, symbol_max, log2max):
    n = len(hist)
    cw = np.zeros(n, np.uint32)
    ln = np.zeros(n, np.uint32)
    tw = np.zeros(1 << 17, np.uint32)
    tb = ctypes.c_uint32()
    r = f(np.ascontiguousarray(hist, np.uint32), n, symbol_max, log2max, cw, ln, tw, len(tw), ctypes.byref(tb))
    return r, cw, ln, tw[: (tb.value + 31) // 32].copy(), tb.value


def random_histograms(count, seed, max_bins=3000):
    """Histograms of the shapes the codec meets: sparse, geometric, peaked,
    many ties, constant."""
    rng = np.random.default_rng(seed)
    out = []
    for t in range(count):
        kind = t % 6
        n = int(rng.integers(1, max_bins))
        if kind == 0:
            h = rng.integers(0, 5, n)
        elif kind == 1:
            h = rng.geometric(0.3, n) * (rng.random(n) < 0.7)
        elif kind == 2:
            h = np.maximum(0, 1000 * np.exp(-np.arange(n) / max(1, n / 20)) + rng.normal(0, 2, n)).astype(np.int64)
        elif kind == 3:
            h = rng.integers(0, 3, n) * rng.integers(0, 2, n)
        elif kind == 4:
            h = np.full(n, int(rng.integers(0, 4)))
        else:
            # Fibonacci-like counts give long codes
            k = min(n, 25)
            fib = [1, 1]
            while len(fib) < k:
                fib.append(fib[-1] + fib[-2])
            h = np.zeros(n, np.int64)
            h[rng.choice(n, k, replace=False)] = fib[:k]
        h = np.asarray(h, dtype=np.uint32)
        nz = np.nonzero(h)[0]
        smax = int(nz[-1]) if len(nz) else 0
        out.append((h[: smax + 1].copy(), smax))
    return out


# ---------------------------------------------------------------- oracle API
class Oracle:
    """ctypes front end of oracle/liboracle.so (the CPU checker)."""

    def __init__(self):
        self.lib = load_oracle()
        L = self.lib
        c = ctypes
        L.orc_dwt_float_fwd.argtypes = [F32P, F32P, c.c_long, c.c_long, c.c_long]
        L.orc_dwt_float_inv.argtypes = [F32P, F32P, c.c_long, c.c_long, c.c_long]
        L.orc_dwt_double_fwd.argtypes = [F64P, F64P, c.c_long, c.c_long, c.c_long]
        L.orc_dwt_double_inv.argtypes = [F64P, F64P, c.c_long, c.c_long, c.c_long]
        L.orc_dwt_int_fwd.argtypes = [I16P, I16P, c.c_long, c.c_long, c.c_long]
        L.orc_dwt_int_inv.argtypes = [I16P, I16P, c.c_long, c.c_long, c.c_long]
        L.orc_quantize_to_symbols16.argtypes = [U16P, F32P, c.c_long, c.c_long, c.c_long, c.c_float, c.c_long, c.c_long]
        L.orc_unquantize_from_symbols16.argtypes = [F32P, U16P, c.c_long, c.c_long, c.c_long, c.c_float, c.c_long, c.c_long]
        L.orc_rle_encode16.argtypes = [U16P, c.c_uint32, U16P, U16P]
        L.orc_rle_encode16.restype = c.c_uint32
        L.orc_encode.argtypes = [c.c_int, c.c_int, c.c_void_p, c.c_uint32, c.c_uint32, c.c_uint32, c.c_uint32, U32P,
                                 c.c_uint32, c.POINTER(c.c_uint32), c.POINTER(c.c_uint32)]
        L.orc_decode.argtypes = [c.c_int, c.c_int, U32P, c.c_uint32, c.POINTER(c.c_uint32), c.c_void_p, c.c_uint32,
                                 c.c_uint32, c.c_uint32, c.c_uint32]
        L.orc_compress_volume_float.argtypes = [F32P, c.c_long, c.c_long, c.c_long, c.c_int, c.c_float, c.c_uint32,
                                                c.c_uint32, U32P, c.c_uint32, c.POINTER(c.c_uint32)]
        L.orc_decompress_volume_float.argtypes = [U32P, c.c_uint32, F32P, c.c_long, c.c_long, c.c_long, c.c_int,
                                                  c.c_float, c.c_uint32, c.c_uint32]
        L.orc_compress_volume_float_ex.argtypes = [F32P, c.c_long, c.c_long, c.c_long, c.c_int, c.c_float,
                                                   c.c_uint32, c.c_uint32, c.c_int, U32P, c.c_uint32,
                                                   c.POINTER(c.c_uint32)]
        L.orc_decompress_volume_float_ex.argtypes = [U32P, c.c_uint32, F32P, c.c_long, c.c_long, c.c_long, c.c_int,
                                                     c.c_float, c.c_uint32, c.c_uint32, c.c_int]
        L.orc_compress_volume_quantfirst.argtypes = [F32P, c.c_long, c.c_long, c.c_long, c.c_int, c.c_float,
                                                     c.c_uint32, c.c_uint32, c.c_int, U32P, c.c_uint32,
                                                     c.POINTER(c.c_uint32)]
        L.orc_decompress_volume_quantfirst.argtypes = [U32P, c.c_uint32, F32P, c.c_long, c.c_long, c.c_long,
                                                       c.c_int, c.c_float, c.c_uint32, c.c_uint32, c.c_int]
        L.orc_volume_symbols.argtypes = [F32P, c.c_long, c.c_long, c.c_long, c.c_int, c.c_float, U16P]
        L.orc_volume_from_symbols.argtypes = [U16P, F32P, c.c_long, c.c_long, c.c_long, c.c_int, c.c_float]
        L.orc_compress_heightfield.argtypes = [I16P, c.c_long, c.c_long, c.c_int, c.c_uint32, c.c_uint32, U32P,
                                               c.c_uint32, c.POINTER(c.c_uint32)]
        L.orc_decompress_heightfield.argtypes = [U32P, c.c_uint32, I16P, c.c_long, c.c_long, c.c_int, c.c_uint32,
                                                 c.c_uint32]

    def dwt_float(self, a, inverse=False):
        a = np.ascontiguousarray(a, np.float32)
        out = np.empty_like(a)
        nz, ny, nx = a.shape if a.ndim == 3 else (1,) + a.shape
        (self.lib.orc_dwt_float_inv if inverse else self.lib.orc_dwt_float_fwd)(a, out, nx, ny, nz)
        return out

    def dwt_double(self, a, inverse=False):
        a = np.ascontiguousarray(a, np.float64)
        out = np.empty_like(a)
        nz, ny, nx = a.shape if a.ndim == 3 else (1,) + a.shape
        (self.lib.orc_dwt_double_inv if inverse else self.lib.orc_dwt_double_fwd)(a, out, nx, ny, nz)
        return out

    def dwt_int(self, a, inverse=False):
        a = np.ascontiguousarray(a, np.int16)
        out = np.empty_like(a)
        nz, ny, nx = a.shape if a.ndim == 3 else (1,) + a.shape
        (self.lib.orc_dwt_int_inv if inverse else self.lib.orc_dwt_int_fwd)(a, out, nx, ny, nz)
        return out

    def quantize(self, a, step):
        a = np.ascontiguousarray(a, np.float32)
        nz, ny, nx = a.shape if a.ndim == 3 else (1,) + a.shape
        out = np.empty(a.size, np.uint16)
        self.lib.orc_quantize_to_symbols16(out, a, nx, ny, nz, step, nx, nx * ny)
        return out.reshape(a.shape)

    def unquantize(self, s, step):
        s = np.ascontiguousarray(s, np.uint16)
        nz, ny, nx = s.shape if s.ndim == 3 else (1,) + s.shape
        out = np.empty(s.shape, np.float32)
        self.lib.orc_unquantize_from_symbols16(out, s, nx, ny, nz, step, nx, nx * ny)
        return out

    def encode(self, kind, streams, cb=128, log2max=14, start_words=None, start_bit_size=0, start_pos=0):
        streams = np.ascontiguousarray(streams)
        sym_bytes = streams.dtype.itemsize
        S, n = streams.shape
        cap = S * n * 3 + 4096 + (0 if start_words is None else len(start_words))
        words = np.zeros(cap, np.uint32)
        if start_words is not None:
            words[: len(start_words)] = start_words
        size = ctypes.c_uint32(start_bit_size)
        pos = ctypes.c_uint32(start_pos)
        r = self.lib.orc_encode(kind, sym_bytes, streams.ctypes.data, S, n, cb, log2max, words, cap,
                                ctypes.byref(size), ctypes.byref(pos))
        if r != 0:
            return None
        return words[: (size.value + 31) // 32].copy(), size.value, pos.value

    def decode(self, kind, words, bit_size, S, n, dtype=np.uint16, cb=128, log2max=14, pos=0):
        out = np.zeros((S, n), dtype)
        p = ctypes.c_uint32(pos)
        self.lib.orc_decode(kind, np.dtype(dtype).itemsize, np.ascontiguousarray(words, np.uint32), bit_size,
                            ctypes.byref(p), out.ctypes.data, S, n, cb, log2max)
        return out, p.value

    def compress_volume(self, vol, levels, q0, cb=128, log2max=14, rle_only_level0=False, quant_first=False):
        vol = np.ascontiguousarray(vol, np.float32)
        nz, ny, nx = vol.shape
        cap = vol.size * 2 + 65536
        words = np.zeros(cap, np.uint32)
        bits = ctypes.c_uint32()
        f = self.lib.orc_compress_volume_quantfirst if quant_first else self.lib.orc_compress_volume_float_ex
        r = f(vol, nx, ny, nz, levels, q0, cb, log2max, int(rle_only_level0), words, cap, ctypes.byref(bits))
        assert r == 0, r
        return words[: (bits.value + 31) // 32].copy(), bits.value

    def decompress_volume(self, words, bits, shape, levels, q0, cb=128, log2max=14, rle_only_level0=False,
                          quant_first=False):
        nz, ny, nx = shape
        out = np.zeros(shape, np.float32)
        f = self.lib.orc_decompress_volume_quantfirst if quant_first else self.lib.orc_decompress_volume_float_ex
        f(np.ascontiguousarray(words, np.uint32), bits, out, nx, ny, nz, levels, q0, cb, log2max, int(rle_only_level0))
        return out

    def compress_heightfield(self, img, levels, cb=128, log2max=14):
        img = np.ascontiguousarray(img, np.int16)
        ny, nx = img.shape
        cap = img.size * 2 + 65536
        words = np.zeros(cap, np.uint32)
        bits = ctypes.c_uint32()
        r = self.lib.orc_compress_heightfield(img, nx, ny, levels, cb, log2max, words, cap, ctypes.byref(bits))
        assert r == 0, r
        return words[: (bits.value + 31) // 32].copy(), bits.value

    def decompress_heightfield(self, words, bits, shape, levels, cb=128, log2max=14):
        ny, nx = shape
        out = np.zeros(shape, np.int16)
        self.lib.orc_decompress_heightfield(np.ascontiguousarray(words, np.uint32), bits, out, nx, ny, levels, cb,
                                            log2max)
        return out


def symbol_streams(kind, S, n, seed, dtype=np.uint16, max_symbol=200):
    """Seeded symbol streams of the shapes the codec meets."""
    rng = np.random.default_rng(seed)
    if kind == "sparse":        # quantized highpass: mostly zeros, long runs
        a = (rng.geometric(0.5, (S, n)) - 1) * (rng.random((S, n)) < 0.15)
    elif kind == "dense":
        a = rng.integers(0, max_symbol, (S, n))
    elif kind == "laplace":
        v = np.rint(rng.laplace(0, 6, (S, n))).astype(np.int64)
        a = 2 * np.abs(v) - (v < 0)
    elif kind == "runs":        # runs longer than 255 and 256-multiples
        a = np.zeros((S, n), np.int64)
        for s in range(S):
            pos = 0
            while pos < n:
                pos += int(rng.choice([0, 1, 255, 256, 257, 511, 512, 1000]))
                if pos < n:
                    a[s, pos] = int(rng.integers(1, 40))
                pos += 1
    elif kind == "zeros":
        a = np.zeros((S, n), np.int64)
    elif kind == "single":
        a = np.full((S, n), 7, np.int64)
    else:
        raise ValueError(kind)
    return np.ascontiguousarray(a.astype(dtype))
