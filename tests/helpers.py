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
        L.orc_max_abs.argtypes = [F32P, c.c_long]
        L.orc_max_abs.restype = c.c_float
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

    def max_abs(self, a):
        a = np.ascontiguousarray(a, np.float32).ravel()
        return np.float32(self.lib.orc_max_abs(a, a.size))

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


class ImageOracle:
    """The oracle's 2D image side (oracle/oracle.cpp): byte DWTs, lowpass-only
    transforms, byte-image quantizers, YCoCg, Bits and the one-level image and
    heightfield codecs, on numpy arrays."""

    def __init__(self):
        self.lib = L = load_oracle()
        c = ctypes
        vp, lg, u32, f32, i32 = c.c_void_p, c.c_long, c.c_uint32, c.c_float, c.c_int
        L.orc_dwt_float_fwd_from_byte.argtypes = [vp, lg, vp, lg, lg, lg]
        L.orc_dwt_float_inv_to_byte.argtypes = [vp, vp, lg, lg, lg, lg]
        L.orc_dwt_float_inv_from_symbols_to_byte.argtypes = [vp, vp, f32, vp, lg, lg, lg, lg]
        L.orc_dwt_float2d_lowpass_from_byte.argtypes = [vp, lg, vp, lg, lg]
        L.orc_dwt_int_lowpass.argtypes = [vp, vp, lg, lg]
        L.orc_float_to_byte_2d.argtypes = [vp, lg, lg, vp, lg, lg, lg]
        L.orc_byte_to_float_2d.argtypes = [vp, vp, lg, lg, lg, lg, lg]
        L.orc_quantize_difference_2d.argtypes = [vp, vp, f32, vp, lg, lg, lg, lg, lg, i32, i32]
        L.orc_unquantize_difference_2d.argtypes = [vp, vp, f32, vp, lg, lg, lg, lg, lg, i32]
        L.orc_ycocg.argtypes = [vp, vp, lg, i32, i32]
        L.orc_lsb.argtypes = [i32, vp, vp, u32, c.c_int16]
        L.orc_shift_elems.argtypes = [vp, u32, c.c_int16]
        L.orc_get_lowpass_image.argtypes = [vp, lg, lg, lg, lg, vp]
        L.orc_get_lowpass_heightfield.argtypes = [vp, lg, lg, vp, c.c_int16]
        L.orc_compress_image_one_level.argtypes = [vp, lg, lg, lg, lg, vp, f32, u32, u32, vp, u32, c.POINTER(u32)]
        L.orc_decompress_image_one_level.argtypes = [vp, u32, vp, lg, lg, lg, lg, vp, f32, u32, u32]
        L.orc_compress_heightfield_one_level.argtypes = [vp, lg, lg, vp, c.c_int16, u32, u32, vp, u32, c.POINTER(u32)]
        L.orc_decompress_heightfield_one_level.argtypes = [vp, u32, vp, lg, lg, vp, c.c_int16, u32, u32]
        for n in ["orc_compress_image_one_level", "orc_decompress_image_one_level",
                  "orc_compress_heightfield_one_level", "orc_decompress_heightfield_one_level"]:
            getattr(L, n).restype = c.c_int

    @staticmethod
    def _p(a, offset=0):
        return ctypes.c_void_p(a.ctypes.data + offset)

    def dwt_fwd_from_byte(self, img, channel):
        """img (..., channels) uint8, dims (z, y, x) or (y, x)."""
        img = np.ascontiguousarray(img)
        ch = img.shape[-1]
        dims = img.shape[:-1]
        nz, ny, nx = (1,) + dims if len(dims) == 2 else dims
        out = np.zeros(dims, np.float32)
        self.lib.orc_dwt_float_fwd_from_byte(self._p(img, channel), ch, self._p(out), nx, ny, nz)
        return out

    def dwt_inv_to_byte(self, coef, target, channel):
        """Writes channel `channel` of target (..., channels) in place."""
        coef = np.ascontiguousarray(coef, np.float32)
        ch = target.shape[-1]
        dims = coef.shape
        nz, ny, nx = (1,) + dims if len(dims) == 2 else dims
        self.lib.orc_dwt_float_inv_to_byte(self._p(coef), self._p(target, channel), ch, nx, ny, nz)

    def dwt_inv_from_symbols_to_byte(self, lowpass, bands, step, target, channel):
        """lowpass: dense (z/2, y/2, x/2) or (y/2, x/2) float; bands: u16 array of 3 or 7 bands."""
        lowpass = np.ascontiguousarray(lowpass, np.float32)
        bands = [np.ascontiguousarray(b, np.uint16) for b in bands]
        ptrs = (ctypes.c_void_p * len(bands))(*[b.ctypes.data for b in bands])
        ch = target.shape[-1]
        dims = target.shape[:-1]
        nz, ny, nx = (1,) + dims if len(dims) == 2 else dims
        self.lib.orc_dwt_float_inv_from_symbols_to_byte(self._p(lowpass), ctypes.cast(ptrs, ctypes.c_void_p), step,
                                                        self._p(target, channel), ch, nx, ny, nz)

    def lowpass_from_byte(self, img, channel):
        img = np.ascontiguousarray(img)
        ny, nx, ch = img.shape
        out = np.zeros((ny // 2, nx // 2), np.float32)
        self.lib.orc_dwt_float2d_lowpass_from_byte(self._p(img, channel), ch, self._p(out), nx, ny)
        return out

    def int_lowpass(self, img):
        img = np.ascontiguousarray(img, np.int16)
        ny, nx = img.shape
        out = np.zeros((ny // 2, nx // 2), np.int16)
        self.lib.orc_dwt_int_lowpass(self._p(img), self._p(out), nx, ny)
        return out

    def float_to_byte_2d(self, out, channel, data, nx, ny, pitch):
        self.lib.orc_float_to_byte_2d(self._p(out), out.shape[-1], channel, self._p(data), nx, ny, pitch)

    def byte_to_float_2d(self, out, img, channel, nx, ny, pitch):
        self.lib.orc_byte_to_float_2d(self._p(out), self._p(img), img.shape[-1], channel, nx, ny, pitch)

    def quantize_difference(self, data, step, ref, channel, nx, ny, pitch, quant_type=0, roundtrip=False):
        """Returns the symbols; data (float32, row pitch `pitch`) is updated by the round trip."""
        sym = np.zeros((ny, nx), np.uint16)
        self.lib.orc_quantize_difference_2d(self._p(sym), self._p(data), step, self._p(ref), ref.shape[-1], channel,
                                            nx, ny, pitch, quant_type, int(roundtrip))
        return sym

    def unquantize_difference(self, out, sym, step, ref, channel, nx, ny, pitch, quant_type=0):
        sym = np.ascontiguousarray(sym, np.uint16)
        self.lib.orc_unquantize_difference_2d(self._p(out), self._p(sym), step, self._p(ref), ref.shape[-1], channel,
                                              nx, ny, pitch, quant_type)

    def ycocg(self, px, to_ycocg=True):
        px = np.ascontiguousarray(px, np.uint8)
        out = np.zeros_like(px)
        self.lib.orc_ycocg(self._p(out), self._p(px), px.shape[0], px.shape[1], int(to_ycocg))
        return out

    def lsb(self, mode, data, bits=None, shift=0):
        """mode 0 get, 1 remove, 2 append; returns (data, bits) copies."""
        data = np.array(data, np.int16)
        n = data.size
        if bits is None and mode == 0:
            bits = np.zeros((n + 31) // 32, np.uint32)
        bits = None if bits is None else np.array(bits, np.uint32)
        self.lib.orc_lsb(mode, self._p(data), None if bits is None else self._p(bits), n, shift)
        return data, bits

    def shift_elems(self, data, shift):
        data = np.array(data, np.int16)
        self.lib.orc_shift_elems(self._p(data), data.size, shift)
        return data

    def lowpass_image(self, img, channels_to_process):
        img = np.ascontiguousarray(img)
        ny, nx, ch = img.shape
        out = np.zeros((ny // 2, nx // 2, ch), np.uint8)
        self.lib.orc_get_lowpass_image(self._p(img), nx, ny, ch, channels_to_process, self._p(out))
        return out

    def lowpass_heightfield(self, img, shift):
        img = np.ascontiguousarray(img, np.int16)
        ny, nx = img.shape
        out = np.zeros((ny // 2, nx // 2), np.int16)
        self.lib.orc_get_lowpass_heightfield(self._p(img), nx, ny, self._p(out), shift)
        return out

    def compress_image(self, img, channels_to_process, lowpass_ref, step, cb=128, log2max=14):
        """Returns (words, bit size, reconstruction)."""
        rec = np.array(img, np.uint8)
        ny, nx, ch = rec.shape
        lowpass_ref = np.ascontiguousarray(lowpass_ref, np.uint8)
        cap = rec.size * 4 + 65536
        words = np.zeros(cap, np.uint32)
        bits = ctypes.c_uint32()
        r = self.lib.orc_compress_image_one_level(self._p(rec), nx, ny, ch, channels_to_process, self._p(lowpass_ref),
                                                  step, cb, log2max, self._p(words), cap, ctypes.byref(bits))
        assert r == 0, r
        return words[: (bits.value + 31) // 32].copy(), bits.value, rec

    def decompress_image(self, words, bit_size, out, channels_to_process, lowpass_ref, step, cb=128, log2max=14):
        ny, nx, ch = out.shape
        words = np.ascontiguousarray(words, np.uint32)
        lowpass_ref = np.ascontiguousarray(lowpass_ref, np.uint8)
        r = self.lib.orc_decompress_image_one_level(self._p(words), bit_size, self._p(out), nx, ny, ch,
                                                    channels_to_process, self._p(lowpass_ref), step, cb, log2max)
        assert r == 0, r

    def compress_heightfield_one_level(self, img, shift, cb=128, log2max=14):
        """Returns (words, bit size, lowpass)."""
        img = np.ascontiguousarray(img, np.int16)
        ny, nx = img.shape
        lp = np.zeros((ny // 2, nx // 2), np.int16)
        cap = img.size + 65536
        words = np.zeros(cap, np.uint32)
        bits = ctypes.c_uint32()
        r = self.lib.orc_compress_heightfield_one_level(self._p(img), nx, ny, self._p(lp), shift, cb, log2max,
                                                        self._p(words), cap, ctypes.byref(bits))
        assert r == 0, r
        return words[: (bits.value + 31) // 32].copy(), bits.value, lp

    def decompress_heightfield_one_level(self, words, bit_size, shape, lowpass, shift, cb=128, log2max=14):
        """Returns (image, restored lowpass)."""
        ny, nx = shape
        out = np.zeros(shape, np.int16)
        lp = np.array(lowpass, np.int16)
        words = np.ascontiguousarray(words, np.uint32)
        r = self.lib.orc_decompress_heightfield_one_level(self._p(words), bit_size, self._p(out), nx, ny, self._p(lp),
                                                          shift, cb, log2max)
        assert r == 0, r
        return out, lp


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
