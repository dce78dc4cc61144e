"""Python mirror of cudaCompress's API (Instance.h, Encode.h, util/DWT.h,
util/Quantize.h) over the C ABI, with torch CUDA tensors as device buffers.

Names and argument meaning follow the reference; like the reference, the
coding calls return bool (False on failure, with the reason in
``last_error()``); the util calls raise ``CudaCompressError`` on failure.
"""
from __future__ import annotations

import ctypes
from typing import List, Optional, Sequence

import numpy as np
import torch

from ._ffi import CudaCompressError, check, lib

RLHUFF = 0
HUFF = 1
QUANTIZE_DEADZONE = 0
QUANTIZE_UNIFORM = 1


def last_error() -> str:
    return lib().cc_last_error().decode(errors="replace")


def _ptr(t: Optional[torch.Tensor]) -> Optional[int]:
    return None if t is None else t.data_ptr()


def _stream(stream) -> Optional[int]:
    if stream is None:
        return None
    if isinstance(stream, torch.cuda.Stream):
        return stream.cuda_stream
    return int(stream)


def _sym_bytes(t: torch.Tensor) -> int:
    if t.dtype in (torch.int16, torch.uint16):
        return 2
    if t.dtype in (torch.int32, torch.uint32):
        return 4
    raise TypeError(f"symbol tensors must be 16- or 32-bit integers, got {t.dtype}")


class Instance:
    """createInstance / destroyInstance and the getters (Instance.h:26-45)."""

    def __init__(self, cuda_device: int, stream_count_max: int, elem_count_per_stream_max: int,
                 coding_block_size: int = 0, log2_huffman_distinct_symbol_count_max: int = 0):
        h = ctypes.c_void_p()
        check(lib().cc_create_instance(ctypes.byref(h), cuda_device, stream_count_max, elem_count_per_stream_max,
                                       coding_block_size, log2_huffman_distinct_symbol_count_max), "createInstance")
        self.handle = h

    def close(self):
        if self.handle:
            lib().cc_destroy_instance(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def cuda_device(self) -> int:
        return lib().cc_get_instance_cuda_device(self.handle)

    @property
    def stream_count_max(self) -> int:
        return lib().cc_get_instance_stream_count_max(self.handle)

    @property
    def elem_count_per_stream_max(self) -> int:
        return lib().cc_get_instance_elem_count_per_stream_max(self.handle)

    @property
    def coding_block_size(self) -> int:
        return lib().cc_get_instance_coding_block_size(self.handle)

    @property
    def log2_huffman_distinct_symbol_count_max(self) -> int:
        return lib().cc_get_instance_log2_huffman_distinct_symbol_count_max(self.handle)

    @property
    def use_long_symbols(self) -> bool:
        return bool(lib().cc_get_instance_use_long_symbols(self.handle))

    def set_stream(self, stream) -> None:
        """setInstanceCudaStream (and its setInstanceStream spelling)."""
        lib().cc_set_instance_stream(self.handle, _stream(stream))

    def get_stream(self) -> Optional[int]:
        return lib().cc_get_instance_stream(self.handle)

    @property
    def required_memory(self) -> int:
        return lib().cc_encode_get_required_memory(self.handle)


class BitStream:
    """Host bit stream (BitStream.h semantics): 32-bit words, bit size, position."""

    def __init__(self, words: Optional[np.ndarray] = None, bit_size: Optional[int] = None):
        self.words = np.zeros(0, np.uint32) if words is None else np.ascontiguousarray(words, np.uint32).copy()
        self.bit_size = len(self.words) * 32 if bit_size is None else int(bit_size)
        self.pos = 0

    def raw(self) -> np.ndarray:
        return self.words[: (self.bit_size + 31) // 32]

    def set_bit_position(self, pos: int) -> bool:
        ok = pos <= self.bit_size
        self.pos = min(pos, self.bit_size)
        return ok


def _encode(inst: Instance, kind: int, bs: BitStream, streams: Sequence[torch.Tensor], count: int) -> bool:
    n = len(streams)
    if n == 0:
        return True
    sb = _sym_bytes(streams[0])
    arr = (ctypes.c_void_p * n)(*[s.data_ptr() for s in streams])
    cap = (bs.bit_size + 31) // 32 + (count * n) // 2 + 1024
    while True:
        if len(bs.words) < cap:
            grown = np.zeros(cap, np.uint32)
            grown[: len(bs.words)] = bs.words
            bs.words = grown
        size = ctypes.c_uint32(bs.bit_size)
        pos = ctypes.c_uint32(bs.pos)
        wp = bs.words.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))
        rc = lib().cc_encode_to_buffer(inst.handle, kind, sb, arr, n, count, wp, len(bs.words), ctypes.byref(size),
                                       ctypes.byref(pos))
        if rc == -7 and size.value // 32 + 1 > len(bs.words):     # CC_ERR_CAPACITY: grow and retry
            cap = size.value // 32 + 2
            continue
        if rc != 0:
            return False
        bs.bit_size = size.value
        bs.pos = pos.value
        return True


def _decode(inst: Instance, kind: int, bs: BitStream, outs: Sequence[torch.Tensor], count: int) -> bool:
    n = len(outs)
    if n == 0:
        return True
    sb = _sym_bytes(outs[0])
    words = bs.raw()
    wp = (ctypes.POINTER(ctypes.c_uint32) * 1)(words.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)))
    sizes = (ctypes.c_uint32 * 1)(bs.bit_size)
    pos = (ctypes.c_uint32 * 1)(bs.pos)
    arr = (ctypes.c_void_p * n)(*[o.data_ptr() for o in outs])
    rc = lib().cc_decode(inst.handle, kind, sb, wp, sizes, pos, 1, None, arr, n, count)
    if rc != 0:
        return False
    bs.pos = pos[0]
    return True


def encode_rlhuff(inst: Instance, bs: BitStream, streams: Sequence[torch.Tensor], symbol_count_per_block: int) -> bool:
    """encodeRLHuff (Encode.h:28)."""
    return _encode(inst, RLHUFF, bs, streams, symbol_count_per_block)


def encode_huff(inst: Instance, bs: BitStream, streams: Sequence[torch.Tensor], symbol_count_per_block: int) -> bool:
    """encodeHuff (Encode.h:31)."""
    return _encode(inst, HUFF, bs, streams, symbol_count_per_block)


def decode_rlhuff(inst: Instance, bs: BitStream, outs: Sequence[torch.Tensor], symbol_count_per_block: int) -> bool:
    """decodeRLHuff (Encode.h:29); every output symbol is written (no zeroing needed)."""
    return _decode(inst, RLHUFF, bs, outs, symbol_count_per_block)


def decode_huff(inst: Instance, bs: BitStream, outs: Sequence[torch.Tensor], symbol_count_per_block: int) -> bool:
    """decodeHuff (Encode.h:32)."""
    return _decode(inst, HUFF, bs, outs, symbol_count_per_block)


def decode_status(inst: Instance) -> int:
    """Synchronizes and returns the device-side status of the last decode."""
    return lib().cc_decode_status(inst.handle)


# ---------------------------------------------------------------- util::DWT
def dwt_float_forward(dst, buf2, buf1, src, size_x, size_y, size_z=1, src_channel_count=1, dst_row_pitch=0,
                      dst_slice_pitch=0, src_row_pitch=0, src_slice_pitch=0, stream=None):
    """dwtFloat2DForward (size_z == 1, buf2 unused) / dwtFloat3DForward."""
    check(lib().cc_dwt_float_forward(_ptr(dst), _ptr(buf2), _ptr(buf1), _ptr(src), size_x, size_y, size_z,
                                      src_channel_count, dst_row_pitch, dst_slice_pitch, src_row_pitch,
                                      src_slice_pitch, _stream(stream)), "dwtFloatForward")


def dwt_float_inverse(dst, buf2, buf1, src, size_x, size_y, size_z=1, dst_channel_count=1, dst_row_pitch=0,
                      dst_slice_pitch=0, src_row_pitch=0, src_slice_pitch=0, stream=None):
    check(lib().cc_dwt_float_inverse(_ptr(dst), _ptr(buf2), _ptr(buf1), _ptr(src), size_x, size_y, size_z,
                                      dst_channel_count, dst_row_pitch, dst_slice_pitch, src_row_pitch,
                                      src_slice_pitch, _stream(stream)), "dwtFloatInverse")


def dwt_float_inverse_from_symbols(dst, buf2, buf1, lowpass, highpass_ptrs: torch.Tensor, symbol_bytes, quant_step,
                                   size_x, size_y, size_z=1, dst_channel_count=1, dst_row_pitch=0,
                                   dst_slice_pitch=0, lowpass_row_pitch=0, lowpass_slice_pitch=0, stream=None):
    """highpass_ptrs: int64 CUDA tensor of 3 (2D) or 7 (3D) band device pointers."""
    check(lib().cc_dwt_float_inverse_from_symbols(_ptr(dst), _ptr(buf2), _ptr(buf1), _ptr(lowpass),
                                                   _ptr(highpass_ptrs), symbol_bytes, quant_step, size_x, size_y,
                                                   size_z, dst_channel_count, dst_row_pitch, dst_slice_pitch,
                                                   lowpass_row_pitch, lowpass_slice_pitch, _stream(stream)),
          "dwtFloatInverseFromSymbols")


def dwt_float_forward_from_byte(dst, buf2, buf1, src, size_x, size_y, size_z=1, src_channel_count=1,
                                dst_row_pitch=0, dst_slice_pitch=0, src_row_pitch=0, src_slice_pitch=0, stream=None):
    """dwtFloat{2D,3D}ForwardFromByte: src is a uint8 tensor (or a view starting
    at the wanted channel) with src_channel_count interleaved channels."""
    check(lib().cc_dwt_float_forward_from_byte(_ptr(dst), _ptr(buf2), _ptr(buf1), _ptr(src), size_x, size_y, size_z,
                                                src_channel_count, dst_row_pitch, dst_slice_pitch, src_row_pitch,
                                                src_slice_pitch, _stream(stream)), "dwtFloatForwardFromByte")


def dwt_float_inverse_to_byte(dst, buf2, buf1, src, size_x, size_y, size_z=1, dst_channel_count=1, dst_row_pitch=0,
                              dst_slice_pitch=0, src_row_pitch=0, src_slice_pitch=0, stream=None):
    check(lib().cc_dwt_float_inverse_to_byte(_ptr(dst), _ptr(buf2), _ptr(buf1), _ptr(src), size_x, size_y, size_z,
                                              dst_channel_count, dst_row_pitch, dst_slice_pitch, src_row_pitch,
                                              src_slice_pitch, _stream(stream)), "dwtFloatInverseToByte")


def dwt_float_inverse_from_symbols_to_byte(dst, buf2, buf1, lowpass, highpass_ptrs: torch.Tensor, symbol_bytes,
                                           quant_step, size_x, size_y, size_z=1, dst_channel_count=1,
                                           dst_row_pitch=0, dst_slice_pitch=0, lowpass_row_pitch=0,
                                           lowpass_slice_pitch=0, stream=None):
    check(lib().cc_dwt_float_inverse_from_symbols_to_byte(_ptr(dst), _ptr(buf2), _ptr(buf1), _ptr(lowpass),
                                                           _ptr(highpass_ptrs), symbol_bytes, quant_step, size_x,
                                                           size_y, size_z, dst_channel_count, dst_row_pitch,
                                                           dst_slice_pitch, lowpass_row_pitch, lowpass_slice_pitch,
                                                           _stream(stream)), "dwtFloatInverseFromSymbolsToByte")


def dwt_float2d_forward_lowpass_only_from_byte(dst, buf, src, size_x, size_y, src_channel_count=1, dst_row_pitch=0,
                                               src_row_pitch=0, stream=None):
    """dwtFloat2DForwardLowpassOnlyFromByte: the LL band only (buf unused)."""
    check(lib().cc_dwt_float2d_forward_lowpass_only_from_byte(_ptr(dst), _ptr(buf), _ptr(src), size_x, size_y,
                                                               src_channel_count, dst_row_pitch, src_row_pitch,
                                                               _stream(stream)),
          "dwtFloat2DForwardLowpassOnlyFromByte")


def dwt_int_forward_lowpass_only(dst, buf, src, size_x, size_y, dst_row_pitch=0, src_row_pitch=0, stream=None):
    """dwtIntForwardLowpassOnly: the LL band only (buf unused)."""
    check(lib().cc_dwt_int_forward_lowpass_only(_ptr(dst), _ptr(buf), _ptr(src), size_x, size_y, dst_row_pitch,
                                                src_row_pitch, _stream(stream)), "dwtIntForwardLowpassOnly")


def dwt_int_forward(dst, buf, src, size_x, size_y, size_z=1, dst_row_pitch=0, dst_slice_pitch=0, src_row_pitch=0,
                    src_slice_pitch=0, stream=None):
    check(lib().cc_dwt_int_forward(_ptr(dst), _ptr(buf), _ptr(src), size_x, size_y, size_z, dst_row_pitch,
                                   dst_slice_pitch, src_row_pitch, src_slice_pitch, _stream(stream)), "dwtIntForward")


def dwt_int_inverse(dst, buf, src, size_x, size_y, size_z=1, dst_row_pitch=0, dst_slice_pitch=0, src_row_pitch=0,
                    src_slice_pitch=0, stream=None):
    check(lib().cc_dwt_int_inverse(_ptr(dst), _ptr(buf), _ptr(src), size_x, size_y, size_z, dst_row_pitch,
                                   dst_slice_pitch, src_row_pitch, src_slice_pitch, _stream(stream)), "dwtIntInverse")


# ----------------------------------------------------------- util::Quantize
def quantize_to_symbols(symbols, data, size_x, size_y, size_z, quant_step, row_pitch_src=0, slice_pitch_src=0,
                        quant_type=QUANTIZE_DEADZONE, stream=None):
    check(lib().cc_quantize_to_symbols(_ptr(symbols), _sym_bytes(symbols), _ptr(data), size_x, size_y, size_z,
                                       quant_step, row_pitch_src, slice_pitch_src, quant_type, _stream(stream)),
          "quantizeToSymbols")


def quantize_to_symbols_roundtrip(symbols, data, size_x, size_y, size_z, quant_step, row_pitch_src=0,
                                  slice_pitch_src=0, quant_type=QUANTIZE_DEADZONE, stream=None):
    check(lib().cc_quantize_to_symbols_roundtrip(_ptr(symbols), _sym_bytes(symbols), _ptr(data), size_x, size_y,
                                                 size_z, quant_step, row_pitch_src, slice_pitch_src, quant_type,
                                                 _stream(stream)), "quantizeToSymbolsRoundtrip")


def unquantize_from_symbols(data, symbols, size_x, size_y, size_z, quant_step, row_pitch_dst=0, slice_pitch_dst=0,
                            quant_type=QUANTIZE_DEADZONE, stream=None):
    check(lib().cc_unquantize_from_symbols(_ptr(data), _ptr(symbols), _sym_bytes(symbols), size_x, size_y, size_z,
                                           quant_step, row_pitch_dst, slice_pitch_dst, quant_type, _stream(stream)),
          "unquantizeFromSymbols")


def symbolize(symbols, data, size_x, size_y, size_z, row_pitch_src=0, slice_pitch_src=0, stream=None):
    check(lib().cc_symbolize(_ptr(symbols), _ptr(data), size_x, size_y, size_z, row_pitch_src, slice_pitch_src,
                             _stream(stream)), "symbolize")


def unsymbolize(data, symbols, size_x, size_y, size_z, row_pitch_dst=0, slice_pitch_dst=0, stream=None):
    check(lib().cc_unsymbolize(_ptr(data), _ptr(symbols), size_x, size_y, size_z, row_pitch_dst, slice_pitch_dst,
                               _stream(stream)), "unsymbolize")


def quantize_to_short(quant, data, size_x, size_y, size_z, quant_step, row_pitch_src=0, slice_pitch_src=0,
                      quant_type=QUANTIZE_DEADZONE, stream=None):
    check(lib().cc_quantize_to_short(_ptr(quant), _ptr(data), size_x, size_y, size_z, quant_step, row_pitch_src,
                                     slice_pitch_src, quant_type, _stream(stream)), "quantizeToShort")


def unquantize_from_short(data, quant, size_x, size_y, size_z, quant_step, row_pitch_dst=0, slice_pitch_dst=0,
                          quant_type=QUANTIZE_DEADZONE, stream=None):
    check(lib().cc_unquantize_from_short(_ptr(data), _ptr(quant), size_x, size_y, size_z, quant_step, row_pitch_dst,
                                         slice_pitch_dst, quant_type, _stream(stream)), "unquantizeFromShort")


def get_max_abs(inst: Instance, data, elem_count, out):
    check(lib().cc_get_max_abs(inst.handle, _ptr(data), elem_count, _ptr(out)), "getMaxAbs")


# ------------------------------------------------------------- pipelines
def volume_stream_capacity_words(nx, ny, nz, log2max=14) -> int:
    """Upper bound of the volume codec's stream size in 32-bit words."""
    n = nx * ny * nz
    return int(n * (log2max + 8) // 32 + 64 * 1024)


RLE_ONLY_LEVEL0 = 1   # CC_VOLUME_RLE_ONLY_LEVEL0 (doRLEOnlyOnLvl0)


def compress_volume_float(inst: Instance, volume: torch.Tensor, levels: int, q0: float,
                          out_words: Optional[torch.Tensor] = None, rle_only_level0: bool = False):
    """Lossy volume codec (CompressVolume.cpp:312-409).  volume: (z, y, x)
    float32 CUDA tensor.  rle_only_level0: doRLEOnlyOnLvl0 (levels above 0
    with encodeHuff).  Returns (words tensor on the device, bit size)."""
    nz, ny, nx = volume.shape
    if out_words is None:
        out_words = torch.empty(volume_stream_capacity_words(nx, ny, nz), dtype=torch.int32, device=volume.device)
    bits = ctypes.c_uint32()
    check(lib().cc_compress_volume_float_ex(inst.handle, volume.data_ptr(), nx, ny, nz, levels, q0,
                                            RLE_ONLY_LEVEL0 if rle_only_level0 else 0, out_words.data_ptr(),
                                            out_words.numel(), ctypes.byref(bits)), "compressVolumeFloat")
    return out_words, bits.value


def decompress_volume_float(inst: Instance, out: torch.Tensor, levels: int, q0: float, words: torch.Tensor,
                            bit_size: int, rle_only_level0: bool = False) -> None:
    nz, ny, nx = out.shape
    check(lib().cc_decompress_volume_float_ex(inst.handle, out.data_ptr(), nx, ny, nz, levels, q0,
                                              RLE_ONLY_LEVEL0 if rle_only_level0 else 0, words.data_ptr(), bit_size),
          "decompressVolumeFloat")


def compress_volume_float_quant_first(inst: Instance, volume: torch.Tensor, levels: int, step: float,
                                      out_words: Optional[torch.Tensor] = None, rle_only_level0: bool = False):
    """Quantize-first lossy codec (CompressVolume.cpp:651-757): uniform
    quantization to short, integer DWT, symbols; error <= step / 2."""
    nz, ny, nx = volume.shape
    if out_words is None:
        out_words = torch.empty(volume_stream_capacity_words(nx, ny, nz, 16), dtype=torch.int32,
                                device=volume.device)
    bits = ctypes.c_uint32()
    check(lib().cc_compress_volume_float_quant_first(inst.handle, volume.data_ptr(), nx, ny, nz, levels, step,
                                                     RLE_ONLY_LEVEL0 if rle_only_level0 else 0,
                                                     out_words.data_ptr(), out_words.numel(), ctypes.byref(bits)),
          "compressVolumeFloatQuantFirst")
    return out_words, bits.value


def decompress_volume_float_quant_first(inst: Instance, out: torch.Tensor, levels: int, step: float,
                                        words: torch.Tensor, bit_size: int, rle_only_level0: bool = False) -> None:
    nz, ny, nx = out.shape
    check(lib().cc_decompress_volume_float_quant_first(inst.handle, out.data_ptr(), nx, ny, nz, levels, step,
                                                       RLE_ONLY_LEVEL0 if rle_only_level0 else 0, words.data_ptr(),
                                                       bit_size), "decompressVolumeFloatQuantFirst")


class _Channel(ctypes.Structure):
    _fields_ = [("d_volume", ctypes.c_void_p), ("d_words", ctypes.c_void_p), ("bit_size", ctypes.c_uint32),
                ("quant_step", ctypes.c_float)]


def decompress_volume_float_multichannel(inst: Instance, outs, words, bit_sizes, steps, levels: int,
                                         rle_only_level0: bool = False, quant_first: bool = False) -> None:
    """decompressVolumeFloat(QuantFirst)MultiChannel (CompressVolume.cpp:518-648,
    863-988): outs, words (device tensors), bit sizes and steps per channel;
    all channels the same shape."""
    n = len(outs)
    if not (len(words) == len(bit_sizes) == len(steps) == n) or n == 0:
        raise ValueError("one stream, bit size and step per channel")
    shape = tuple(outs[0].shape)
    if any(tuple(o.shape) != shape for o in outs):
        raise ValueError("all channels must have the same shape")
    nz, ny, nx = shape
    ch = (_Channel * n)(*[_Channel(o.data_ptr(), w.data_ptr(), int(b), float(s))
                          for o, w, b, s in zip(outs, words, bit_sizes, steps)])
    flags = RLE_ONLY_LEVEL0 if rle_only_level0 else 0
    f = lib().cc_decompress_volume_float_quant_first_multichannel if quant_first \
        else lib().cc_decompress_volume_float_multichannel
    check(f(inst.handle, ctypes.cast(ch, ctypes.c_void_p), n, nx, ny, nz, levels, flags),
          "decompressVolumeFloatMultiChannel")


def compress_heightfield(inst: Instance, image: torch.Tensor, levels: int, out_words: Optional[torch.Tensor] = None):
    """Lossless 2D integer codec.  image: (y, x) int16 CUDA tensor."""
    ny, nx = image.shape
    if out_words is None:
        out_words = torch.empty(nx * ny + 64 * 1024, dtype=torch.int32, device=image.device)
    bits = ctypes.c_uint32()
    check(lib().cc_compress_heightfield(inst.handle, image.data_ptr(), nx, ny, levels, out_words.data_ptr(),
                                        out_words.numel(), ctypes.byref(bits)), "compressHeightfield")
    return out_words, bits.value


def decompress_heightfield(inst: Instance, out: torch.Tensor, levels: int, words: torch.Tensor, bit_size: int) -> None:
    ny, nx = out.shape
    check(lib().cc_decompress_heightfield(inst.handle, out.data_ptr(), nx, ny, levels, words.data_ptr(), bit_size),
          "decompressHeightfield")


# ------------------------------------------------------ batched volume codec
class VolumeBatch:
    """Batched lossy volume codec (cc_volume_batch_*): `sizes` is a list of
    (z, y, x) shapes, `quant_steps` one step per volume.  Each volume's
    stream equals compress_volume_float's."""

    def __init__(self, inst: Instance, sizes, levels: int, quant_steps, graph: bool = False, z_chunk: int = 0):
        self.inst = inst
        self.count = len(sizes)
        self.shapes = [tuple(int(v) for v in s) for s in sizes]
        flat = []
        for (nz, ny, nx) in self.shapes:
            flat += [nx, ny, nz]
        arr = (ctypes.c_uint32 * len(flat))(*flat)
        steps = (ctypes.c_float * self.count)(*[float(q) for q in quant_steps])
        h = ctypes.c_void_p()
        check(lib().cc_volume_batch_create_ex(inst.handle, self.count, arr, levels, steps, z_chunk, ctypes.byref(h)),
              "cc_volume_batch_create")
        self.z_chunk = z_chunk
        self.handle = h
        self.levels = levels
        if graph:
            check(lib().cc_volume_batch_use_graph(self.handle, 1), "cc_volume_batch_use_graph")

    def close(self):
        if getattr(self, "handle", None):
            lib().cc_volume_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_active(self, k: int) -> None:
        check(lib().cc_volume_batch_set_active(self.handle, k), "cc_volume_batch_set_active")
        self.active = k

    def set_stream(self, stream) -> None:
        check(lib().cc_volume_batch_set_stream(self.handle, _stream(stream)), "cc_volume_batch_set_stream")

    def compress(self, volumes) -> None:
        if len(volumes) < getattr(self, "active", self.count):
            raise ValueError("one volume per active slot is needed")
        arr = (ctypes.c_void_p * max(len(volumes), 1))(*[v.data_ptr() for v in volumes])
        check(lib().cc_volume_batch_compress(self.handle, arr), "cc_volume_batch_compress")

    def decompress(self, outs) -> None:
        if len(outs) < getattr(self, "active", self.count):
            raise ValueError("one output per active slot is needed")
        arr = (ctypes.c_void_p * max(len(outs), 1))(*[o.data_ptr() for o in outs])
        check(lib().cc_volume_batch_decompress(self.handle, arr), "cc_volume_batch_decompress")

    def status(self) -> None:
        check(lib().cc_volume_batch_status(self.handle), "cc_volume_batch_status")

    def read_stream(self, v: int):
        """(host words, bit size) of volume v's stream (synchronizes)."""
        bits = ctypes.c_uint64()
        check(lib().cc_volume_batch_read_stream(self.handle, v, None, 0, ctypes.byref(bits)), "read_stream")
        words = np.zeros((bits.value + 31) // 32, np.uint32)
        check(lib().cc_volume_batch_read_stream(self.handle, v, words.ctypes.data, len(words), ctypes.byref(bits)),
              "read_stream")
        return words, int(bits.value)

    def load_streams(self, words, bit_sizes) -> None:
        """Loads one stream per volume (host numpy uint32 arrays, or CUDA
        int32 tensors) for decompress()."""
        ptrs = []
        for w in words:
            ptrs.append(w.data_ptr() if isinstance(w, torch.Tensor) else np.ascontiguousarray(w, np.uint32).ctypes.data)
        arr = (ctypes.c_void_p * len(ptrs))(*ptrs)
        bits = (ctypes.c_uint64 * len(ptrs))(*[int(b) for b in bit_sizes])
        check(lib().cc_volume_batch_load_streams(self.handle, arr, bits), "cc_volume_batch_load_streams")

    def download_streams(self, host_words: torch.Tensor, host_extents: torch.Tensor) -> None:
        """Enqueues the copy of the active volumes' streams into page-locked
        host tensors (int32 words, int64 extents: offsets then bit sizes);
        complete once the batch's stream reaches it."""
        check(lib().cc_volume_batch_download_streams(self.handle, host_words.data_ptr(), host_words.numel(),
                                                     host_extents.data_ptr()), "cc_volume_batch_download_streams")

    def upload_streams(self, host_words: torch.Tensor, host_extents: torch.Tensor) -> None:
        """Enqueues the copy of streams laid out as download_streams writes
        them back into the batch, for decompress()."""
        check(lib().cc_volume_batch_upload_streams(self.handle, host_words.data_ptr(), host_extents.data_ptr()),
              "cc_volume_batch_upload_streams")

    def collect_timings(self) -> None:
        lib().cc_volume_batch_collect_timings(self.handle)
