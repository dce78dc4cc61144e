"""The 2D image side of the library over torch CUDA tensors: byte-image
quantizers (util::floatToByte2D, byteToFloat2D, quantizeDifference*2D),
YCoCg colour conversion (util/YCoCg.h), least-significant-bit planes
(util/Bits.h), and the one-level image and heightfield codecs of the
reference's examples (CompressImage.h, CompressHeightfield.h)."""
from __future__ import annotations

import ctypes
from typing import List, Optional, Sequence

import torch

from ._ffi import check, lib
from .codec import QUANTIZE_DEADZONE, Instance, _ptr, _stream


# --------------------------------------------------------------- byte images
def float_to_byte_2d(quant, channel_count, channel, data, size_x, size_y, row_pitch_src=0, stream=None):
    check(lib().cc_float_to_byte_2d(_ptr(quant), channel_count, channel, _ptr(data), size_x, size_y, row_pitch_src,
                                    _stream(stream)), "floatToByte2D")


def byte_to_float_2d(data, quant, channel_count, channel, size_x, size_y, row_pitch_dst=0, stream=None):
    check(lib().cc_byte_to_float_2d(_ptr(data), _ptr(quant), channel_count, channel, size_x, size_y, row_pitch_dst,
                                    _stream(stream)), "byteToFloat2D")


def quantize_difference_to_symbols_2d(symbols, data, quant_step, reference, channel_count, channel, size_x, size_y,
                                      row_pitch_src=0, quant_type=QUANTIZE_DEADZONE, stream=None):
    check(lib().cc_quantize_difference_to_symbols_2d(_ptr(symbols), _ptr(data), quant_step, _ptr(reference),
                                                     channel_count, channel, size_x, size_y, row_pitch_src,
                                                     quant_type, _stream(stream)), "quantizeDifferenceToSymbols2D")


def quantize_difference_to_symbols_roundtrip_2d(symbols, data, quant_step, reference, channel_count, channel, size_x,
                                                size_y, row_pitch_src=0, quant_type=QUANTIZE_DEADZONE, stream=None):
    check(lib().cc_quantize_difference_to_symbols_roundtrip_2d(_ptr(symbols), _ptr(data), quant_step, _ptr(reference),
                                                               channel_count, channel, size_x, size_y, row_pitch_src,
                                                               quant_type, _stream(stream)),
          "quantizeDifferenceToSymbolsRoundtrip2D")


def unquantize_difference_from_symbols_2d(data, symbols, quant_step, reference, channel_count, channel, size_x, size_y,
                                          row_pitch_dst=0, quant_type=QUANTIZE_DEADZONE, stream=None):
    check(lib().cc_unquantize_difference_from_symbols_2d(_ptr(data), _ptr(symbols), quant_step, _ptr(reference),
                                                         channel_count, channel, size_x, size_y, row_pitch_dst,
                                                         quant_type, _stream(stream)),
          "unquantizeDifferenceFromSymbols2D")


# -------------------------------------------------------------------- YCoCg
def convert_rgb_to_ycocg(target: torch.Tensor, data: torch.Tensor, stream=None) -> None:
    """target, data: uint8 (..., 3 or 4) tensors (may be the same tensor)."""
    ch = data.shape[-1]
    check(lib().cc_convert_rgb_to_ycocg(_ptr(target), _ptr(data), data.numel() // ch, ch, _stream(stream)),
          "convertRGBtoYCoCg")


def convert_ycocg_to_rgb(target: torch.Tensor, data: torch.Tensor, stream=None) -> None:
    ch = data.shape[-1]
    check(lib().cc_convert_ycocg_to_rgb(_ptr(target), _ptr(data), data.numel() // ch, ch, _stream(stream)),
          "convertYCoCgtoRGB")


# --------------------------------------------------------------------- Bits
def get_lsb(data, bits, elem_count, stream=None):
    check(lib().cc_get_lsb(_ptr(data), _ptr(bits), elem_count, _stream(stream)), "getLSB")


def remove_lsb(data, bits, elem_count, shift=0, stream=None):
    check(lib().cc_remove_lsb(_ptr(data), _ptr(bits), elem_count, shift, _stream(stream)), "removeLSB")


def append_lsb(data, bits, elem_count, shift=0, stream=None):
    check(lib().cc_append_lsb(_ptr(data), _ptr(bits), elem_count, shift, _stream(stream)), "appendLSB")


def shift_elems(data, elem_count, shift, stream=None):
    check(lib().cc_shift_elems(_ptr(data), elem_count, shift, _stream(stream)), "shiftElems")


# ------------------------------------------------------------- image codec
def image_stream_capacity_words(size_x: int, size_y: int, channels: int) -> int:
    """Upper bound of one image level's stream in 32-bit words."""
    return int(size_x * size_y * channels * 24 // 32 + 64 * 1024)


def _image_dims(image: torch.Tensor):
    if image.dim() != 3 or image.dtype != torch.uint8:
        raise ValueError("image must be a (y, x, channels) uint8 tensor")
    return image.shape[1], image.shape[0], image.shape[2]


def compress_image_one_level(inst: Instance, image: torch.Tensor, channels_to_process: int,
                             lowpass_reference: torch.Tensor, quant_step: float,
                             out_words: Optional[torch.Tensor] = None):
    """compressImageOneLevel: image (y, x, c) uint8 CUDA tensor, overwritten
    with its reconstruction; lowpass_reference (y/2, x/2, c).  Returns (device
    words, bit size)."""
    sx, sy, ch = _image_dims(image)
    if out_words is None:
        out_words = torch.empty(image_stream_capacity_words(sx, sy, channels_to_process), dtype=torch.int32,
                                device=image.device)
    bits = ctypes.c_uint32()
    check(lib().cc_compress_image_one_level(inst.handle, image.data_ptr(), sx, sy, ch, channels_to_process,
                                            lowpass_reference.data_ptr(), quant_step, out_words.data_ptr(),
                                            out_words.numel(), ctypes.byref(bits)), "compressImageOneLevel")
    return out_words, bits.value


def decompress_image_one_level(inst: Instance, image: torch.Tensor, channels_to_process: int,
                               lowpass_reference: torch.Tensor, quant_step: float, words: torch.Tensor,
                               bit_size: int) -> None:
    sx, sy, ch = _image_dims(image)
    check(lib().cc_decompress_image_one_level(inst.handle, image.data_ptr(), sx, sy, ch, channels_to_process,
                                              lowpass_reference.data_ptr(), quant_step, words.data_ptr(), bit_size),
          "decompressImageOneLevel")


class _Image(ctypes.Structure):
    _fields_ = [("d_image", ctypes.c_void_p), ("d_lowpass_reference", ctypes.c_void_p),
                ("d_words", ctypes.c_void_p), ("capacity_words", ctypes.c_uint64), ("bit_size", ctypes.c_uint32),
                ("quant_step", ctypes.c_float)]


def compress_images_one_level(inst: Instance, images: Sequence[torch.Tensor], channels_to_process: int,
                              lowpass_references: Sequence[torch.Tensor], quant_steps: Sequence[float]):
    """compressImagesOneLevel: many images of one shape in one encode call.
    Returns [(device words, bit size)] per image."""
    n = len(images)
    sx, sy, ch = _image_dims(images[0])
    outs = [torch.empty(image_stream_capacity_words(sx, sy, channels_to_process), dtype=torch.int32,
                        device=images[0].device) for _ in range(n)]
    arr = (_Image * n)(*[_Image(im.data_ptr(), ref.data_ptr(), w.data_ptr(), w.numel(), 0, float(q))
                         for im, ref, w, q in zip(images, lowpass_references, outs, quant_steps)])
    check(lib().cc_compress_images_one_level(inst.handle, ctypes.cast(arr, ctypes.c_void_p), n, sx, sy, ch,
                                             channels_to_process), "compressImagesOneLevel")
    return [(outs[i], arr[i].bit_size) for i in range(n)]


def decompress_images_one_level(inst: Instance, images: Sequence[torch.Tensor], channels_to_process: int,
                                lowpass_references: Sequence[torch.Tensor], quant_steps: Sequence[float],
                                words: Sequence[torch.Tensor], bit_sizes: Sequence[int]) -> None:
    n = len(images)
    sx, sy, ch = _image_dims(images[0])
    arr = (_Image * n)(*[_Image(im.data_ptr(), ref.data_ptr(), w.data_ptr(), 0, int(b), float(q))
                         for im, ref, w, b, q in zip(images, lowpass_references, words, bit_sizes, quant_steps)])
    check(lib().cc_decompress_images_one_level(inst.handle, ctypes.cast(arr, ctypes.c_void_p), n, sx, sy, ch,
                                               channels_to_process), "decompressImagesOneLevel")


def get_lowpass_image(image: torch.Tensor, channels_to_process: int, out: Optional[torch.Tensor] = None,
                      stream=None) -> torch.Tensor:
    """getLowpassImage: (y/2, x/2, c) uint8 LL band of the processed channels."""
    sx, sy, ch = _image_dims(image)
    if out is None:
        out = torch.zeros((sy // 2, sx // 2, ch), dtype=torch.uint8, device=image.device)
    check(lib().cc_get_lowpass_image(image.data_ptr(), sx, sy, ch, channels_to_process, out.data_ptr(),
                                     _stream(stream)), "getLowpassImage")
    return out


# ----------------------------------------------------- one heightfield level
def compress_heightfield_one_level(inst: Instance, image: torch.Tensor, lowpass: torch.Tensor, lowpass_shift: int,
                                   out_words: Optional[torch.Tensor] = None):
    """compressHeightfieldOneLevel: image (y, x) int16; lowpass (y/2, x/2)
    int16 receives the truncated LL band.  Returns (device words, bit size)."""
    sy, sx = image.shape
    if out_words is None:
        out_words = torch.empty(sx * sy + 64 * 1024, dtype=torch.int32, device=image.device)
    bits = ctypes.c_uint32()
    check(lib().cc_compress_heightfield_one_level(inst.handle, image.data_ptr(), sx, sy, lowpass.data_ptr(),
                                                  lowpass_shift, out_words.data_ptr(), out_words.numel(),
                                                  ctypes.byref(bits)), "compressHeightfieldOneLevel")
    return out_words, bits.value


def decompress_heightfield_one_level(inst: Instance, image: torch.Tensor, lowpass: torch.Tensor, lowpass_shift: int,
                                     words: torch.Tensor, bit_size: int) -> None:
    sy, sx = image.shape
    check(lib().cc_decompress_heightfield_one_level(inst.handle, image.data_ptr(), sx, sy, lowpass.data_ptr(),
                                                    lowpass_shift, words.data_ptr(), bit_size),
          "decompressHeightfieldOneLevel")


def get_lowpass_heightfield(image: torch.Tensor, lowpass_shift: int, out: Optional[torch.Tensor] = None,
                            stream=None) -> torch.Tensor:
    sy, sx = image.shape
    if out is None:
        out = torch.empty((sy // 2, sx // 2), dtype=torch.int16, device=image.device)
    check(lib().cc_get_lowpass_heightfield(image.data_ptr(), sx, sy, out.data_ptr(), lowpass_shift, _stream(stream)),
          "getLowpassHeightfield")
    return out
