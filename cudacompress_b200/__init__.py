"""cudacompress_b200: B200-native (sm_100a) implementation of cudaCompress's
compress/decompress hot path - float/int DWT, quantization, zero-run RLE and
Huffman coding - behind the reference's C++ API (include/cudaCompress/*.h)
and a C ABI (include/cudacompress_b200.h).  This package holds the Python
mirror of that API over torch CUDA tensors."""
from ._ffi import CudaCompressError, LIB_PATH, exported_names, lib  # noqa: F401
from .codec import (  # noqa: F401
    HUFF, QUANTIZE_DEADZONE, QUANTIZE_UNIFORM, RLE_ONLY_LEVEL0, RLHUFF, BitStream, Instance, compress_heightfield,
    compress_volume_float, compress_volume_float_quant_first, decode_huff, decode_rlhuff, decode_status,
    decompress_heightfield, decompress_volume_float, decompress_volume_float_multichannel, decompress_volume_float_quant_first,
    dwt_float2d_forward_lowpass_only_from_byte, dwt_float_forward, dwt_float_forward_from_byte, dwt_float_inverse,
    dwt_float_inverse_from_symbols, dwt_float_inverse_from_symbols_to_byte, dwt_float_inverse_to_byte,
    dwt_int_forward, dwt_int_forward_lowpass_only, dwt_int_inverse, encode_huff, encode_rlhuff, get_max_abs, last_error, quantize_to_short, quantize_to_symbols,
    quantize_to_symbols_roundtrip, symbolize, unquantize_from_short, unquantize_from_symbols, unsymbolize,
    volume_stream_capacity_words, VolumeBatch)

from . import image  # noqa: F401,E402

__version__ = "0.1.0"
