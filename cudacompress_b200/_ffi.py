"""ctypes bindings of the C ABI (include/cudacompress_b200.h).

Loading fails loudly when the CUDA library is missing: there is no CPU
fallback for any entry point.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libcudacompress_b200.so")

c_u32 = ctypes.c_uint32
c_u64 = ctypes.c_uint64
c_int = ctypes.c_int
c_float = ctypes.c_float
c_vp = ctypes.c_void_p
c_u32p = ctypes.POINTER(ctypes.c_uint32)
c_vpp = ctypes.POINTER(ctypes.c_void_p)

_SIGS = {
    "cc_last_error": (ctypes.c_char_p, []),
    "cc_version": (ctypes.c_char_p, []),
    "cc_kernel_launches": (c_u64, []),
    "cc_inject_allocation_failures": (c_int, [c_int, c_int]),
    "cc_create_instance": (c_int, [ctypes.POINTER(c_vp), c_int, c_u32, c_u32, c_u32, c_u32]),
    "cc_destroy_instance": (None, [c_vp]),
    "cc_get_instance_cuda_device": (c_int, [c_vp]),
    "cc_get_instance_stream_count_max": (c_u32, [c_vp]),
    "cc_get_instance_elem_count_per_stream_max": (c_u32, [c_vp]),
    "cc_get_instance_coding_block_size": (c_u32, [c_vp]),
    "cc_get_instance_log2_huffman_distinct_symbol_count_max": (c_u32, [c_vp]),
    "cc_get_instance_use_long_symbols": (c_int, [c_vp]),
    "cc_set_instance_stream": (None, [c_vp, c_vp]),
    "cc_get_instance_stream": (c_vp, [c_vp]),
    "cc_encode_get_required_memory": (ctypes.c_size_t, [c_vp]),
    "cc_set_timing": (None, [c_vp, c_int]),
    "cc_timing_count": (c_int, [c_vp]),
    "cc_timing_entry": (c_int, [c_vp, c_u32, ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(ctypes.c_double), c_u32p]),
    "cc_reset_timings": (None, [c_vp]),
    "cc_encode": (c_int, [c_vp, c_int, c_int, c_vpp, c_u32, c_u32, c_u32p]),
    "cc_encoded_segment": (c_int, [c_vp, c_u32, ctypes.POINTER(c_u32p), c_u32p, c_u32p, c_u32p]),
    "cc_encode_to_buffer": (c_int, [c_vp, c_int, c_int, c_vpp, c_u32, c_u32, c_u32p, c_u32, c_u32p, c_u32p]),
    "cc_decode": (c_int, [c_vp, c_int, c_int, ctypes.POINTER(c_u32p), c_u32p, c_u32p, c_u32, c_u32p, c_vpp, c_u32, c_u32]),
    "cc_decode_status": (c_int, [c_vp]),
    "cc_dwt_float_forward": (c_int, [c_vp, c_vp, c_vp, c_vp, c_int, c_int, c_int, c_int, c_int, c_int, c_int, c_int, c_vp]),
    "cc_dwt_float_inverse": (c_int, [c_vp, c_vp, c_vp, c_vp, c_int, c_int, c_int, c_int, c_int, c_int, c_int, c_int, c_vp]),
    "cc_dwt_float_inverse_from_symbols": (c_int, [c_vp, c_vp, c_vp, c_vp, c_vp, c_int, c_float, c_int, c_int, c_int,
                                                  c_int, c_int, c_int, c_int, c_int, c_vp]),
    "cc_dwt_float_forward_static": (c_int, [c_vp, c_vp, c_int, c_int, c_int, c_int, c_int, c_int, c_int, c_int, c_vp]),
    "cc_dwt_int_forward": (c_int, [c_vp, c_vp, c_vp, c_int, c_int, c_int, c_int, c_int, c_int, c_int, c_vp]),
    "cc_dwt_int_inverse": (c_int, [c_vp, c_vp, c_vp, c_int, c_int, c_int, c_int, c_int, c_int, c_int, c_vp]),
    "cc_quantize_to_symbols": (c_int, [c_vp, c_int, c_vp, c_u32, c_u32, c_u32, c_float, c_u32, c_u32, c_int, c_vp]),
    "cc_quantize_to_symbols_roundtrip": (c_int, [c_vp, c_int, c_vp, c_u32, c_u32, c_u32, c_float, c_u32, c_u32, c_int, c_vp]),
    "cc_unquantize_from_symbols": (c_int, [c_vp, c_vp, c_int, c_u32, c_u32, c_u32, c_float, c_u32, c_u32, c_int, c_vp]),
    "cc_symbolize": (c_int, [c_vp, c_vp, c_u32, c_u32, c_u32, c_u32, c_u32, c_vp]),
    "cc_unsymbolize": (c_int, [c_vp, c_vp, c_u32, c_u32, c_u32, c_u32, c_u32, c_vp]),
    "cc_quantize_to_short": (c_int, [c_vp, c_vp, c_u32, c_u32, c_u32, c_float, c_u32, c_u32, c_int, c_vp]),
    "cc_unquantize_from_short": (c_int, [c_vp, c_vp, c_u32, c_u32, c_u32, c_float, c_u32, c_u32, c_int, c_vp]),
    "cc_get_max_abs": (c_int, [c_vp, c_vp, c_u32, c_vp]),
    "cc_compress_volume_float": (c_int, [c_vp, c_vp, c_u32, c_u32, c_u32, c_u32, c_float, c_vp, c_u64, c_u32p]),
    "cc_decompress_volume_float": (c_int, [c_vp, c_vp, c_u32, c_u32, c_u32, c_u32, c_float, c_vp, c_u32]),
    "cc_compress_volume_float_ex": (c_int, [c_vp, c_vp, c_u32, c_u32, c_u32, c_u32, c_float, c_u32, c_vp, c_u64,
                                            c_u32p]),
    "cc_decompress_volume_float_ex": (c_int, [c_vp, c_vp, c_u32, c_u32, c_u32, c_u32, c_float, c_u32, c_vp, c_u32]),
    "cc_decompress_volume_float_multichannel": (c_int, [c_vp, c_vp, c_u32, c_u32, c_u32, c_u32, c_u32, c_u32]),
    "cc_compress_volume_float_quant_first": (c_int, [c_vp, c_vp, c_u32, c_u32, c_u32, c_u32, c_float, c_u32, c_vp,
                                                     c_u64, c_u32p]),
    "cc_decompress_volume_float_quant_first": (c_int, [c_vp, c_vp, c_u32, c_u32, c_u32, c_u32, c_float, c_u32, c_vp,
                                                       c_u32]),
    "cc_decompress_volume_float_quant_first_multichannel": (c_int, [c_vp, c_vp, c_u32, c_u32, c_u32, c_u32, c_u32,
                                                                    c_u32]),
    "cc_compress_heightfield": (c_int, [c_vp, c_vp, c_u32, c_u32, c_u32, c_vp, c_u64, c_u32p]),
    "cc_decompress_heightfield": (c_int, [c_vp, c_vp, c_u32, c_u32, c_u32, c_vp, c_u32]),
    "cc_dwt_float_forward_from_byte": (c_int, [c_vp, c_vp, c_vp, c_vp, c_int, c_int, c_int, c_int, c_int, c_int,
                                               c_int, c_int, c_vp]),
    "cc_dwt_float_inverse_to_byte": (c_int, [c_vp, c_vp, c_vp, c_vp, c_int, c_int, c_int, c_int, c_int, c_int, c_int,
                                             c_int, c_vp]),
    "cc_dwt_float_inverse_from_symbols_to_byte": (c_int, [c_vp, c_vp, c_vp, c_vp, c_vp, c_int, c_float, c_int, c_int,
                                                          c_int, c_int, c_int, c_int, c_int, c_int, c_vp]),
    "cc_dwt_float2d_forward_lowpass_only_from_byte": (c_int, [c_vp, c_vp, c_vp, c_int, c_int, c_int, c_int, c_int,
                                                              c_vp]),
    "cc_dwt_int_forward_lowpass_only": (c_int, [c_vp, c_vp, c_vp, c_int, c_int, c_int, c_int, c_vp]),
    "cc_float_to_byte_2d": (c_int, [c_vp, c_u32, c_u32, c_vp, c_u32, c_u32, c_u32, c_vp]),
    "cc_byte_to_float_2d": (c_int, [c_vp, c_vp, c_u32, c_u32, c_u32, c_u32, c_u32, c_vp]),
    "cc_quantize_difference_to_symbols_2d": (c_int, [c_vp, c_vp, c_float, c_vp, c_u32, c_u32, c_u32, c_u32, c_u32,
                                                     c_int, c_vp]),
    "cc_quantize_difference_to_symbols_roundtrip_2d": (c_int, [c_vp, c_vp, c_float, c_vp, c_u32, c_u32, c_u32, c_u32,
                                                               c_u32, c_int, c_vp]),
    "cc_unquantize_difference_from_symbols_2d": (c_int, [c_vp, c_vp, c_float, c_vp, c_u32, c_u32, c_u32, c_u32, c_u32,
                                                         c_int, c_vp]),
    "cc_convert_rgb_to_ycocg": (c_int, [c_vp, c_vp, c_int, c_int, c_vp]),
    "cc_convert_ycocg_to_rgb": (c_int, [c_vp, c_vp, c_int, c_int, c_vp]),
    "cc_get_lsb": (c_int, [c_vp, c_vp, c_u32, c_vp]),
    "cc_remove_lsb": (c_int, [c_vp, c_vp, c_u32, ctypes.c_int16, c_vp]),
    "cc_append_lsb": (c_int, [c_vp, c_vp, c_u32, ctypes.c_int16, c_vp]),
    "cc_shift_elems": (c_int, [c_vp, c_u32, ctypes.c_int16, c_vp]),
    "cc_compress_heightfield_one_level": (c_int, [c_vp, c_vp, c_u32, c_u32, c_vp, ctypes.c_int16, c_vp, c_u64,
                                                  c_u32p]),
    "cc_decompress_heightfield_one_level": (c_int, [c_vp, c_vp, c_u32, c_u32, c_vp, ctypes.c_int16, c_vp, c_u32]),
    "cc_get_lowpass_heightfield": (c_int, [c_vp, c_int, c_int, c_vp, ctypes.c_int16, c_vp]),
    "cc_compress_image_one_level": (c_int, [c_vp, c_vp, c_u32, c_u32, c_u32, c_u32, c_vp, c_float, c_vp, c_u64,
                                            c_u32p]),
    "cc_decompress_image_one_level": (c_int, [c_vp, c_vp, c_u32, c_u32, c_u32, c_u32, c_vp, c_float, c_vp, c_u32]),
    "cc_compress_images_one_level": (c_int, [c_vp, c_vp, c_u32, c_u32, c_u32, c_u32, c_u32]),
    "cc_decompress_images_one_level": (c_int, [c_vp, c_vp, c_u32, c_u32, c_u32, c_u32, c_u32]),
    "cc_get_lowpass_image": (c_int, [c_vp, c_int, c_int, c_int, c_int, c_vp, c_vp]),
    "cc_container_bytes": (c_u64, [c_u32, ctypes.POINTER(c_u64)]),
    "cc_container_write": (c_int, [c_vp, c_u64, c_vp, c_vp, c_u32, ctypes.POINTER(c_u64)]),
    "cc_container_read": (c_int, [c_vp, c_u64, c_vp, c_vp, c_u32, c_u32p]),
    "cc_volume_batch_create": (c_int, [c_vp, c_u32, c_u32p, c_u32, ctypes.POINTER(c_float), ctypes.POINTER(c_vp)]),
    "cc_volume_batch_create_ex": (c_int, [c_vp, c_u32, c_u32p, c_u32, ctypes.POINTER(c_float), c_u32,
                                          ctypes.POINTER(c_vp)]),
    "cc_volume_batch_destroy": (None, [c_vp]),
    "cc_volume_batch_use_graph": (c_int, [c_vp, c_int]),
    "cc_volume_batch_set_active": (c_int, [c_vp, c_u32]),
    "cc_volume_batch_set_stream": (c_int, [c_vp, c_vp]),
    "cc_volume_batch_compress": (c_int, [c_vp, c_vpp]),
    "cc_volume_batch_decompress": (c_int, [c_vp, c_vpp]),
    "cc_volume_batch_stream": (c_int, [c_vp, ctypes.POINTER(c_vp), ctypes.POINTER(c_vp), ctypes.POINTER(c_vp),
                                       ctypes.POINTER(c_u64)]),
    "cc_volume_batch_read_stream": (c_int, [c_vp, c_u32, c_vp, c_u64, ctypes.POINTER(c_u64)]),
    "cc_volume_batch_load_streams": (c_int, [c_vp, c_vpp, ctypes.POINTER(c_u64)]),
    "cc_volume_batch_download_streams": (c_int, [c_vp, c_vp, c_u64, c_vp]),
    "cc_volume_batch_upload_streams": (c_int, [c_vp, c_vp, c_vp]),
    "cc_volume_batch_status": (c_int, [c_vp]),
    "cc_volume_batch_collect_timings": (None, [c_vp]),
}

_lib = None


def exported_names():
    """Every entry point this module binds (the C header's declarations)."""
    return sorted(_SIGS)


def lib() -> ctypes.CDLL:
    """The loaded CUDA library; raises if it was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"cudacompress_b200 CUDA library not found at {LIB_PATH}; build it with "
                "`python -m cudacompress_b200.build` (there is no CPU fallback)")
        l = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(l, name)
            f.restype = res
            f.argtypes = args
        _lib = l
    return _lib


class CudaCompressError(RuntimeError):
    def __init__(self, status: int, what: str):
        msg = lib().cc_last_error().decode(errors="replace")
        super().__init__(f"{what}: status {status}: {msg}")
        self.status = status


def check(status: int, what: str) -> None:
    if status != 0:
        raise CudaCompressError(status, what)
