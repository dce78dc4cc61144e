/*
 * cudacompress_b200.h - C ABI of the B200-native cudaCompress hot path.
 *
 * Plain pointers and sizes only.  Device pointers are CUDA device addresses
 * (e.g. from cudaMalloc or a framework allocator); streams are cudaStream_t
 * passed as void*.  Every function returning int returns CC_OK (0) or a
 * negative status; cc_last_error() describes the last failure on the calling
 * thread.  The C++ drop-in layer (include/cudaCompress/*.h, namespace
 * cudaCompress) is built on these entry points.
 *
 * Each declaration cites the reference interface it replaces (paths relative
 * to the cudaCompress project root).
 */
#ifndef CUDACOMPRESS_B200_H
#define CUDACOMPRESS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CC_OK 0
#define CC_ERR_INVALID_ARGUMENT (-1)
#define CC_ERR_CUDA (-2)
#define CC_ERR_OUT_OF_MEMORY (-3)
#define CC_ERR_SYMBOL_RANGE (-4)
#define CC_ERR_CODEWORD_TOO_LONG (-5)
#define CC_ERR_CORRUPT_STREAM (-6)
#define CC_ERR_CAPACITY (-7)
#define CC_ERR_DEVICE_TIMEOUT (-8)

#define CC_KIND_RLHUFF 0
#define CC_KIND_HUFF 1

typedef struct cc_instance cc_instance;

/* Last error message of the calling thread ("" if none). */
const char* cc_last_error(void);
/* Kernel launches issued by the library in this process so far. */
uint64_t cc_kernel_launches(void);
/* Library version string. */
const char* cc_version(void);
/* Test hook, no counterpart in the reference: the library's next `skip`
 * device or page-locked host allocations succeed, then the following `fail`
 * report out-of-memory without allocating (every entry point must then
 * return a status and release what it holds).  0, 0 turns it off; returns
 * the previous pending failure count. */
int cc_inject_allocation_failures(int skip, int fail);

/* ---- Instance (include/cudaCompress/Instance.h:26-45, src/cudaCompress/Instance.cpp:8-67) ---- */

/* createInstance(cudaDevice, streamCountMax, elemCountPerStreamMax,
 * codingBlockSize = 0 -> 128, log2HuffmanDistinctSymbolCountMax = 0 -> 14).
 * Instance.h:26-31.  *out is NULL on failure. */
int cc_create_instance(cc_instance** out, int cuda_device, uint32_t stream_count_max,
                       uint32_t elem_count_per_stream_max, uint32_t coding_block_size,
                       uint32_t log2_huffman_distinct_symbol_count_max);
/* destroyInstance, Instance.h:33. */
void cc_destroy_instance(cc_instance* inst);
/* getInstance* queries, Instance.h:36-41. */
int cc_get_instance_cuda_device(const cc_instance* inst);
uint32_t cc_get_instance_stream_count_max(const cc_instance* inst);
uint32_t cc_get_instance_elem_count_per_stream_max(const cc_instance* inst);
uint32_t cc_get_instance_coding_block_size(const cc_instance* inst);
uint32_t cc_get_instance_log2_huffman_distinct_symbol_count_max(const cc_instance* inst);
int cc_get_instance_use_long_symbols(const cc_instance* inst);
/* setInstanceCudaStream / getInstanceCudaStream, Instance.h:44-45
 * (defined as setInstanceStream / getInstanceStream in Instance.cpp:59-67). */
void cc_set_instance_stream(cc_instance* inst, void* cuda_stream);
void* cc_get_instance_stream(const cc_instance* inst);
/* encodeGetRequiredMemory, Encode.h:17: device bytes the instance holds. */
size_t cc_encode_get_required_memory(const cc_instance* inst);

/* Kernel timing (Timing.h:15-27 / util::CudaTimer): when enabled, named
 * sections are timed with CUDA events on the instance stream and accumulated
 * per name.  cc_timing_count resolves pending sections (synchronizing) and
 * returns the number of names; cc_timing_entry reads one (name, total
 * milliseconds, section count). */
void cc_set_timing(cc_instance* inst, int enable);
int cc_timing_count(cc_instance* inst);
int cc_timing_entry(cc_instance* inst, uint32_t i, const char** name, double* ms, uint32_t* count);
void cc_reset_timings(cc_instance* inst);

/* ---- Entropy coding (include/cudaCompress/Encode.h:28-52, src/cudaCompress/Encode.cpp:207-1042) ----
 *
 * Encode: `kind` CC_KIND_RLHUFF (encodeRLHuff) or CC_KIND_HUFF (encodeHuff);
 * `symbol_bytes` 2 (Symbol16) or 4 (Symbol32, instances with log2Max > 16).
 * d_streams[i] holds symbol_count_per_stream symbols.  Input buffers are not
 * modified (the reference pads encodeHuff inputs; this library needs no
 * padding).  The result is one segment per stream, each a run of 32-bit
 * words; start_bits[i] (0..31, NULL = all 0) is the bit offset, inside its
 * first word, at which stream i's segment starts - only meaningful for
 * encodeHuff streams that start a bit stream at an unaligned position.
 * Segments stay in the instance's host staging until the next call.
 * Synchronous, like the reference (Encode.cpp:394,744). */
int cc_encode(cc_instance* inst, int kind, int symbol_bytes, const void* const* d_streams,
              uint32_t stream_count, uint32_t symbol_count_per_stream, const uint32_t* start_bits);
/* Segment i of the last cc_encode: host words, word count, bit offset of its
 * first bit in word 0, and bit length measured from word 0 bit 0. */
int cc_encoded_segment(const cc_instance* inst, uint32_t i, const uint32_t** words, uint32_t* word_count,
                       uint32_t* start_bit, uint32_t* bit_length);

/* Convenience form of the single-bit-stream overloads (Encode.h:28-38): the
 * bit stream is a caller-owned word buffer with its bit size and write
 * position (in/out), appended to exactly as BitStream::write* would.
 * CC_ERR_CAPACITY (with *bit_size = required bits) if it does not fit. */
int cc_encode_to_buffer(cc_instance* inst, int kind, int symbol_bytes, const void* const* d_streams,
                        uint32_t stream_count, uint32_t symbol_count_per_stream, uint32_t* words,
                        uint32_t capacity_words, uint32_t* bit_size, uint32_t* bit_pos);

/* Decode (decodeRLHuff / decodeHuff, Encode.h:29-52).  Stream i is read from
 * bit stream bs_index[i] (NULL = all from bit stream 0) of `bitstream_count`
 * host word buffers; positions advance in stream order.  Every output
 * symbol is written (the reference asks the caller to zero decodeRLHuff's
 * outputs first, Encode.h:22; here that is not needed, and harmless); no
 * output padding is required.  Asynchronous on the instance stream: returns once the work is
 * queued; host memory may be reused on return. */
int cc_decode(cc_instance* inst, int kind, int symbol_bytes, const uint32_t* const* words,
              const uint32_t* bit_sizes, uint32_t* bit_positions, uint32_t bitstream_count,
              const uint32_t* bs_index, void* const* d_out_streams, uint32_t stream_count,
              uint32_t symbol_count_per_stream);

/* Synchronizes the instance stream and reports whether the last decode found
 * the bit stream corrupt (CC_ERR_CORRUPT_STREAM) - the device-side checks of
 * an asynchronous decode surface here. */
int cc_decode_status(cc_instance* inst);

/* ---- util::DWT (include/cudaCompress/util/DWT.h:21-157, src/cudaCompress/util/DWTFloat.cu, DWTInt.cu) ----
 * Same argument meaning as the reference; pitches in elements, 0 = tight;
 * channel counts 1..4; all sizes even.  stream: cudaStream_t as void*. */
int cc_dwt_float_forward(float* d_dst, float* d_buf2, float* d_buf1, const float* d_src, int size_x, int size_y,
                         int size_z, int src_channel_count, int dst_row_pitch, int dst_slice_pitch,
                         int src_row_pitch, int src_slice_pitch, void* stream);
int cc_dwt_float_inverse(float* d_dst, float* d_buf2, float* d_buf1, const float* d_src, int size_x, int size_y,
                         int size_z, int dst_channel_count, int dst_row_pitch, int dst_slice_pitch,
                         int src_row_pitch, int src_slice_pitch, void* stream);
/* dwtFloat{2D,3D}InverseFromSymbols: d_highpass is a device array of 3 (2D) or
 * 7 (3D) device pointers to the quantized highpass bands (band index
 * x+2y+4z-1); symbol_bytes 2 or 4. */
int cc_dwt_float_inverse_from_symbols(float* d_dst, float* d_buf2, float* d_buf1, const float* d_lowpass,
                                      const void* const* d_highpass, int symbol_bytes, float quant_step,
                                      int size_x, int size_y, int size_z, int dst_channel_count,
                                      int dst_row_pitch, int dst_slice_pitch, int lowpass_row_pitch,
                                      int lowpass_slice_pitch, void* stream);
/* Byte variants (DWT.h:79-123): dwtFloat{2D,3D}ForwardFromByte reads one
 * channel of an interleaved byte image (b -> b - 128; d_src addresses the
 * channel, src_channel_count 1..4); ...InverseToByte and
 * ...InverseFromSymbolsToByte write one channel of one
 * (v -> clamp(v + 128.5, 0, 255), truncated).  2D: size_z = 1, d_buf2 unused. */
int cc_dwt_float_forward_from_byte(float* d_dst, float* d_buf2, float* d_buf1, const uint8_t* d_src, int size_x,
                                   int size_y, int size_z, int src_channel_count, int dst_row_pitch,
                                   int dst_slice_pitch, int src_row_pitch, int src_slice_pitch, void* stream);
int cc_dwt_float_inverse_to_byte(uint8_t* d_dst, float* d_buf2, float* d_buf1, const float* d_src, int size_x,
                                 int size_y, int size_z, int dst_channel_count, int dst_row_pitch, int dst_slice_pitch,
                                 int src_row_pitch, int src_slice_pitch, void* stream);
int cc_dwt_float_inverse_from_symbols_to_byte(uint8_t* d_dst, float* d_buf2, float* d_buf1, const float* d_lowpass,
                                              const void* const* d_highpass, int symbol_bytes, float quant_step,
                                              int size_x, int size_y, int size_z, int dst_channel_count,
                                              int dst_row_pitch, int dst_slice_pitch, int lowpass_row_pitch,
                                              int lowpass_slice_pitch, void* stream);
/* dwtFloat2DForwardLowpassOnlyFromByte (DWT.h:126-131): only the LL band of
 * one 2D level (size_x/2 x size_y/2, row pitch default size_x/2).  d_buf is
 * accepted for the reference's signature and not used. */
int cc_dwt_float2d_forward_lowpass_only_from_byte(float* d_dst, float* d_buf, const uint8_t* d_src, int size_x,
                                                  int size_y, int src_channel_count, int dst_row_pitch,
                                                  int src_row_pitch, void* stream);
/* No counterpart in the reference (whose dwtFloat{2D,3D}Forward take two
 * caller-allocated buffers): cc_dwt_float_forward with both intermediates in
 * a fixed 8 MiB device array inside this library, for callers that cannot
 * allocate device memory (under a host allocator lock, inside a stream
 * capture, or in a host application that owns the device memory pool).
 * Limit: (size_z-1)*dst_slice_pitch + (size_y-1)*dst_row_pitch + size_x
 * <= 2^20 floats (e.g. 128 x 128 x 64, or 1024 x 1024 in 2D); larger volumes
 * are rejected with CC_ERR_CAPACITY.  Runs on the current device; its first
 * call there resolves the array's device address (make it before any stream
 * capture); that address is kept for the life of the process, so after a
 * cudaDeviceReset on that device this entry point must not be called again.
 * Calls share the array: calls that overlap on the GPU race. */
int cc_dwt_float_forward_static(float* d_dst, const float* d_src, int size_x, int size_y, int size_z,
                                int src_channel_count, int dst_row_pitch, int dst_slice_pitch, int src_row_pitch,
                                int src_slice_pitch, void* stream);
int cc_dwt_int_forward(int16_t* d_dst, int16_t* d_buf, const int16_t* d_src, int size_x, int size_y, int size_z,
                       int dst_row_pitch, int dst_slice_pitch, int src_row_pitch, int src_slice_pitch, void* stream);
int cc_dwt_int_inverse(int16_t* d_dst, int16_t* d_buf, const int16_t* d_src, int size_x, int size_y, int size_z,
                       int dst_row_pitch, int dst_slice_pitch, int src_row_pitch, int src_slice_pitch, void* stream);
/* dwtIntForwardLowpassOnly (DWT.h:152-157): only the LL band of one 2D
 * level of the 5/3 lifting (row pitch default size_x/2); d_buf not used.
 * The reference fills only whole blocks of 512 columns x 64 rows; this
 * computes every LL sample (identical where the reference writes one). */
int cc_dwt_int_forward_lowpass_only(int16_t* d_dst, int16_t* d_buf, const int16_t* d_src, int size_x, int size_y,
                                    int dst_row_pitch, int src_row_pitch, void* stream);

/* ---- util::Quantize (include/cudaCompress/util/Quantize.h:25-65, src/cudaCompress/util/Quantize.cu) ----
 * quant_type 0 = QUANTIZE_DEADZONE, 1 = QUANTIZE_UNIFORM.  The reference
 * launches these on the default stream; `stream` NULL does the same. */
int cc_quantize_to_symbols(void* d_symbols, int symbol_bytes, const float* d_data, uint32_t size_x,
                           uint32_t size_y, uint32_t size_z, float quant_step, uint32_t row_pitch_src,
                           uint32_t slice_pitch_src, int quant_type, void* stream);
int cc_quantize_to_symbols_roundtrip(void* d_symbols, int symbol_bytes, float* d_data, uint32_t size_x,
                                     uint32_t size_y, uint32_t size_z, float quant_step, uint32_t row_pitch_src,
                                     uint32_t slice_pitch_src, int quant_type, void* stream);
int cc_unquantize_from_symbols(float* d_data, const void* d_symbols, int symbol_bytes, uint32_t size_x,
                               uint32_t size_y, uint32_t size_z, float quant_step, uint32_t row_pitch_dst,
                               uint32_t slice_pitch_dst, int quant_type, void* stream);
int cc_symbolize(uint16_t* d_symbols, const int16_t* d_data, uint32_t size_x, uint32_t size_y, uint32_t size_z,
                 uint32_t row_pitch_src, uint32_t slice_pitch_src, void* stream);
int cc_unsymbolize(int16_t* d_data, const uint16_t* d_symbols, uint32_t size_x, uint32_t size_y, uint32_t size_z,
                   uint32_t row_pitch_dst, uint32_t slice_pitch_dst, void* stream);
int cc_quantize_to_short(int16_t* d_quant, const float* d_data, uint32_t size_x, uint32_t size_y, uint32_t size_z,
                         float quant_step, uint32_t row_pitch_src, uint32_t slice_pitch_src, int quant_type,
                         void* stream);
int cc_unquantize_from_short(float* d_data, const int16_t* d_quant, uint32_t size_x, uint32_t size_y,
                             uint32_t size_z, float quant_step, uint32_t row_pitch_dst, uint32_t slice_pitch_dst,
                             int quant_type, void* stream);
/* getMaxAbs(pInstance, dpImage, elemCount, dpValMax): max |x| into d_max. */
int cc_get_max_abs(cc_instance* inst, const float* d_data, uint32_t elem_count, float* d_max);
/* Byte images (Quantize.h:24-26, 58-61): channel `channel` of a byte image
 * with `channel_count` interleaved channels (dense, size_x per row).
 * floatToByte: clamp(v + 128.5, 0, 255) truncated; byteToFloat: b - 128.
 * quantizeDifference*: the float minus the byte reference (b - 128),
 * quantized to 16-bit symbols; the round trip writes back reference + the
 * stored symbol's value.  unquantizeDifference is its inverse.  The
 * reference launches these on the default stream (unquantizeDifference
 * takes a stream); `stream` NULL does the same. */
int cc_float_to_byte_2d(uint8_t* d_quant, uint32_t channel_count, uint32_t channel, const float* d_data,
                        uint32_t size_x, uint32_t size_y, uint32_t row_pitch_src, void* stream);
int cc_byte_to_float_2d(float* d_data, const uint8_t* d_quant, uint32_t channel_count, uint32_t channel,
                        uint32_t size_x, uint32_t size_y, uint32_t row_pitch_dst, void* stream);
int cc_quantize_difference_to_symbols_2d(uint16_t* d_symbols, const float* d_data, float quant_step,
                                         const uint8_t* d_reference, uint32_t channel_count, uint32_t channel,
                                         uint32_t size_x, uint32_t size_y, uint32_t row_pitch_src, int quant_type,
                                         void* stream);
int cc_quantize_difference_to_symbols_roundtrip_2d(uint16_t* d_symbols, float* d_data, float quant_step,
                                                   const uint8_t* d_reference, uint32_t channel_count,
                                                   uint32_t channel, uint32_t size_x, uint32_t size_y,
                                                   uint32_t row_pitch_src, int quant_type, void* stream);
int cc_unquantize_difference_from_symbols_2d(float* d_data, const uint16_t* d_symbols, float quant_step,
                                             const uint8_t* d_reference, uint32_t channel_count, uint32_t channel,
                                             uint32_t size_x, uint32_t size_y, uint32_t row_pitch_dst,
                                             int quant_type, void* stream);

/* ---- util::YCoCg (include/cudaCompress/util/YCoCg.h:14-20) ----
 * RGB <-> YCoCg of `pixel_count` pixels of `channels` bytes (3 = uchar3,
 * 4 = uchar4, the 4th byte copied; uchar4 pixels 4-byte aligned); in place
 * allowed.  Y = (R + 2G + B + 2) / 4, Co = (R - B + 1) / 2 + 127,
 * Cg = (2G - R - B + 2) / 4 + 127 (integer division), inverse clamped. */
int cc_convert_rgb_to_ycocg(uint8_t* d_target, const uint8_t* d_data, int pixel_count, int channels, void* stream);
int cc_convert_ycocg_to_rgb(uint8_t* d_target, const uint8_t* d_data, int pixel_count, int channels, void* stream);

/* ---- util::Bits (include/cudaCompress/util/Bits.h:14-27) ----
 * Bit j of word w of d_bits belongs to element 32 w + j (ceil(n/32) words).
 * removeLSB: v -> (v + shift) with its lowest bit removed (floor of half),
 * the removed bits into d_bits when not NULL; appendLSB: v -> 2v + bit +
 * shift.  The reference processes whole blocks of 4096 elements (its callers
 * pad); these touch exactly elem_count elements, bits past it are 0. */
int cc_get_lsb(const int16_t* d_data, uint32_t* d_bits, uint32_t elem_count, void* stream);
int cc_remove_lsb(int16_t* d_data, uint32_t* d_bits, uint32_t elem_count, int16_t shift, void* stream);
int cc_append_lsb(int16_t* d_data, const uint32_t* d_bits, uint32_t elem_count, int16_t shift, void* stream);
int cc_shift_elems(int16_t* d_data, uint32_t elem_count, int16_t shift, void* stream);

/* ---- Volume / heightfield codecs (examples CompressVolume.cpp:312-516, CompressHeightfield.cpp:82-216) ----
 * Whole-pipeline entry points: device-resident input, device-resident bit
 * stream (32-bit words).  The byte stream equals the reference pipeline's
 * (LP encodeHuff, then per level coarse->fine the HP bands encodeRLHuff).
 * *bit_size receives the stream length; capacity in words. */
int cc_compress_volume_float(cc_instance* inst, const float* d_volume, uint32_t size_x, uint32_t size_y,
                             uint32_t size_z, uint32_t levels, float quant_step_level0, uint32_t* d_words,
                             uint64_t capacity_words, uint32_t* bit_size);
int cc_decompress_volume_float(cc_instance* inst, float* d_volume, uint32_t size_x, uint32_t size_y,
                               uint32_t size_z, uint32_t levels, float quant_step_level0, const uint32_t* d_words,
                               uint32_t bit_size);
/* Variants of examples/CompressVolume.h:60-79.  flags: CC_VOLUME_RLE_ONLY_LEVEL0
 * (doRLEOnlyOnLvl0: the levels above 0 code their bands with encodeHuff
 * instead of encodeRLHuff, CompressVolume.cpp:389-395, 491-495). */
#define CC_VOLUME_RLE_ONLY_LEVEL0 1u
int cc_compress_volume_float_ex(cc_instance* inst, const float* d_volume, uint32_t size_x, uint32_t size_y,
                                uint32_t size_z, uint32_t levels, float quant_step_level0, uint32_t flags,
                                uint32_t* d_words, uint64_t capacity_words, uint32_t* bit_size);
int cc_decompress_volume_float_ex(cc_instance* inst, float* d_volume, uint32_t size_x, uint32_t size_y,
                                  uint32_t size_z, uint32_t levels, float quant_step_level0, uint32_t flags,
                                  const uint32_t* d_words, uint32_t bit_size);
/* One channel of a multi-channel decode (VolumeChannel, CompressVolume.h:36-42):
 * its output volume, its device bit stream and its quantization step. */
typedef struct cc_volume_channel {
    float* d_volume;
    const uint32_t* d_words;
    uint32_t bit_size;
    float quant_step;
} cc_volume_channel;
/* decompressVolumeFloatMultiChannel (CompressVolume.cpp:518-648): `count`
 * volumes of the same sizes; all lowpass streams in one decode call, each
 * level's bands of all channels in one call.  The instance needs
 * 7 * count streams.  Results equal `count` single-channel decodes. */
int cc_decompress_volume_float_multichannel(cc_instance* inst, const cc_volume_channel* channels, uint32_t count,
                                            uint32_t size_x, uint32_t size_y, uint32_t size_z, uint32_t levels,
                                            uint32_t flags);
/* compressVolumeFloatQuantFirst / decompressVolumeFloatQuantFirst(MultiChannel)
 * (CompressVolume.cpp:651-988): uniform quantization to short, integer DWT,
 * symbolize, then the same stream layout; error <= quant_step / 2.  The
 * reference's decoder reads the wrong ping-pong buffer for odd level counts;
 * this one inverts every level count correctly (streams are identical). */
int cc_compress_volume_float_quant_first(cc_instance* inst, const float* d_volume, uint32_t size_x,
                                         uint32_t size_y, uint32_t size_z, uint32_t levels, float quant_step,
                                         uint32_t flags, uint32_t* d_words, uint64_t capacity_words,
                                         uint32_t* bit_size);
int cc_decompress_volume_float_quant_first(cc_instance* inst, float* d_volume, uint32_t size_x, uint32_t size_y,
                                           uint32_t size_z, uint32_t levels, float quant_step, uint32_t flags,
                                           const uint32_t* d_words, uint32_t bit_size);
int cc_decompress_volume_float_quant_first_multichannel(cc_instance* inst, const cc_volume_channel* channels,
                                                        uint32_t count, uint32_t size_x, uint32_t size_y,
                                                        uint32_t size_z, uint32_t levels, uint32_t flags);
int cc_compress_heightfield(cc_instance* inst, const int16_t* d_image, uint32_t size_x, uint32_t size_y,
                            uint32_t levels, uint32_t* d_words, uint64_t capacity_words, uint32_t* bit_size);
int cc_decompress_heightfield(cc_instance* inst, int16_t* d_image, uint32_t size_x, uint32_t size_y,
                              uint32_t levels, const uint32_t* d_words, uint32_t bit_size);
/* One heightfield level (examples CompressHeightfield.cpp:82-216): the stream
 * holds the ceil(n/32) words of the least significant bits of (LL + shift),
 * n = size_x/2 * size_y/2, then one encodeRLHuff call over the 3 symbolized
 * highpass bands.  d_lowpass (n shorts) receives (LL + shift) without that
 * bit; decompress appends the bit to it in place and adds its own shift
 * (appendLSB), then rebuilds the image - so, as in the reference, shift 0 on
 * both sides (or the negated shift to decompress) reproduces the image.
 * getLowpassHeightfield (:218-235): the same d_lowpass, without coding. */
int cc_compress_heightfield_one_level(cc_instance* inst, const int16_t* d_image, uint32_t size_x, uint32_t size_y,
                                      int16_t* d_lowpass, int16_t lowpass_shift, uint32_t* d_words,
                                      uint64_t capacity_words, uint32_t* bit_size);
int cc_decompress_heightfield_one_level(cc_instance* inst, int16_t* d_image, uint32_t size_x, uint32_t size_y,
                                        int16_t* d_lowpass, int16_t lowpass_shift, const uint32_t* d_words,
                                        uint32_t bit_size);
int cc_get_lowpass_heightfield(const int16_t* d_image, int size_x, int size_y, int16_t* d_lowpass,
                               int16_t lowpass_shift, void* stream);

/* ---- one image level (examples CompressImage.h:36-71, CompressImage.cpp) ----
 * Byte images with channel_count_total interleaved channels (1..4), of which
 * the first channel_count_to_process are coded.  Per channel: 9/7 DWT, the
 * LL band minus the lowpass reference (a size_x/2 x size_y/2 byte image with
 * the same interleaving, normally the decoded next-coarser level) and the 3
 * highpass bands round-trip quantized with quant_step; compress overwrites
 * d_image with the reconstruction.  Stream: one encodeRLHuff call over the
 * LL-difference streams of all channels, then each channel's 3 bands.
 * Colour conversion is the caller's (cc_convert_rgb_to_ycocg). */
int cc_compress_image_one_level(cc_instance* inst, uint8_t* d_image, uint32_t size_x, uint32_t size_y,
                                uint32_t channel_count_total, uint32_t channel_count_to_process,
                                const uint8_t* d_lowpass_reference, float quant_step, uint32_t* d_words,
                                uint64_t capacity_words, uint32_t* bit_size);
int cc_decompress_image_one_level(cc_instance* inst, uint8_t* d_image, uint32_t size_x, uint32_t size_y,
                                  uint32_t channel_count_total, uint32_t channel_count_to_process,
                                  const uint8_t* d_lowpass_reference, float quant_step, const uint32_t* d_words,
                                  uint32_t bit_size);
/* Many images of the same sizes (Image / ImageV, compressImagesOneLevel):
 * one DWT/quantize sequence per image, one encode (decode) call for all.
 * Compress fills bit_size; decompress reads d_words / bit_size.  Decompress
 * needs an instance with 4 x channels x count streams. */
typedef struct cc_image {
    uint8_t* d_image;
    const uint8_t* d_lowpass_reference;
    uint32_t* d_words;
    uint64_t capacity_words;      /* compress only */
    uint32_t bit_size;
    float quant_step;
} cc_image;
int cc_compress_images_one_level(cc_instance* inst, cc_image* images, uint32_t count, uint32_t size_x,
                                 uint32_t size_y, uint32_t channel_count_total, uint32_t channel_count_to_process);
int cc_decompress_images_one_level(cc_instance* inst, const cc_image* images, uint32_t count, uint32_t size_x,
                                   uint32_t size_y, uint32_t channel_count_total,
                                   uint32_t channel_count_to_process);
/* getLowpassImage (CompressImage.cpp:342-365): the LL band of one 9/7 level
 * of each processed channel, as bytes (floatToByte), into d_lowpass
 * (size_x/2 x size_y/2, channel_count_total interleaved channels). */
int cc_get_lowpass_image(const uint8_t* d_image, int size_x, int size_y, int channel_count_total,
                         int channel_count_to_process, uint8_t* d_lowpass, void* stream);

/* ---- stream container (B200 addition; no counterpart in the reference) ----
 * The reference's example stores a stream as raw concatenated u32 words
 * (examples.cpp:527-536), leaving codec, levels, sizes and steps to the
 * caller.  This container keeps them with the streams (layout in
 * cudacompress_b200/csrc/container.cu).  Host memory only. */
typedef struct cc_container_info {
    uint32_t codec;               /* 0 float volume, 1 quant-first volume, 2 heightfield */
    uint32_t flags;               /* CC_VOLUME_RLE_ONLY_LEVEL0 */
    uint32_t levels;
    uint32_t coding_block_size;
    uint32_t log2_symbol_count;
} cc_container_info;
typedef struct cc_container_entry {
    uint32_t size_x, size_y, size_z;
    float quant_step;
    uint64_t bit_size;
    const uint32_t* words;        /* host; on read: points into the container */
} cc_container_entry;
/* Bytes of a container holding `count` streams of the given bit sizes. */
uint64_t cc_container_bytes(uint32_t count, const uint64_t* bit_sizes);
int cc_container_write(void* dst, uint64_t capacity, const cc_container_info* info, const cc_container_entry* entries,
                       uint32_t count, uint64_t* written);
/* entries NULL: *count receives the entry count only. */
int cc_container_read(const void* src, uint64_t bytes, cc_container_info* info, cc_container_entry* entries,
                      uint32_t capacity, uint32_t* count);

/* ---- batched volume codec (B200 addition; callers: CompressVolume.cpp:312-516) ----
 * Compresses and decompresses `count` float32 volumes of any sizes (each
 * divisible by 2^levels, coarsest level >= 8) with one launch per stage for
 * the whole batch.  Each volume's stream is byte-identical to
 * cc_compress_volume_float's with its own quantization step.  Planned once
 * at creation (its own device memory; the instance gives device, stream,
 * coding block size and symbol range, which must be 16-bit); compress and
 * decompress only enqueue work on the instance stream (no host
 * synchronization) and, with cc_volume_batch_use_graph, replay it as one
 * CUDA graph.  sizes: x, y, z per volume. */
typedef struct cc_volume_batch cc_volume_batch;
int cc_volume_batch_create(cc_instance* inst, uint32_t count, const uint32_t* sizes, uint32_t levels,
                           const float* quant_steps, cc_volume_batch** out);
/* The same with the forward transform's tile depth: each CTA of a level's
 * fused pass codes z_chunk output slices (0 = the default 32; else even,
 * 8..256).  A
 * tuning knob only (cudacompress_b200.autotune): the streams do not change. */
int cc_volume_batch_create_ex(cc_instance* inst, uint32_t count, const uint32_t* sizes, uint32_t levels,
                              const float* quant_steps, uint32_t z_chunk, cc_volume_batch** out);
void cc_volume_batch_destroy(cc_volume_batch* batch);
int cc_volume_batch_use_graph(cc_volume_batch* batch, int enable);
/* Later calls process only the first `active` volumes (1..count); pointer
 * arrays and loaded streams then cover those volumes. */
int cc_volume_batch_set_active(cc_volume_batch* batch, uint32_t active);
/* Runs the batch's work on `stream` (cudaStream_t) instead of the instance
 * stream, so that several batches can overlap on the device. */
int cc_volume_batch_set_stream(cc_volume_batch* batch, void* stream);
/* d_volumes: `count` device pointers (dense x-fastest volumes). */
int cc_volume_batch_compress(cc_volume_batch* batch, const float* const* d_volumes);
/* Decodes the batch's own streams (those of the last compress, or streams
 * written into the buffer cc_volume_batch_stream returns). */
int cc_volume_batch_decompress(cc_volume_batch* batch, float* const* d_volumes);
/* Device views of the streams: words, per-volume word offset and bit size. */
int cc_volume_batch_stream(const cc_volume_batch* batch, const uint32_t** d_words, const uint64_t** d_word_offsets,
                           const uint64_t** d_bit_sizes, uint64_t* capacity_words);
/* Synchronizes and copies volume v's stream (host or device dst; NULL dst:
 * size only). */
int cc_volume_batch_read_stream(cc_volume_batch* batch, uint32_t volume, uint32_t* dst, uint64_t capacity_words,
                                uint64_t* bit_size);
/* Loads `count` streams (host or device words, bit sizes) back to back into
 * the batch's buffer for cc_volume_batch_decompress (e.g. streams of
 * cc_compress_volume_float or of another batch with the same shapes). */
int cc_volume_batch_load_streams(cc_volume_batch* batch, const uint32_t* const* words, const uint64_t* bit_sizes);
/* The streams of the active volumes between the batch and page-locked host
 * memory (cudaHostAlloc / cudaHostRegister), fully asynchronous on the
 * batch's stream: kernels move exactly the used words, whose extent only the
 * device knows, so the host never waits.  h_extents: 2 x active u64, the word
 * offset of each stream in h_words, then each bit size.  download after a
 * compress; upload (the same layout) before a decompress.  A download larger
 * than capacity_words, or an upload larger than the batch's buffer, is
 * reported by cc_volume_batch_status. */
int cc_volume_batch_download_streams(cc_volume_batch* batch, uint32_t* h_words, uint64_t capacity_words,
                                     uint64_t* h_extents);
int cc_volume_batch_upload_streams(cc_volume_batch* batch, const uint32_t* h_words, const uint64_t* h_extents);
/* Synchronizes the instance stream; reports device errors of the last calls. */
int cc_volume_batch_status(cc_volume_batch* batch);
/* Adds the batch's timing sections to the instance's (cc_timing_*). */
void cc_volume_batch_collect_timings(cc_volume_batch* batch);

#ifdef __cplusplus
}
#endif

#endif /* CUDACOMPRESS_B200_H */
