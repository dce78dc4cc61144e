// capi_internal.cuh - declarations shared by the library's translation units.
#pragma once

#include <algorithm>
#include <cstdarg>
#include <cstdio>

#include "../../include/cudacompress_b200.h"
#include "codec.cuh"

namespace ccb {

void setError(const char* fmt, ...);
int cudaFail(cudaError_t e, const char* what);
u32 headerWordsFor(u32 leaves, u32 log2Max);
u64 segmentWordsMax(u32 n, u32 cb, u32 log2Max, u32 hdrWords);

// Maps the device error flags of a call to a status (and message).
inline int deviceErrorStatus(u32 flags, const char* what) {
    if (!flags) return CC_OK;
    if (flags & DEV_ERR_SYMBOL_RANGE) { setError("%s: symbol out of range for log2HuffmanDistinctSymbolCountMax", what); return CC_ERR_SYMBOL_RANGE; }
    if (flags & DEV_ERR_CODEWORD_TOO_LONG) { setError("%s: Huffman codeword longer than 31 bits", what); return CC_ERR_CODEWORD_TOO_LONG; }
    if (flags & DEV_ERR_TIMEOUT) { setError("%s: device wait timed out", what); return CC_ERR_DEVICE_TIMEOUT; }
    if (flags & DEV_ERR_TABLE_CAPACITY) { setError("%s: table exceeds instance capacity", what); return CC_ERR_CAPACITY; }
    setError("%s: corrupt or truncated bit stream", what);
    return CC_ERR_CORRUPT_STREAM;
}

#define CC_TRY_CUDA(expr, what)                                  \
    do {                                                         \
        cudaError_t _e = (expr);                                 \
        if (_e != cudaSuccess) return ::ccb::cudaFail(_e, what); \
    } while (0)

// Encode / decode entry points used by the C ABI and the fused pipelines.
// `streams` are host descriptors; results land in the instance buffers.
int encodeDevice(cc_instance* I, int kind, const EncStream* streams, u32 S, bool download, u64* totalWords = nullptr);
// Grows the instance's pipeline workspace to at least `bytes` (allocates only when it must grow).
int ensurePipelineWork(cc_instance* I, size_t bytes);
int decodeDevice(cc_instance* I, int kind, const u32* const* words, const u32* bitSizes, u32* bitPos, u32 bsCount,
                 const u32* bsIndex, void* const* outs, u32 S, u32 n);

}  // namespace ccb
