// capi_internal.cuh - declarations shared by the library's translation units.
#pragma once

#include <algorithm>
#include <cstdarg>
#include <cstdio>

#include "../../include/cudacompress_b200.h"
#include "codec.cuh"

namespace ccb {

// Counts kernel launches issued by this library (cc_kernel_launches).
void countLaunch(unsigned n = 1);

void setError(const char* fmt, ...);
int cudaFail(cudaError_t e, const char* what);

// Maps the device error flags of a call to a status (and message).
inline int deviceErrorStatus(u32 flags, const char* what) {
    if (!flags) return CC_OK;
    if (flags & DEV_ERR_SYMBOL_RANGE) { setError("%s: symbol out of range for log2HuffmanDistinctSymbolCountMax", what); return CC_ERR_SYMBOL_RANGE; }
    if (flags & DEV_ERR_CODEWORD_TOO_LONG) { setError("%s: Huffman codeword longer than 31 bits", what); return CC_ERR_CODEWORD_TOO_LONG; }
    if (flags & DEV_ERR_TIMEOUT) { setError("%s: device wait timed out", what); return CC_ERR_DEVICE_TIMEOUT; }
    if (flags & DEV_ERR_TABLE_CAPACITY) { setError("%s: tables exceed the instance capacity", what); return CC_ERR_CAPACITY; }
    if (flags & DEV_ERR_OUTPUT_CAPACITY) { setError("%s: output buffer too small", what); return CC_ERR_CAPACITY; }
    setError("%s: corrupt or truncated bit stream", what);
    return CC_ERR_CORRUPT_STREAM;
}

#define CC_TRY_CUDA(expr, what)                                  \
    do {                                                         \
        cudaError_t _e = (expr);                                 \
        if (_e != cudaSuccess) return ::ccb::cudaFail(_e, what); \
    } while (0)

// Encode / decode entry points used by the C ABI and the fused pipelines.
// `streams` are host descriptors of any sizes and kinds; the segments are
// written back to back (each word aligned) into `out.words` (device, at most
// `out.capacity` words) or, when that is null, the instance output buffer.
// The call waits for the device; the layout is kept in I->lastLayout.
struct EncOutput {
    u32* words = nullptr;
    u64 capacity = 0;
};
int encodeDevice(cc_instance* I, const EncStream* streams, u32 S, const EncOutput& out, bool download,
                 u64* totalWords = nullptr);
// Grows the instance's pipeline workspace to at least `bytes` (allocates only when it must grow).
int ensurePipelineWork(cc_instance* I, size_t bytes);
int decodeDevice(cc_instance* I, int kind, const u32* const* words, const u32* bitSizes, u32* bitPos, u32 bsCount,
                 const u32* bsIndex, void* const* outs, u32 S, u32 n);

// Records a named, event-timed section on the instance stream when the
// instance has timing enabled (setTimingDetail / cc_set_timing).
struct SectionTimer {
    cc_instance* I;
    const char* name;
    cudaStream_t st;
    cudaEvent_t a = nullptr;
    SectionTimer(cc_instance* inst, const char* n, cudaStream_t s) : I(inst), name(n), st(s) {
        if (I && I->timing) {
            a = I->takeEvent();
            cudaEventRecord(a, st);
        }
    }
    ~SectionTimer() {
        if (a) {
            cudaEvent_t b = I->takeEvent();
            cudaEventRecord(b, st);
            I->pendingSections.push_back({name, a, b});
        }
    }
};

}  // namespace ccb
