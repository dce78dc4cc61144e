// capi_internal.cuh - declarations shared by the library's translation units.
#pragma once

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <vector>

#include "../../include/cudacompress_b200.h"
#include "codec.cuh"

namespace ccb {

// Counts kernel launches issued by this library (cc_kernel_launches).
void countLaunch(unsigned n = 1);

void setError(const char* fmt, ...);
int cudaFail(cudaError_t e, const char* what);

// Every device (cudaMalloc) and page-locked host (cudaHostAlloc) allocation
// of the library goes through these, so that a test can make chosen ones
// fail as an out-of-memory would (cc_inject_allocation_failures).
cudaError_t deviceAlloc(void** p, size_t bytes);
cudaError_t pinnedAlloc(void** p, size_t bytes);

// Makes `device` current for the scope of an entry point and restores the
// caller's current device on exit (the reference's calls leave it alone).
struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int device) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (device >= 0 && device != prev) cudaSetDevice(device);
    }
    ~DeviceGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
    DeviceGuard(const DeviceGuard&) = delete;
    DeviceGuard& operator=(const DeviceGuard&) = delete;
};

// Capacities of an instance made for a batch of volumes (instead of the
// reference's streamCountMax x elemCountPerStreamMax contract).
struct InstanceCaps {
    u32 streams;      // streams of one call
    u64 symbols;      // run-length symbols of one call
    u64 histBins;     // histogram bins of one call
};
int createInstance(cc_instance** out, int cudaDevice, u32 streamCountMax, u32 elemCountPerStreamMax,
                   u32 codingBlockSize, u32 log2Max, const InstanceCaps* caps);

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
// The same in two steps, for callers that keep the descriptors on the device
// and replay the launches (batches, CUDA graphs): encodePrepare writes the
// descriptors to a host buffer; the caller copies them to plan.dev; then
// encodeLaunch enqueues only kernels and device memsets.
struct EncPlan {
    u32 S = 0, T = 0, tiles = 0, blocks = 0, maxCount = 0;
    u64 compact = 0;
    size_t offTables = 0, bytes = 0;
    const void* dev = nullptr;
};
int encodePrepare(cc_instance* I, const EncStream* streams, u32 S, char* slot, size_t slotBytes, EncPlan& plan);
int encodeLaunch(cc_instance* I, const EncPlan& plan, u32* out, u64 outCap);
// Grows the instance's pipeline workspace to at least `bytes` (allocates only when it must grow).
int ensurePipelineWork(cc_instance* I, size_t bytes);
// One reference encode call of a codec pipeline: `count` streams from `first`.
struct EncGroup {
    u32 first, count;
};
// Encodes groups of streams back to back into dWords (pipeline.cu); with
// groupStart, entry k receives the first word of group k and entry
// groups.size() the end of the last.
int encodeGroups(cc_instance* I, const std::vector<EncStream>& streams, const std::vector<EncGroup>& groups,
                 u32* dWords, u64 cap, u64* wordsOut, std::vector<u64>* groupStart = nullptr);
int decodeDevice(cc_instance* I, int kind, const u32* const* words, const u32* bitSizes, u32* bitPos, u32 bsCount,
                 const u32* bsIndex, void* const* outs, u32 S, u32 n);

// Decode of device-resident bit streams walked on the device, in two steps
// like the encoder: decodePrepare writes the descriptors of stream i (kind,
// n symbols into out) read from source streams[i].source - the streams of one
// source consecutive and in stream order from its startBit - into a host
// buffer; decodeLaunch enqueues the walk and the decode (kernels and device
// memsets only).  A source's words are words + wordOff[k] with bitSize[k]
// bits when the plan gives device arrays for them (the output of a batched
// encode), else the pointer and size given here.  Errors surface through the
// instance's decode status.
struct DecStreamSpec {
    u32 kind;
    u32 n;
    void* out;
    u32 source;
};
struct DecSourceSpec {
    const u32* words;
    u64 bitSize;
    u64 startBit;
};
struct DecPlan {
    u32 S = 0, T = 0, B = 0, nRl = 0, nH = 0, rlBlocks = 0, hBlocks = 0;
    u32 rlMaxN = 0;   // largest output of an RLHuff stream (symbols)
    size_t bytes = 0;
    size_t offStreams = 0, offTables = 0, offSources = 0, offRl = 0, offH = 0;   // within dev
    void* dev = nullptr;
    const u32* wordsBase = nullptr;   // with wordOff / bitSize: indirect sources
    const u64* wordOff = nullptr;
    const u64* bitSize = nullptr;
};
int decodePrepare(cc_instance* I, const DecStreamSpec* streams, u32 S, const DecSourceSpec* sources, u32 B,
                  char* slot, size_t slotBytes, DecPlan& plan);
int decodeLaunch(cc_instance* I, const DecPlan& plan);

// Per-device cache of the dynamic shared memory limits set on kernels (so
// that repeated launches, and launches recorded in a stream capture, do not
// set them again): returns cudaSuccess once the kernel allows `bytes`.
enum SmemAttrKernel {
    kAttrTableBuild = 0,
    kAttrDecHuff16,
    kAttrDecHuff32,
    kAttrWrite16,
    kAttrWrite32,
    kAttrCount
};
cudaError_t ensureSmemAttribute(const void* kernel, int which, int device, size_t bytes);
// Sets the largest shared memory the encoder and decoder kernels may ask for
// on the instance's device.
int prepareKernelAttributes(cc_instance* I);
// Batched encode: per volume (streams first[v] .. first[v+1]-1) its word
// offset and bit size in the output, from the device layout.
void volumeExtents(cc_instance* I, const u32* first, u32 count, u64* wordOff, u64* bitSize, cudaStream_t st);

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
