// instance.cu - cc_instance lifetime, device arena and host staging
// (replaces Instance.cpp:8-67 and InstanceImpl.cpp:46-279 of the reference).
//
// All device memory an instance needs is allocated once at creation, sized
// from (streamCountMax, elemCountPerStreamMax, codingBlockSize,
// log2HuffmanDistinctSymbolCountMax); calls never allocate.
#include <atomic>
#include <cstring>
#include <iterator>
#include <string>

#include "capi_internal.cuh"

using namespace ccb;

namespace ccb {

static thread_local std::string g_lastError;
static std::atomic<unsigned long long> g_launches{0};

void countLaunch(unsigned n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

void setError(const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_lastError = buf;
}

// Allocation fault injection (cc_inject_allocation_failures): the next
// `skip` allocations succeed, then `fail` of them report
// cudaErrorMemoryAllocation without allocating.
static std::atomic<int> g_allocSkip{0}, g_allocFail{0};

static bool injectedFailure() {
    if (g_allocFail.load(std::memory_order_relaxed) <= 0) return false;
    int s = g_allocSkip.load();
    while (s > 0) {
        if (g_allocSkip.compare_exchange_weak(s, s - 1)) return false;
    }
    int f = g_allocFail.load();
    while (f > 0) {
        if (g_allocFail.compare_exchange_weak(f, f - 1)) return true;
    }
    return false;
}

cudaError_t deviceAlloc(void** p, size_t bytes) {
    if (injectedFailure()) { *p = nullptr; return cudaErrorMemoryAllocation; }
    return cudaMalloc(p, bytes);
}

cudaError_t pinnedAlloc(void** p, size_t bytes) {
    if (injectedFailure()) { *p = nullptr; return cudaErrorMemoryAllocation; }
    return cudaHostAlloc(p, bytes, cudaHostAllocDefault);
}

int cudaFail(cudaError_t e, const char* what) {
    setError("%s: %s", what, cudaGetErrorString(e));
    // the error is reported here: clear it from the runtime's per-thread
    // last error (a failed allocation is not sticky), so that a later call's
    // launch check does not report it again
    (void)cudaGetLastError();
    return e == cudaErrorMemoryAllocation ? CC_ERR_OUT_OF_MEMORY : CC_ERR_CUDA;
}

static std::atomic<size_t> g_smemSet[64][kAttrCount];

cudaError_t ensureSmemAttribute(const void* kernel, int which, int device, size_t bytes) {
    if (device < 0 || device >= 64) return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
    std::atomic<size_t>& cur = g_smemSet[device][which];
    if (cur.load() >= bytes) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
    if (e == cudaSuccess) {
        size_t c = cur.load();
        while (c < bytes && !cur.compare_exchange_weak(c, bytes)) {}
    }
    return e;
}

int ensurePipelineWork(cc_instance* I, size_t bytes) {
    if (I->pipeWorkBytes >= bytes) return CC_OK;
    cudaStreamSynchronize(I->stream);
    if (I->pipeWork) cudaFree(I->pipeWork);
    I->pipeWork = nullptr;
    I->pipeWorkBytes = 0;
    cudaError_t e = deviceAlloc(reinterpret_cast<void**>(&I->pipeWork), bytes);
    if (e != cudaSuccess) return cudaFail(e, "cudaMalloc(pipeline workspace)");
    I->pipeWorkBytes = bytes;
    return CC_OK;
}

}  // namespace ccb

cudaEvent_t cc_instance::takeEvent() {
    if (!freeEvents.empty()) {
        cudaEvent_t e = freeEvents.back();
        freeEvents.pop_back();
        return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
}

void cc_instance::resolveTimings() {
    for (const Section& s : pendingSections) {
        cudaEventSynchronize(s.b);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, s.a, s.b);
        auto& acc = timings[s.name];
        acc.first += ms;
        acc.second += 1;
        freeEvents.push_back(s.a);
        freeEvents.push_back(s.b);
    }
    pendingSections.clear();
}

char* cc_instance::takeRingSlot() {
    int i = ringNext;
    ringNext = (ringNext + 1) % kRing;
    cudaEventSynchronize(ringEvent[i]);
    return hostRing[i];
}

namespace {

struct Carver {
    char* base;
    size_t off = 0;
    template <class T>
    T* take(u64 count) {
        off = alignUp(off, 256);
        T* p = reinterpret_cast<T*>(base + off);
        off += count * sizeof(T);
        return p;
    }
};

void layoutArena(cc_instance* I, char* base, size_t* total) {
    Carver c{base};
    I->compact = c.take<char>(I->capCompact * I->symBytes + 64);
    I->zc = c.take<char>((I->capCompact + 8ull * I->capStreams) * I->symBytes + 64);   // per stream 16-byte aligned
    I->tiles = c.take<RunSum>(I->capTiles);
    I->tileStart = c.take<TileStart>(I->capTiles);
    I->streamMax = c.take<u32>(I->capStreams);
    I->hist = c.take<u32>(I->capHist);
    I->enc = c.take<uint2>(I->capHist);
    I->meta = c.take<TableMeta>(I->capTables);
    I->tierTables = c.take<u32>(4ull * I->capTables);
    I->planPart = c.take<u64>(2 * planPartWords(I->capTables));   // encode's, then decode's
    I->headers = c.take<u32>(I->capHdr);
    I->blockBits = c.take<u32>(I->capBlocks + 1);
    I->blockOff = c.take<u32>(I->capBlocks + 1);
    I->blockTable = c.take<u32>(I->capBlocks + 1);
    I->runTable = c.take<u32>(I->capBlocks + 1);
    I->tileStream = c.take<u32>(I->capTiles + 1);
    I->layout = c.take<SegmentLayout>(I->capStreams);
    I->out = c.take<u32>(I->outWordsMax);
    I->counts = c.take<u32>(I->capStreams);
    I->errors = c.take<u32>(8);
    I->totals = c.take<u64>(8);
    I->dPlan = c.take<char>(I->hostRingBytes);
    I->leafWork = c.take<u64>(I->capLeaves);
    I->parentWork = c.take<u32>(2 * I->capLeaves);
    I->orderWork = c.take<u32>(I->capLeaves);
    I->leafSymWork = c.take<u32>(I->capLeaves);
    // decode (one call of at most streamCountMax streams)
    // decode
    I->decTables = c.take<DecTable>(I->capTables);
    I->decSyms = c.take<u32>(I->capLeaves + 1);
    I->decLut = c.take<u32>(u64(I->capTables) << kLutBits);
    I->stagedWordsMax = I->hostWordsMax + 64;
    I->stagedWords = c.take<u32>(I->stagedWordsMax);
    I->blockSum = c.take<u32>(I->capBlocks + 1);
    I->decRlTasks = c.take<u64>(u64(I->capBlocks) / 32 + I->capStreams + 2);
    *total = alignUp(c.off, 256);
}

// Capacities of one encode or decode call.  The instance promises
// streamCountMax streams of elemCountPerStreamMax symbols; internally a call
// may split the same symbol budget over up to capStreams streams of any
// sizes.  An instance made for a batch of volumes gets its capacities from
// `caps` instead.
void sizeCapacities(cc_instance* I, const InstanceCaps* caps) {
    const u32 S = I->streamCountMax;
    const u64 SN = caps ? caps->symbols : u64(S) * I->elemCountPerStreamMax;
    I->capStreams = caps ? caps->streams : std::max<u32>(S, 1024u);
    I->capTables = 2 * I->capStreams;
    I->capCompact = SN;
    I->capTiles = u32(ceilDiv(SN, kRleTile) + I->capStreams);
    I->capBlocks = u32(2 * (ceilDiv(SN, I->codingBlockSize) + I->capStreams));
    // histograms: at most 2^log2Max bins for symbols and 256 for zero counts
    // per stream of a full call (a batch gives a bin budget instead; the
    // device plan checks every call against it)
    I->capHist = caps ? caps->histBins : u64(S) * I->bins + u64(S) * std::min<u32>(256u, I->bins);
    I->capLeaves = std::min<u64>(I->capHist, 2 * SN + I->capTables);
    const u64 symBits = I->log2Max > 16 ? 24 : 16;
    I->capHdr = u64(I->capTables) * (headerWordsFor(0, I->log2Max) + 1) + ceilDiv(I->capLeaves * symBits, 32);
    // output: headers + per-segment words + codewords (a Huffman code is never
    // longer than a fixed-length one: log2Max bits per symbol, 8 per zero
    // count) + 16-bit offsets
    I->outWordsMax = I->capHdr + 16ull * I->capStreams + ceilDiv(SN * (I->log2Max + 8), 32) +
                     ceilDiv(SN, I->codingBlockSize) + 64;
    I->hostWordsMax = caps ? 1024 : I->outWordsMax;   // batches keep their results on the device
    const u64 encPlan = u64(I->capStreams) * sizeof(EncStreamDev) + 64 + u64(I->capTables) * sizeof(EncTableDev);
    const u64 decPlan = u64(I->capStreams) * (sizeof(DecStreamDesc) + sizeof(DecSource) + 2 * sizeof(u32)) +
                        u64(I->capTables) * sizeof(DecTableDesc) + 5 * 64;
    I->hostRingBytes = alignUp(std::max(encPlan, decPlan) + 4096, 4096);
}

}  // namespace

extern "C" {

const char* cc_last_error(void) { return g_lastError.c_str(); }
uint64_t cc_kernel_launches(void) { return g_launches.load(); }
const char* cc_version(void) { return "cudacompress_b200 0.1 (sm_100a)"; }

int cc_create_instance(cc_instance** out, int cudaDevice, uint32_t streamCountMax, uint32_t elemCountPerStreamMax,
                       uint32_t codingBlockSize, uint32_t log2Max) {
    return ccb::createInstance(out, cudaDevice, streamCountMax, elemCountPerStreamMax, codingBlockSize, log2Max, nullptr);
}

}  // extern "C"

namespace ccb {

int createInstance(cc_instance** out, int cudaDevice, u32 streamCountMax, u32 elemCountPerStreamMax,
                   u32 codingBlockSize, u32 log2Max, const InstanceCaps* caps) {
    if (!out) { setError("cc_create_instance: out is NULL"); return CC_ERR_INVALID_ARGUMENT; }
    *out = nullptr;
    if (codingBlockSize == 0) codingBlockSize = 128;          // InstanceImpl.cpp:65-69
    if (log2Max == 0) log2Max = 14;                           // InstanceImpl.cpp:71-75
    if (log2Max > 24) { setError("log2HuffmanDistinctSymbolCountMax must be <= 24 (got %u)", log2Max); return CC_ERR_INVALID_ARGUMENT; }
    if (codingBlockSize != 32 && codingBlockSize != 64 && codingBlockSize != 128 && codingBlockSize != 256) {
        setError("codingBlockSize must be 32, 64, 128 or 256 (got %u)", codingBlockSize);  // Huffman.h:42
        return CC_ERR_INVALID_ARGUMENT;
    }
    if (streamCountMax == 0 || elemCountPerStreamMax == 0) { setError("stream/elem count max must be > 0"); return CC_ERR_INVALID_ARGUMENT; }
    cudaError_t e;
    if (cudaDevice >= 0) {
        if ((e = cudaSetDevice(cudaDevice)) != cudaSuccess) return cudaFail(e, "cudaSetDevice");
    } else {
        if ((e = cudaGetDevice(&cudaDevice)) != cudaSuccess) return cudaFail(e, "cudaGetDevice");
    }
    cc_instance* I = new cc_instance();
    I->device = cudaDevice;
    I->streamCountMax = streamCountMax;
    I->elemCountPerStreamMax = elemCountPerStreamMax;
    I->codingBlockSize = codingBlockSize;
    I->log2Max = log2Max;
    I->bins = 1u << log2Max;
    I->symBytes = log2Max > 16 ? 4 : 2;
    I->tilesMax = u32(ceilDiv(elemCountPerStreamMax, kRleTile));
    I->blocksMax = u32(ceilDiv(elemCountPerStreamMax, codingBlockSize));
    I->leavesMax = std::max<u32>(1u, std::min<u32>(I->bins, elemCountPerStreamMax));
    I->hdrWordsMax = headerWordsFor(I->leavesMax, log2Max);
    if (u64(streamCountMax) * elemCountPerStreamMax > (1ull << 36)) {
        delete I;
        setError("streamCountMax * elemCountPerStreamMax must be <= 2^36");
        return CC_ERR_INVALID_ARGUMENT;
    }
    sizeCapacities(I, caps);

    size_t bytes = 0;
    layoutArena(I, nullptr, &bytes);
    if ((e = deviceAlloc(reinterpret_cast<void**>(&I->arena), bytes)) != cudaSuccess) { delete I; return cudaFail(e, "cudaMalloc(instance arena)"); }
    I->arenaBytes = bytes;
    layoutArena(I, I->arena, &bytes);
    cudaMemset(I->arena, 0, bytes);

    for (int i = 0; i < cc_instance::kRing; ++i) {
        if ((e = pinnedAlloc(reinterpret_cast<void**>(&I->hostRing[i]), I->hostRingBytes)) != cudaSuccess) {
            cc_destroy_instance(I);
            return cudaFail(e, "cudaHostAlloc(ring)");
        }
        cudaEventCreateWithFlags(&I->ringEvent[i], cudaEventDisableTiming);
        cudaEventRecord(I->ringEvent[i], 0);
    }
    I->hostDownBytes = alignUp(u64(I->capStreams) * sizeof(SegmentLayout) + 256, 4096);
    if ((e = pinnedAlloc(reinterpret_cast<void**>(&I->hostDown), I->hostDownBytes)) != cudaSuccess) {
        cc_destroy_instance(I);
        return cudaFail(e, "cudaHostAlloc(down)");
    }
    if ((e = pinnedAlloc(reinterpret_cast<void**>(&I->hostWords), I->hostWordsMax * 4)) != cudaSuccess) {
        cc_destroy_instance(I);
        return cudaFail(e, "cudaHostAlloc(words)");
    }
    if ((e = cudaStreamCreateWithFlags(&I->buildSide, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&I->buildSide2, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&I->buildFork, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&I->buildJoin, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&I->buildJoin2, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&I->decFork, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&I->decJoin, cudaEventDisableTiming)) != cudaSuccess) {
        cc_destroy_instance(I);
        return cudaFail(e, "table build stream");
    }
    if ((e = cudaDeviceSynchronize()) != cudaSuccess) { cc_destroy_instance(I); return cudaFail(e, "instance init"); }
    *out = I;
    return CC_OK;
}

}  // namespace ccb

extern "C" {

int cc_inject_allocation_failures(int skip, int fail) {
    const int prev = g_allocFail.load();
    g_allocSkip.store(skip > 0 ? skip : 0);
    g_allocFail.store(fail > 0 ? fail : 0);
    return prev;
}

void cc_destroy_instance(cc_instance* I) {
    if (!I) return;
    int prev = -1;
    cudaGetDevice(&prev);
    if (I->device >= 0) cudaSetDevice(I->device);
    cudaDeviceSynchronize();
    for (auto& pb : I->plainBatch)
        if (pb.b) cc_volume_batch_destroy(pb.b);   // they refer to this instance
    for (int i = 0; i < cc_instance::kRing; ++i) {
        if (I->ringEvent[i]) cudaEventDestroy(I->ringEvent[i]);
        if (I->hostRing[i]) cudaFreeHost(I->hostRing[i]);
    }
    if (I->hostDown) cudaFreeHost(I->hostDown);
    if (I->hostWords) cudaFreeHost(I->hostWords);
    if (I->buildFork) cudaEventDestroy(I->buildFork);
    if (I->buildJoin) cudaEventDestroy(I->buildJoin);
    if (I->buildJoin2) cudaEventDestroy(I->buildJoin2);
    if (I->decFork) cudaEventDestroy(I->decFork);
    if (I->decJoin) cudaEventDestroy(I->decJoin);
    if (I->buildSide) cudaStreamDestroy(I->buildSide);
    if (I->buildSide2) cudaStreamDestroy(I->buildSide2);
    I->resolveTimings();
    for (cudaEvent_t e : I->freeEvents) cudaEventDestroy(e);
    if (I->arena) cudaFree(I->arena);
    if (I->pipeWork) cudaFree(I->pipeWork);
    if (prev >= 0) cudaSetDevice(prev);
    delete I;
}

int cc_get_instance_cuda_device(const cc_instance* I) { return I ? I->device : -1; }
uint32_t cc_get_instance_stream_count_max(const cc_instance* I) { return I ? I->streamCountMax : 0; }
uint32_t cc_get_instance_elem_count_per_stream_max(const cc_instance* I) { return I ? I->elemCountPerStreamMax : 0; }
uint32_t cc_get_instance_coding_block_size(const cc_instance* I) { return I ? I->codingBlockSize : 0; }
uint32_t cc_get_instance_log2_huffman_distinct_symbol_count_max(const cc_instance* I) { return I ? I->log2Max : 0; }
int cc_get_instance_use_long_symbols(const cc_instance* I) { return I && I->log2Max > 16 ? 1 : 0; }
void cc_set_instance_stream(cc_instance* I, void* s) { if (I) I->stream = static_cast<cudaStream_t>(s); }
void* cc_get_instance_stream(const cc_instance* I) { return I ? static_cast<void*>(I->stream) : nullptr; }
size_t cc_encode_get_required_memory(const cc_instance* I) { return I ? I->arenaBytes : 0; }

void cc_set_timing(cc_instance* I, int enable) {
    if (I) I->timing = enable != 0;
}

int cc_timing_count(cc_instance* I) {
    if (!I) return 0;
    I->resolveTimings();
    return int(I->timings.size());
}

int cc_timing_entry(cc_instance* I, uint32_t i, const char** name, double* ms, uint32_t* count) {
    if (!I || i >= I->timings.size()) { setError("cc_timing_entry: index out of range"); return CC_ERR_INVALID_ARGUMENT; }
    auto it = I->timings.begin();
    std::advance(it, i);
    if (name) *name = it->first.c_str();
    if (ms) *ms = it->second.first;
    if (count) *count = it->second.second;
    return CC_OK;
}

void cc_reset_timings(cc_instance* I) {
    if (!I) return;
    I->resolveTimings();
    I->timings.clear();
}

}  // extern "C"
