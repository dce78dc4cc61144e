// batch.cu - batched lossy volume codec: any number of float32 volumes
// ("bricks") of any sizes, each with its own quantization step, compressed
// and decompressed with one launch per stage for the whole batch.
//
// Each volume's bit stream is exactly cc_compress_volume_float's (the
// reference's compressVolumeFloat layout, CompressVolume.cpp:312-409: the
// lowpass band with encodeHuff, then per level coarse -> fine the 7 highpass
// bands with encodeRLHuff), so the batch is a drop-in for N calls of the
// plain codec.  Everything a call needs is planned once at creation and kept
// on the device: DWT / quantizer descriptors, the encoder's stream and table
// descriptors, the decoder's descriptors (its header walk runs on the
// device).  A compress or decompress call therefore enqueues only kernels,
// device memsets and one small upload of the volume pointer table, on the
// instance stream, with no host synchronization - and can run as a CUDA
// graph that replays the whole sequence in one launch.
//
// Work areas (one allocation): per level l a dense level-l volume for every
// brick (forward coefficients, and the reconstructions on the way back),
// two transform temporaries, the symbols (per brick: lowpass, then the 7
// bands of each level coarse -> fine, every band 16-byte aligned), the
// descriptors, the bricks' streams, and per brick the word offset and bit
// size of its stream there.
//
// Compress runs as two encodes: the lowpass streams (one Huffman stream per
// brick; its table is the largest of the brick, and its sequential tree
// build the longest single step) on a side stream with an instance of its
// own, concurrently with the highpass streams on the main stream.  After
// both, every brick's stream is assembled as [lowpass segment][highpass
// segments] - segments are whole words, so this is a word copy.
#include <algorithm>
#include <cstring>
#include <map>

#include "batch.cuh"

// Pinned pointer tables per batch (volume pointers of compress / decompress calls).
constexpr unsigned kTabRing = 8;

struct cc_volume_batch {
    cc_instance* I = nullptr;          // own instance, sized for the batch (highpass encode, decode)
    cc_instance* ILP = nullptr;        // own instance of the lowpass encode
    cudaStream_t sideStream = nullptr; // the lowpass encode's stream
    cudaEvent_t evFork = nullptr, evJoin = nullptr;
    ccb::u32* words = nullptr;         // device: the bricks' streams
    ccb::u64 wordsCap = 0;
    cc_instance* user = nullptr;
    ccb::u32 count = 0, levels = 0;
    std::vector<ccb::u32> nx, ny, nz;
    std::vector<float> q0;
    char* mem = nullptr;               // device
    size_t memBytes = 0;
    char* hostPlan = nullptr;          // pinned: a ring of kTabRing pointer tables
    ccb::u64* hostExt = nullptr;       // pinned: loaded streams' offsets and sizes
    cudaEvent_t extEvent = nullptr;
    cudaEvent_t tabEvent[kTabRing] = {};   // per ring slot: its last upload has read it
    unsigned tabNext = 0;
    // host copies of the descriptors that carry quantization steps (one per
    // volume and level, as uploaded), patched by batchSetQuantSteps
    std::vector<std::vector<ccb::BLevelDesc>> flHost;
    std::vector<std::vector<ccb::BColDesc>> izHost;
    std::vector<ccb::BQuantDesc> qdHost, dqHost;
    // device pieces
    ccb::u16* syms = nullptr;
    size_t symBytes = 0;
    const float** inTab = nullptr;
    float** outTab = nullptr;
    ccb::u64* wordOff = nullptr;
    ccb::u64* bitSize = nullptr;
    // launch lists
    // per volume v: descriptors and CTAs of volumes 0..v (prefix launches)
    struct Rows { const ccb::BRowDesc* d; const ccb::u32* map; ccb::u32 n, ctas; std::vector<ccb::u32> descEnd, ctaEnd; };
    struct Cols { const ccb::BColDesc* d; const ccb::u32* map; ccb::u32 n, ctas; std::vector<ccb::u32> descEnd, ctaEnd; };
    struct Quant { const ccb::BQuantDesc* d; const ccb::u32* map; ccb::u32 n, ctas; std::vector<ccb::u32> descEnd, ctaEnd; };
    struct Levels { const ccb::BLevelDesc* d; const ccb::u32* map; ccb::u32 n, ctas; std::vector<ccb::u32> descEnd, ctaEnd; };
    std::vector<Levels> fwdLevel;              // per level: the fused forward pass
    std::vector<Rows> fwdRows, invRows;        // per level
    std::vector<Cols> fwdY, fwdZ, invZ, invY;  // per level
    Quant quant{}, dequantLP{};
    ccb::EncPlan enc, encLP;           // highpass streams (I), lowpass streams (ILP)
    ccb::DecPlan dec;
    // per volume v: encoder / decoder counts of volumes 0..v
    std::vector<ccb::u32> encS, encT, encTiles, encBlocks;
    std::vector<ccb::u32> lpTiles, lpBlocks;
    std::vector<ccb::u32> decS;
    std::vector<ccb::u32> decT, decRl, decH, decRlBlocks, decHBlocks;
    std::vector<ccb::u64> symEnd;       // symbols of volumes 0..v
    ccb::u32 active = 0;                // volumes a call processes (the first `active`)
    cudaStream_t ownStream = nullptr;   // set: the batch's work goes here instead of the instance stream
    bool hasOwnStream = false;
    // graphs
    bool useGraph = false;
    std::map<ccb::u32, cudaGraphExec_t> gCompress, gDecompress;   // by active count
    cudaStream_t captureStream = nullptr;
    std::map<ccb::u32, unsigned> launchesCompress, launchesDecompress;
};

namespace ccb {

namespace {

struct Arena {
    size_t off = 0;
    size_t take(size_t bytes, size_t align = 256) {
        off = alignUp(off, align);
        const size_t at = off;
        off += bytes;
        return at;
    }
};

u64 vol3(u32 x, u32 y, u32 z) { return u64(x) * y * z; }

void addRows(std::vector<BRowDesc>& v, u32& ctas, BRowDesc d) {
    batchRowTiling(d.nx, d.W, d.R);
    d.tilesX = int(ceilDiv(d.nx, d.W));
    d.vec = (d.nx % 8 == 0 && d.W % 8 == 0 && d.srcRow % 4 == 0 && d.srcSlice % 4 == 0 && d.dstRow % 4 == 0 &&
             d.dstSlice % 4 == 0) ? 1 : 0;
    d.ctaOff = ctas;
    ctas += u32(d.tilesX) * u32(ceilDiv(u64(d.ny) * d.nz, d.R));
    v.push_back(d);
}

void addCols(std::vector<BColDesc>& v, u32& ctas, BColDesc d) {
    d.tilesX = u32(ceilDiv(d.nx, kBColTileX));
    d.tilesA = u32(ceilDiv(d.na, kBColTileA));
    d.ctaOff = ctas;
    ctas += d.tilesX * d.tilesA * u32(d.nc);
    v.push_back(d);
}

void addLevel(std::vector<BLevelDesc>& v, u32& ctas, BLevelDesc d) {
    d.tilesX = int(ceilDiv(d.nx, kLvTX));
    d.tilesY = int(ceilDiv(d.ny, kLvTY));
    d.chunksZ = int(ceilDiv(d.nz, u64(d.zChunk)));
    d.ctaOff = ctas;
    ctas += u32(d.tilesX) * u32(d.tilesY) * u32(d.chunksZ);
    v.push_back(d);
}

// CTA -> descriptor index of one launch (descriptors are in CTA order)
template <class Desc>
std::vector<u32> ctaMapOf(const std::vector<Desc>& v, u32 ctas) {
    std::vector<u32> m(ctas);
    for (size_t i = 0; i < v.size(); ++i) {
        const u32 end = i + 1 < v.size() ? v[i + 1].ctaOff : ctas;
        std::fill(m.begin() + v[i].ctaOff, m.begin() + end, u32(i));
    }
    return m;
}

void addQuant(std::vector<BQuantDesc>& v, u32& ctas, BQuantDesc d) {
    d.ctaOff = ctas;
    ctas += u32(ceilDiv(vol3(d.nx, d.ny, d.nz), kBQuantPerCta));
    v.push_back(d);
}

// Symbol layout of one volume: lowpass, then levels L-1 .. 0, 7 bands each.
struct SymLayout {
    u64 lp = 0;                 // offset of the lowpass (symbols)
    std::vector<u64> level;     // offset of the first band of level l
    std::vector<u64> bandStride;
    u64 total = 0;
};

SymLayout symLayout(u32 nx, u32 ny, u32 nz, u32 L) {
    SymLayout s;
    s.level.assign(L, 0);
    s.bandStride.assign(L, 0);
    u64 at = 0;
    s.lp = at;
    at = alignUp(at + vol3(nx >> L, ny >> L, nz >> L), 8);
    for (int l = int(L) - 1; l >= 0; --l) {
        const u64 band = alignUp(vol3(nx >> (l + 1), ny >> (l + 1), nz >> (l + 1)), 8);
        s.level[l] = at;
        s.bandStride[l] = band;
        at += 7 * band;
    }
    s.total = at;
    return s;
}

}  // namespace

// Per brick: words of its lowpass segment plus its highpass segments, and
// the exclusive scan of those totals (its offset in the stream words).
__global__ void __launch_bounds__(1024) k_brickOffsets(const SegmentLayout* lp, const SegmentLayout* hp, u32 hpPer,
                                                       u32 count, u64* wordOff, u64* bitSize, const u32* errLP,
                                                       const u32* errHP) {
    __shared__ u32 scratch[40];
    __shared__ unsigned long long carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const bool failed = *errLP != 0 || *errHP != 0;
    for (u32 base = 0; base < count; base += 1024) {
        const u32 v = base + threadIdx.x;
        u32 words = 0;
        if (v < count && !failed) {
            const SegmentLayout& f = hp[u64(v) * hpPer];
            const SegmentLayout& l = hp[u64(v) * hpPer + hpPer - 1];
            words = lp[v].words + u32(l.startWord + l.words - f.startWord);
        }
        u32 tot;
        const u32 ex = blockExclusiveSum<1024>(words, scratch, &tot);
        if (v < count) {
            wordOff[v] = carry + ex;
            bitSize[v] = u64(words) * 32ull;
        }
        __syncthreads();
        if (threadIdx.x == 0) carry += tot;
        __syncthreads();
    }
}

// Brick v's stream: its lowpass words, then its highpass words; `parts` CTAs
// per brick.
__global__ void __launch_bounds__(256) k_brickConcat(const u32* lpOut, const u32* hpOut, const SegmentLayout* lp,
                                                     const SegmentLayout* hp, u32 hpPer, u32 parts, const u64* wordOff,
                                                     const u64* bitSize, u32* dst) {
    const u32 v = blockIdx.x / parts, part = blockIdx.x - v * parts;
    const u64 total = bitSize[v] / 32u;
    if (total == 0) return;
    const u64 lpW = lp[v].words, lpS = lp[v].startWord, hpS = hp[u64(v) * hpPer].startWord;
    const u64 chunk = (total + parts - 1) / parts;
    const u64 w0 = u64(part) * chunk, w1 = min(total, w0 + chunk);
    u32* out = dst + wordOff[v];
    for (u64 w = w0 + threadIdx.x; w < w1; w += blockDim.x) out[w] = w < lpW ? lpOut[lpS + w] : hpOut[hpS + (w - lpW)];
}

// Streams of the first n volumes between the batch's word buffer (HBM) and
// page-locked host memory, moved by kernels so that nothing waits on the
// host: the used extent (the streams lie back to back, the last one ending at
// wordOff[n-1] + its words) is known on the device only.  hExt holds the n
// word offsets, then the n bit sizes.  16-byte copies when both sides allow.
template <bool kVec>
__global__ void __launch_bounds__(256) k_streamsToHost(const u32* __restrict__ words, const u64* __restrict__ wordOff,
                                                       const u64* __restrict__ bitSize, u32 n, u32* hWords, u64 cap,
                                                       u64* hExt, u32* err) {
    const u64 total = wordOff[n - 1] + (bitSize[n - 1] + 31) / 32;
    const u64 tid = u64(blockIdx.x) * blockDim.x + threadIdx.x, nth = u64(gridDim.x) * blockDim.x;
    if (tid < n) {
        hExt[tid] = wordOff[tid];
        hExt[n + tid] = bitSize[tid];
    }
    if (total > cap) {
        if (tid == 0) atomicOr(err, u32(DEV_ERR_OUTPUT_CAPACITY));
        return;
    }
    u64 done = 0;
    if (kVec) {
        const u64 q = total / 4;
        for (u64 i = tid; i < q; i += nth) reinterpret_cast<uint4*>(hWords)[i] = reinterpret_cast<const uint4*>(words)[i];
        done = q * 4;
    }
    for (u64 i = done + tid; i < total; i += nth) hWords[i] = words[i];
}

template <bool kVec>
__global__ void __launch_bounds__(256) k_streamsFromHost(const u32* hWords, const u64* hExt, u32 n, u32* words,
                                                         u64* wordOff, u64* bitSize, u64 cap, u32* err) {
    __shared__ u64 sTotal;
    if (threadIdx.x == 0) sTotal = hExt[n - 1] + (hExt[2 * n - 1] + 31) / 32;   // one host read per CTA
    __syncthreads();
    const u64 total = sTotal;
    const u64 tid = u64(blockIdx.x) * blockDim.x + threadIdx.x, nth = u64(gridDim.x) * blockDim.x;
    if (total > cap) {
        if (tid == 0) atomicOr(err, u32(DEV_ERR_CORRUPT));
        return;
    }
    if (tid < n) {
        wordOff[tid] = hExt[tid];
        bitSize[tid] = hExt[n + tid];
    }
    u64 done = 0;
    if (kVec) {
        const u64 q = total / 4;
        for (u64 i = tid; i < q; i += nth) reinterpret_cast<uint4*>(words)[i] = reinterpret_cast<const uint4*>(hWords)[i];
        done = q * 4;
    }
    for (u64 i = done + tid; i < total; i += nth) words[i] = hWords[i];
}

template <class List>
static void prefixOf(const List& li, u32 k, u32& nd, u32& ctas) {
    nd = li.descEnd[k - 1];
    ctas = li.ctaEnd[k - 1];
}

static int batchEnqueueCompress(cc_volume_batch* b) {
    cc_instance* I = b->I;
    cudaStream_t st = I->stream;
    const u32 k = b->active;
    u32 nd, ctas;
    for (u32 l = 0; l < b->levels; ++l) {
        // one fused pass per level: X, Y, Z filters and the deadzone quantization
        SectionTimer t(I, "batch.dwt_forward", st);
        prefixOf(b->fwdLevel[l], k, nd, ctas);
        launchBatchLevelFwd(b->fwdLevel[l].d, b->fwdLevel[l].map, ctas, b->inTab, st);
    }
    // fork: the lowpass streams on the side stream
    cc_instance* ILP = b->ILP;
    ILP->stream = b->sideStream;
    CC_TRY_CUDA(cudaEventRecord(b->evFork, st), "fork");
    CC_TRY_CUDA(cudaStreamWaitEvent(b->sideStream, b->evFork, 0), "fork");
    EncPlan lp = b->encLP;
    lp.S = k;
    lp.T = k;
    lp.tiles = b->lpTiles[k - 1];
    lp.blocks = b->lpBlocks[k - 1];
    int rc;
    {
        SectionTimer t(I, "batch.lowpass_encode", b->sideStream);
        rc = encodeLaunch(ILP, lp, ILP->out, ILP->outWordsMax);
    }
    if (rc) return rc;
    CC_TRY_CUDA(cudaEventRecord(b->evJoin, b->sideStream), "join");
    // the highpass streams here
    EncPlan ep = b->enc;
    ep.S = b->encS[k - 1];
    ep.T = b->encT[k - 1];
    ep.tiles = b->encTiles[k - 1];
    ep.blocks = b->encBlocks[k - 1];
    rc = encodeLaunch(I, ep, I->out, I->outWordsMax);
    if (rc) return rc;
    CC_TRY_CUDA(cudaStreamWaitEvent(st, b->evJoin, 0), "join");
    {
        SectionTimer t(I, "batch.assemble", st);
        const u32 hpPer = 7 * b->levels;
        k_brickOffsets<<<1, 1024, 0, st>>>(ILP->layout, I->layout, hpPer, k, b->wordOff, b->bitSize, ILP->errors,
                                           I->errors);
        const u32 sms = u32(std::max(1, I->smCount > 0 ? I->smCount : 148));
        const u32 parts = std::max<u32>(1, std::min<u32>(1024, u32(ceilDiv(16 * sms, k))));
        k_brickConcat<<<k * parts, 256, 0, st>>>(ILP->out, I->out, ILP->layout, I->layout, hpPer, parts, b->wordOff,
                                                 b->bitSize, b->words);
        countLaunch(2);
    }
    CC_TRY_CUDA(cudaGetLastError(), "batch compress");
    return CC_OK;
}

static int batchEnqueueDecompress(cc_volume_batch* b) {
    cc_instance* I = b->I;
    cudaStream_t st = I->stream;
    const u32 k = b->active;
    u32 nd, ctas;
    // no zeroing of the symbols: the decoder writes every element of every band
    DecPlan dp = b->dec;
    dp.S = b->decS[k - 1];
    dp.T = b->decT[k - 1];
    dp.B = k;
    dp.nRl = b->decRl[k - 1];
    dp.nH = b->decH[k - 1];
    dp.rlBlocks = b->decRlBlocks[k - 1];
    dp.hBlocks = b->decHBlocks[k - 1];
    int rc = decodeLaunch(I, dp);
    if (rc) return rc;
    prefixOf(b->dequantLP, k, nd, ctas);
    { SectionTimer t(I, "batch.dequantize", st); launchBatchQuant(b->dequantLP.d, b->dequantLP.map, ctas, true, st); }
    for (int l = int(b->levels) - 1; l >= 0; --l) {
        SectionTimer t(I, "batch.dwt_inverse", st);
        prefixOf(b->invZ[l], k, nd, ctas);
        launchBatchCols(b->invZ[l].d, b->invZ[l].map, ctas, true, true, st);
        prefixOf(b->invY[l], k, nd, ctas);
        launchBatchCols(b->invY[l].d, b->invY[l].map, ctas, true, false, st);
        prefixOf(b->invRows[l], k, nd, ctas);
        launchBatchRows(b->invRows[l].d, b->invRows[l].map, ctas, true, b->inTab, b->outTab, st);
    }
    CC_TRY_CUDA(cudaGetLastError(), "batch decompress");
    return CC_OK;
}

// Copies a volume pointer table to the device (outside any captured graph)
// through the next slot of a ring of pinned tables: the host waits only for
// the upload kTabRing calls back, so it can enqueue several steps ahead of the
// device instead of one call.
static int uploadTable(cc_volume_batch* b, const void* const* ptrs, void* dTable) {
    const unsigned r = b->tabNext++ % kTabRing;
    cudaEventSynchronize(b->tabEvent[r]);   // the slot's last upload has read it
    void** slot = reinterpret_cast<void**>(b->hostPlan) + size_t(r) * b->count;
    std::memcpy(slot, ptrs, sizeof(void*) * b->active);
    CC_TRY_CUDA(cudaMemcpyAsync(dTable, slot, sizeof(void*) * b->active, cudaMemcpyHostToDevice, b->I->stream),
                "upload volume pointers");
    cudaEventRecord(b->tabEvent[r], b->I->stream);
    return CC_OK;
}

using Enqueue = int (*)(cc_volume_batch*);

// Runs an enqueue function directly, or through its CUDA graph (captured on
// the first use; later calls replay it).
static int runMaybeGraph(cc_volume_batch* b, Enqueue fn, std::map<u32, cudaGraphExec_t>& graphs,
                         std::map<u32, unsigned>& counts) {
    cc_instance* I = b->I;
    if (!b->useGraph) return fn(b);
    cudaGraphExec_t& exec = graphs[b->active];
    unsigned& launches = counts[b->active];
    if (!exec) {
        // Capture on the batch's own stream (the instance stream may be the
        // legacy default stream, which cannot be captured); the graph is then
        // launched on the instance stream.
        if (!b->captureStream)
            CC_TRY_CUDA(cudaStreamCreateWithFlags(&b->captureStream, cudaStreamNonBlocking), "capture stream");
        const bool timing = I->timing, timingLP = b->ILP->timing;
        cudaStream_t userStream = I->stream;
        I->timing = false;   // no event records inside the graph
        b->ILP->timing = false;
        I->stream = b->captureStream;
        cudaError_t e = cudaStreamBeginCapture(I->stream, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) {
            I->stream = userStream;
            I->timing = timing;
            b->ILP->timing = timingLP;
            return cudaFail(e, "begin capture");
        }
        const unsigned long long c0 = cc_kernel_launches();
        int rc = fn(b);
        cudaGraph_t g = nullptr;
        e = cudaStreamEndCapture(I->stream, &g);
        I->stream = userStream;
        I->timing = timing;
        b->ILP->timing = timingLP;
        if (rc) { if (g) cudaGraphDestroy(g); return rc; }
        if (e != cudaSuccess) return cudaFail(e, "end capture");
        launches = unsigned(cc_kernel_launches() - c0);
        e = cudaGraphInstantiate(&exec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) { exec = nullptr; return cudaFail(e, "graph instantiate"); }
    }
    CC_TRY_CUDA(cudaGraphLaunch(exec, I->stream), "graph launch");
    countLaunch(launches);
    return CC_OK;
}

// New quantization steps for the batch's volumes: the descriptors that carry
// them (forward levels, LP quantizer, inverse Z passes, LP dequantizer) are
// recomputed as at creation and re-uploaded, stream-ordered on the batch's
// stream, so calls enqueued before keep their steps.
int batchSetQuantSteps(cc_volume_batch* b, const float* q) {
    if (!b || !q) { setError("volume batch quantization steps: null argument"); return CC_ERR_INVALID_ARGUMENT; }
    bool same = true;
    for (u32 v = 0; v < b->count; ++v) {
        if (!(q[v] > 0.0f)) { setError("volume batch: volume %u: quantization step must be > 0", v); return CC_ERR_INVALID_ARGUMENT; }
        same = same && q[v] == b->q0[v];
    }
    if (same) return CC_OK;
    const u32 L = b->levels;
    for (u32 v = 0; v < b->count; ++v) {
        const float q0 = q[v];
        b->q0[v] = q0;
        for (u32 l = 0; l < L; ++l) {
            b->flHost[l][v].inv = 1.0f / (q0 / float(1u << l));              // Quantize.cu:90: reciprocal on the host
            b->flHost[l][v].invLP = 1.0f / (q0 / float(1u << (L - 1)));
            b->izHost[l][v].step = q0 / float(1u << l);
        }
        BQuantDesc* qv = &b->qdHost[size_t(v) * (1 + 7 * L)];
        qv[0].step = q0 / float(1u << (L - 1));
        qv[0].inv = 1.0f / qv[0].step;
        b->dqHost[v].step = qv[0].step;
        b->dqHost[v].inv = qv[0].inv;
        u32 k = 1;
        for (int l = int(L) - 1; l >= 0; --l)
            for (u32 bi = 1; bi < 8; ++bi, ++k) {
                qv[k].step = q0 / float(1u << l);
                qv[k].inv = 1.0f / qv[k].step;
            }
    }
    cudaStream_t st = b->hasOwnStream ? b->ownStream : b->user->stream;
    auto up = [&](const void* dst, const void* src, size_t bytes) {
        return cudaMemcpyAsync(const_cast<void*>(dst), src, bytes, cudaMemcpyHostToDevice, st);
    };
    for (u32 l = 0; l < L; ++l) {
        CC_TRY_CUDA(up(b->fwdLevel[l].d, b->flHost[l].data(), b->flHost[l].size() * sizeof(BLevelDesc)), "patch steps");
        CC_TRY_CUDA(up(b->invZ[l].d, b->izHost[l].data(), b->izHost[l].size() * sizeof(BColDesc)), "patch steps");
    }
    CC_TRY_CUDA(up(b->quant.d, b->qdHost.data(), b->qdHost.size() * sizeof(BQuantDesc)), "patch steps");
    CC_TRY_CUDA(up(b->dequantLP.d, b->dqHost.data(), b->dqHost.size() * sizeof(BQuantDesc)), "patch steps");
    return CC_OK;
}

// Error flags of one direction only: the encoders' (highpass and lowpass
// instances) or the decoder's, each reset by its own launches, so a failed
// call of one direction does not surface on the next call of the other.
int batchStatusOf(cc_volume_batch* b, bool decode) {
    if (!b) return CC_ERR_INVALID_ARGUMENT;
    u32 flags[8] = {}, lp = 0;
    CC_TRY_CUDA(cudaMemcpyAsync(flags, b->I->errors, sizeof(flags), cudaMemcpyDeviceToHost, b->I->stream), "batch status");
    CC_TRY_CUDA(cudaMemcpyAsync(&lp, b->ILP->errors, sizeof(lp), cudaMemcpyDeviceToHost, b->I->stream), "batch status");
    CC_TRY_CUDA(cudaStreamSynchronize(b->I->stream), "batch status");
    if (decode) return deviceErrorStatus(flags[4], "batch decompress");
    if (lp) return deviceErrorStatus(lp, "batch compress (lowpass streams)");
    return deviceErrorStatus(flags[0], "batch compress");
}

}  // namespace ccb

using namespace ccb;

extern "C" {

int cc_volume_batch_create(cc_instance* user, uint32_t count, const uint32_t* sizes, uint32_t levels,
                           const float* quantSteps, cc_volume_batch** out) {
    return cc_volume_batch_create_ex(user, count, sizes, levels, quantSteps, 0, out);
}

int cc_volume_batch_create_ex(cc_instance* user, uint32_t count, const uint32_t* sizes, uint32_t levels,
                              const float* quantSteps, uint32_t zChunk, cc_volume_batch** out) {
    if (!out) { setError("cc_volume_batch_create: out is NULL"); return CC_ERR_INVALID_ARGUMENT; }
    if (zChunk == 0) zChunk = kLvZCDefault;
    if (zChunk < 8 || zChunk > 256 || (zChunk & 1)) {
        setError("cc_volume_batch_create_ex: z_chunk must be 0 (default) or even in 8..256 (got %u)", zChunk);
        *out = nullptr;
        return CC_ERR_INVALID_ARGUMENT;
    }
    *out = nullptr;
    if (!user || !sizes || !quantSteps || count == 0 || levels == 0 || levels > 8) {
        setError("cc_volume_batch_create: bad argument");
        return CC_ERR_INVALID_ARGUMENT;
    }
    if (user->symBytes != 2) { setError("cc_volume_batch_create: needs a 16-bit-symbol instance (log2 symbol count <= 16)"); return CC_ERR_INVALID_ARGUMENT; }
    const u32 L = levels, f = 1u << L;
    u64 N0sum = 0, histBins = 0, LPsum = 0;
    u32 maxStream = 1, maxLP = 1;
    for (u32 v = 0; v < count; ++v) {
        const u32 x = sizes[3 * v], y = sizes[3 * v + 1], z = sizes[3 * v + 2];
        if (x % f || y % f || z % f || (x >> (L - 1)) < 8 || (y >> (L - 1)) < 8 || (z >> (L - 1)) < 8) {
            setError("cc_volume_batch_create: volume %u (%u x %u x %u): sizes must be divisible by 2^levels with the coarsest level >= 8",
                     v, x, y, z);
            return CC_ERR_INVALID_ARGUMENT;
        }
        if (!(quantSteps[v] > 0.0f)) { setError("cc_volume_batch_create: volume %u: quantization step must be > 0", v); return CC_ERR_INVALID_ARGUMENT; }
        if (vol3(x, y, z) >= (u64(1) << 31)) {
            setError("cc_volume_batch_create: volume %u (%u x %u x %u): at most 2^31 - 1 elements per volume", v, x, y, z);
            return CC_ERR_INVALID_ARGUMENT;
        }
        N0sum += vol3(x, y, z);
        LPsum += vol3(x >> L, y >> L, z >> L);
        maxStream = std::max<u32>(maxStream, u32(vol3(x >> 1, y >> 1, z >> 1)));
        maxLP = std::max<u32>(maxLP, u32(vol3(x >> L, y >> L, z >> L)));
    }
    const u32 S = count * (1 + 7 * L);
    // histogram bins: every table at most 2^log2Max; budget 2^26 bins (the
    // device plan fails a call that needs more)
    histBins = std::min<u64>(u64(2 * S) * user->bins, u64(1) << 26);
    DeviceGuard deviceGuard(user->device);
    cc_volume_batch* b = new cc_volume_batch();
    b->user = user;
    b->count = count;
    b->levels = L;
    for (u32 v = 0; v < count; ++v) {
        b->nx.push_back(sizes[3 * v]);
        b->ny.push_back(sizes[3 * v + 1]);
        b->nz.push_back(sizes[3 * v + 2]);
        b->q0.push_back(quantSteps[v]);
    }
    // symbols: every stream's (the lowpass streams' coding blocks count too)
    InstanceCaps caps{S, std::max<u64>(N0sum, 1), histBins};
    int rc = createInstance(&b->I, user->device, S, maxStream, user->codingBlockSize, user->log2Max, &caps);
    if (rc) { delete b; return rc; }
    cc_instance* I = b->I;
    I->stream = user->stream;
    I->timing = user->timing;
    // the lowpass encode's instance: one stream, one table per brick
    InstanceCaps capsLP{count, std::max<u64>(LPsum, 1), std::min<u64>(u64(2 * count) * user->bins, u64(1) << 26)};
    rc = createInstance(&b->ILP, user->device, count, maxLP, user->codingBlockSize, user->log2Max, &capsLP);
    if (rc) { cc_volume_batch_destroy(b); return rc; }
    b->ILP->timing = false;   // follows the user instance's timing on each compress call
    // the lowpass tables are built while the highpass encode runs: one SM each
    b->ILP->tableBuildSoloSM = true;
    cudaDeviceGetAttribute(&b->ILP->smCount, cudaDevAttrMultiProcessorCount, user->device);
    // kernel attributes set once here, so that captured launches do not set them
    rc = prepareKernelAttributes(I);
    if (!rc) rc = prepareKernelAttributes(b->ILP);
    if (rc) { cc_volume_batch_destroy(b); return rc; }
    cudaError_t ce = cudaStreamCreateWithFlags(&b->sideStream, cudaStreamNonBlocking);
    if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&b->evFork, cudaEventDisableTiming);
    if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&b->evJoin, cudaEventDisableTiming);
    if (ce != cudaSuccess) { cc_volume_batch_destroy(b); return cudaFail(ce, "volume batch streams"); }
    b->wordsCap = I->outWordsMax + b->ILP->outWordsMax;

    // ---- layout of the work areas ----
    // Descriptors hold offsets until the allocation exists, and a null
    // pointer means "the volume pointer table": no piece may start at 0.
    Arena A;
    A.take(256);
    std::vector<std::vector<u64>> levOff(L + 1, std::vector<u64>(count));
    std::vector<size_t> levAt(L + 1);
    for (u32 l = 0; l <= L; ++l) {
        u64 tot = 0;
        for (u32 v = 0; v < count; ++v) {
            levOff[l][v] = tot;
            tot += alignUp(vol3(b->nx[v] >> l, b->ny[v] >> l, b->nz[v] >> l), 64);
        }
        levAt[l] = A.take(tot * sizeof(float));
    }
    std::vector<u64> tOff(count);
    u64 tTot = 0;
    for (u32 v = 0; v < count; ++v) { tOff[v] = tTot; tTot += alignUp(vol3(b->nx[v], b->ny[v], b->nz[v]), 64); }
    const size_t t1At = A.take(tTot * sizeof(float)), t2At = A.take(tTot * sizeof(float));
    std::vector<SymLayout> sl(count);
    std::vector<u64> symOff(count);
    u64 symTot = 0;
    for (u32 v = 0; v < count; ++v) {
        sl[v] = symLayout(b->nx[v], b->ny[v], b->nz[v], L);
        symOff[v] = symTot;
        symTot += sl[v].total;
    }
    const size_t symAt = A.take((symTot + 64) * sizeof(u16));
    const size_t inTabAt = A.take(sizeof(void*) * count), outTabAt = A.take(sizeof(void*) * count);
    const size_t wordOffAt = A.take(sizeof(u64) * count), bitSizeAt = A.take(sizeof(u64) * count);
    const size_t wordsAt = A.take(b->wordsCap * sizeof(u32));

    // ---- descriptors (host) ----
    auto lev = [&](u32 l, u32 v) { return reinterpret_cast<float*>(levAt[l]) + levOff[l][v]; };   // offsets, rebased below
    auto t1 = [&](u32 v) { return reinterpret_cast<float*>(t1At) + tOff[v]; };
    auto t2 = [&](u32 v) { return reinterpret_cast<float*>(t2At) + tOff[v]; };
    auto sy = [&](u32 v) { return reinterpret_cast<u16*>(symAt) + symOff[v]; };
    std::vector<std::vector<BLevelDesc>> fl(L);
    std::vector<u32> flC(L, 0);
    std::vector<std::vector<BRowDesc>> fr(L), ir(L);
    std::vector<std::vector<BColDesc>> fy(L), fz(L), iz(L), iy(L);
    std::vector<u32> frC(L, 0), irC(L, 0), fyC(L, 0), fzC(L, 0), izC(L, 0), iyC(L, 0);
    std::vector<BQuantDesc> qd, dq;
    u32 qC = 0, dqC = 0;
    std::vector<EncStream> es;
    std::vector<DecStreamSpec> ds;
    std::vector<DecSourceSpec> dsrc(count);
    std::vector<u32> firstStream(count + 1);
    for (u32 v = 0; v < count; ++v) {
        const u32 X = b->nx[v], Y = b->ny[v], Z = b->nz[v];
        for (u32 l = 0; l < L; ++l) {
            const int sx = int(X >> l), syz = int(Y >> l), sz = int(Z >> l);
            // the fused forward level: input (level 0: the caller's volume;
            // else the LLL octant of level l-1, tight in lev(l-1)) -> the
            // highpass symbols and the LLL octant, tight in lev(l) (or the
            // lowpass band's symbols at the coarsest level)
            BLevelDesc fd{};
            fd.vol = int(v);
            fd.src = l == 0 ? nullptr : lev(l - 1, v);
            fd.nx = sx; fd.ny = syz; fd.nz = sz;
            fd.srcRow = sx;
            fd.srcSlice = sx * syz;
            fd.lpOut = lev(l, v);
            fd.symOut = sy(v) + sl[v].level[l];
            fd.lpSymOut = sy(v) + sl[v].lp;
            fd.bandStride = sl[v].bandStride[l];
            fd.inv = 1.0f / (b->q0[v] / float(1u << l));              // Quantize.cu:90: reciprocal on the host
            fd.invLP = 1.0f / (b->q0[v] / float(1u << (L - 1)));
            fd.lastLevel = l + 1 == L ? 1 : 0;
            fd.zChunk = int(zChunk);
            addLevel(fl[l], flC[l], fd);
            // X: input (level 0: the caller's volume, tight; else the LLL octant of level l-1) -> t1
            BRowDesc r{};
            r.vol = int(v);
            r.src = l == 0 ? nullptr : lev(l - 1, v);
            r.dst = t1(v);
            r.nx = sx; r.ny = syz; r.nz = sz;
            r.srcRow = l == 0 ? int(X) : int(X >> (l - 1));
            r.srcSlice = l == 0 ? int(X * Y) : int((X >> (l - 1)) * (Y >> (l - 1)));
            r.dstRow = sx; r.dstSlice = sx * syz;
            addRows(fr[l], frC[l], r);
            // Y: t1 -> t2 (dense level l)
            BColDesc c{};
            c.src = t1(v); c.dst = t2(v);
            c.nx = sx; c.na = syz; c.nc = sz;
            c.sa = sx; c.sc = sx * syz;
            c.da = sx; c.dc = sx * syz;
            addCols(fy[l], fyC[l], c);
            // Z: t2 -> level l coefficients, quantized in the store: the LLL
            // octant stays float (next level's input) except at the coarsest
            // level, where it is the lowpass band
            BColDesc cz = c;
            cz.src = t2(v); cz.dst = lev(l, v);
            cz.na = sz; cz.nc = syz;
            cz.sa = sx * syz; cz.sc = sx;
            cz.da = sx * syz; cz.dc = sx;
            cz.symOut = sy(v) + sl[v].level[l];
            cz.lpSymOut = sy(v) + sl[v].lp;
            cz.bandStride = sl[v].bandStride[l];
            cz.hx = sx / 2; cz.hy = syz / 2; cz.hz = sz / 2;
            cz.inv = 1.0f / (b->q0[v] / float(1u << l));              // Quantize.cu:90: reciprocal on the host
            cz.invLP = 1.0f / (b->q0[v] / float(1u << (L - 1)));
            cz.lastLevel = l + 1 == L ? 1 : 0;
            addCols(fz[l], fzC[l], cz);
            // inverse of level l: Z from symbols (lowpass = level l+1 reconstruction) -> t2, Y -> t1, X -> level l
            BColDesc ic{};
            ic.src = lev(l + 1, v);
            ic.dst = t2(v);
            ic.nx = sx; ic.na = sz; ic.nc = syz;
            ic.da = sx * syz; ic.dc = sx;
            ic.bands = sy(v) + sl[v].level[l];
            ic.bandStride = sl[v].bandStride[l];
            ic.step = b->q0[v] / float(1u << l);
            ic.hx = sx / 2; ic.hy = syz / 2; ic.hz = sz / 2;
            ic.lpRow = sx / 2; ic.lpSlice = (sx / 2) * (syz / 2);
            addCols(iz[l], izC[l], ic);
            BColDesc iyd{};
            iyd.src = t2(v); iyd.dst = t1(v);
            iyd.nx = sx; iyd.na = syz; iyd.nc = sz;
            iyd.sa = sx; iyd.sc = sx * syz;
            iyd.da = sx; iyd.dc = sx * syz;
            addCols(iy[l], iyC[l], iyd);
            BRowDesc irw{};
            irw.vol = int(v);
            irw.src = t1(v);
            irw.dst = l == 0 ? nullptr : lev(l, v);
            irw.nx = sx; irw.ny = syz; irw.nz = sz;
            irw.srcRow = sx; irw.srcSlice = sx * syz;
            irw.dstRow = sx; irw.dstSlice = sx * syz;
            addRows(ir[l], irC[l], irw);
        }
        // quantization: lowpass (step q0 / 2^(L-1)), then levels coarse -> fine (step q0 / 2^l)
        const u32 Lx = X >> (L - 1), Ly = Y >> (L - 1);
        BQuantDesc q{};
        q.src = lev(L - 1, v);
        q.sym = sy(v) + sl[v].lp;
        q.nx = int(X >> L); q.ny = int(Y >> L); q.nz = int(Z >> L);
        q.row = int(Lx); q.slice = int(Lx * Ly);
        q.step = b->q0[v] / float(1u << (L - 1));
        q.inv = 1.0f / q.step;   // Quantize.cu:90: reciprocal computed on the host
        addQuant(qd, qC, q);
        BQuantDesc d = q;
        d.src = nullptr;
        d.dstF = lev(L, v);
        addQuant(dq, dqC, d);
        firstStream[v] = u32(es.size());
        es.push_back(EncStream{reinterpret_cast<void*>(q.sym), u32(vol3(X >> L, Y >> L, Z >> L)), 0, 0, 1, KIND_HUFF});
        ds.push_back(DecStreamSpec{KIND_HUFF, u32(vol3(X >> L, Y >> L, Z >> L)), q.sym, v});
        for (int l = int(L) - 1; l >= 0; --l) {
            const u32 sx = X >> l, syv = Y >> l, sz = Z >> l;
            const u32 hx = sx / 2, hy = syv / 2, hz = sz / 2;
            const u32 first = u32(es.size());
            for (u32 bi = 1; bi < 8; ++bi) {
                const u32 x = bi % 2, y = (bi / 2) % 2, z = bi / 4;
                BQuantDesc qb{};
                qb.src = lev(u32(l), v) + u64(z) * hz * sx * syv + u64(y) * hy * sx + u64(x) * hx;
                qb.sym = sy(v) + sl[v].level[l] + (bi - 1) * sl[v].bandStride[l];
                qb.nx = int(hx); qb.ny = int(hy); qb.nz = int(hz);
                qb.row = int(sx); qb.slice = int(sx * syv);
                qb.step = b->q0[v] / float(1u << l);
                qb.inv = 1.0f / qb.step;
                addQuant(qd, qC, qb);
                es.push_back(EncStream{reinterpret_cast<void*>(qb.sym), hx * hy * hz, 0, first, 7, KIND_RLHUFF});
                ds.push_back(DecStreamSpec{KIND_RLHUFF, hx * hy * hz, qb.sym, v});
            }
        }
        dsrc[v] = DecSourceSpec{nullptr, 0, 0};
    }
    firstStream[count] = u32(es.size());

    // ---- device plan ----
    auto bytesOf = [](size_t n, size_t e) { return n * e; };
    std::vector<size_t> flAt(L), frAt(L), irAt(L), fyAt(L), fzAt(L), izAt(L), iyAt(L);
    A.off = alignUp(A.off, 256);
    for (u32 l = 0; l < L; ++l) {
        flAt[l] = A.take(bytesOf(fl[l].size(), sizeof(BLevelDesc)), 64);
        frAt[l] = A.take(bytesOf(fr[l].size(), sizeof(BRowDesc)), 64);
        irAt[l] = A.take(bytesOf(ir[l].size(), sizeof(BRowDesc)), 64);
        fyAt[l] = A.take(bytesOf(fy[l].size(), sizeof(BColDesc)), 64);
        fzAt[l] = A.take(bytesOf(fz[l].size(), sizeof(BColDesc)), 64);
        izAt[l] = A.take(bytesOf(iz[l].size(), sizeof(BColDesc)), 64);
        iyAt[l] = A.take(bytesOf(iy[l].size(), sizeof(BColDesc)), 64);
    }
    const size_t qAt = A.take(bytesOf(qd.size(), sizeof(BQuantDesc)), 64);
    const size_t dqAt = A.take(bytesOf(dq.size(), sizeof(BQuantDesc)), 64);
    // CTA maps, one per launch
    std::vector<std::vector<u32>> maps;
    std::vector<size_t> mapAt;
    auto addMap = [&](std::vector<u32> m) {
        mapAt.push_back(A.take(bytesOf(m.size(), sizeof(u32)), 64));
        maps.push_back(std::move(m));
        return maps.size() - 1;
    };
    std::vector<size_t> flMap(L), frMap(L), irMap(L), fyMap(L), fzMap(L), izMap(L), iyMap(L);
    for (u32 l = 0; l < L; ++l) {
        flMap[l] = addMap(ctaMapOf(fl[l], flC[l]));
        frMap[l] = addMap(ctaMapOf(fr[l], frC[l]));
        irMap[l] = addMap(ctaMapOf(ir[l], irC[l]));
        fyMap[l] = addMap(ctaMapOf(fy[l], fyC[l]));
        fzMap[l] = addMap(ctaMapOf(fz[l], fzC[l]));
        izMap[l] = addMap(ctaMapOf(iz[l], izC[l]));
        iyMap[l] = addMap(ctaMapOf(iy[l], iyC[l]));
    }
    const size_t qMap = addMap(ctaMapOf(qd, qC)), dqMap = addMap(ctaMapOf(dq, dqC));
    // the encodes' streams: the lowpass streams, and the highpass streams with
    // their group indices rebased to the highpass list
    std::vector<EncStream> esLP, esHP;
    for (u32 v = 0; v < count; ++v) {
        esLP.push_back(es[firstStream[v]]);
        for (u32 t = firstStream[v] + 1; t < firstStream[v + 1]; ++t) {
            EncStream e = es[t];
            e.groupFirst -= v + 1;
            esHP.push_back(e);
        }
    }
    // encoder / decoder descriptors: sized by preparing into a host buffer
    const size_t planMax = size_t(I->hostRingBytes), planLPMax = size_t(b->ILP->hostRingBytes);
    std::vector<char> encHost(planMax), encLPHost(planLPMax), decHost(planMax);
    rc = encodePrepare(I, esHP.data(), u32(esHP.size()), encHost.data(), planMax, b->enc);
    if (!rc) rc = encodePrepare(b->ILP, esLP.data(), u32(esLP.size()), encLPHost.data(), planLPMax, b->encLP);
    if (!rc) rc = decodePrepare(I, ds.data(), u32(ds.size()), dsrc.data(), count, decHost.data(), planMax, b->dec);
    if (rc) { cc_volume_batch_destroy(b); return rc; }
    const size_t encAt = A.take(b->enc.bytes, 256), encLPAt = A.take(b->encLP.bytes, 256);
    const size_t decAt = A.take(b->dec.bytes, 256);
    b->memBytes = alignUp(A.off, 256);
    cudaError_t e = deviceAlloc(reinterpret_cast<void**>(&b->mem), b->memBytes);
    if (e != cudaSuccess) { b->mem = nullptr; cc_volume_batch_destroy(b); return cudaFail(e, "cudaMalloc(volume batch)"); }
    char* base = b->mem;
    // rebase the device pointers written as offsets
    auto rebaseF = [&](const float* p) -> float* { return p ? reinterpret_cast<float*>(base + reinterpret_cast<uintptr_t>(p)) : nullptr; };
    auto rebaseS = [&](const u16* p) -> u16* { return p ? reinterpret_cast<u16*>(base + reinterpret_cast<uintptr_t>(p)) : nullptr; };
    for (u32 l = 0; l < L; ++l) {
        for (auto& d : fl[l]) {
            d.src = rebaseF(d.src);
            d.lpOut = rebaseF(d.lpOut);
            d.symOut = rebaseS(d.symOut);
            d.lpSymOut = rebaseS(d.lpSymOut);
        }
        for (auto& d : fr[l]) { d.src = rebaseF(d.src); d.dst = rebaseF(d.dst); }
        for (auto& d : ir[l]) { d.src = rebaseF(d.src); d.dst = rebaseF(d.dst); }
        for (auto* vv : {&fy[l], &fz[l], &iz[l], &iy[l]})
            for (auto& d : *vv) {
                d.src = rebaseF(d.src);
                d.dst = rebaseF(d.dst);
                d.bands = rebaseS(d.bands);
                d.symOut = rebaseS(d.symOut);
                d.lpSymOut = rebaseS(d.lpSymOut);
            }
    }
    for (auto& d : qd) { d.src = rebaseF(d.src); d.sym = rebaseS(d.sym); }
    for (auto& d : dq) { d.sym = rebaseS(d.sym); d.dstF = rebaseF(d.dstF); }
    // encoder inputs and decoder outputs are symbol pointers: rebase inside the prepared descriptors
    {
        EncStreamDev* sdv = reinterpret_cast<EncStreamDev*>(encHost.data());
        for (u32 s = 0; s < b->enc.S; ++s) sdv[s].in = base + reinterpret_cast<uintptr_t>(sdv[s].in);
        EncStreamDev* ldv = reinterpret_cast<EncStreamDev*>(encLPHost.data());
        for (u32 s = 0; s < b->encLP.S; ++s) ldv[s].in = base + reinterpret_cast<uintptr_t>(ldv[s].in);
        DecStreamDesc* ddv = reinterpret_cast<DecStreamDesc*>(decHost.data());
        for (u32 s = 0; s < b->dec.S; ++s) ddv[s].out = base + reinterpret_cast<uintptr_t>(ddv[s].out);
    }
    b->syms = reinterpret_cast<u16*>(base + symAt);
    b->symBytes = size_t(symTot) * sizeof(u16);
    b->inTab = reinterpret_cast<const float**>(base + inTabAt);
    b->outTab = reinterpret_cast<float**>(base + outTabAt);
    b->wordOff = reinterpret_cast<u64*>(base + wordOffAt);
    b->bitSize = reinterpret_cast<u64*>(base + bitSizeAt);
    b->words = reinterpret_cast<u32*>(base + wordsAt);
    b->enc.dev = base + encAt;
    b->encLP.dev = base + encLPAt;
    b->dec.dev = base + decAt;
    b->dec.wordsBase = b->words;
    b->dec.wordOff = b->wordOff;
    b->dec.bitSize = b->bitSize;
    // upload everything once
    auto up = [&](size_t at, const void* src, size_t bytes) -> cudaError_t {
        return bytes ? cudaMemcpy(base + at, src, bytes, cudaMemcpyHostToDevice) : cudaSuccess;
    };
    e = cudaMemset(b->mem, 0, b->memBytes);
    for (u32 l = 0; l < L && e == cudaSuccess; ++l) {
        e = up(flAt[l], fl[l].data(), fl[l].size() * sizeof(BLevelDesc));
        if (e == cudaSuccess) e = up(frAt[l], fr[l].data(), fr[l].size() * sizeof(BRowDesc));
        if (e == cudaSuccess) e = up(irAt[l], ir[l].data(), ir[l].size() * sizeof(BRowDesc));
        if (e == cudaSuccess) e = up(fyAt[l], fy[l].data(), fy[l].size() * sizeof(BColDesc));
        if (e == cudaSuccess) e = up(fzAt[l], fz[l].data(), fz[l].size() * sizeof(BColDesc));
        if (e == cudaSuccess) e = up(izAt[l], iz[l].data(), iz[l].size() * sizeof(BColDesc));
        if (e == cudaSuccess) e = up(iyAt[l], iy[l].data(), iy[l].size() * sizeof(BColDesc));
    }
    for (size_t m = 0; m < maps.size() && e == cudaSuccess; ++m) e = up(mapAt[m], maps[m].data(), maps[m].size() * sizeof(u32));
    if (e == cudaSuccess) e = up(qAt, qd.data(), qd.size() * sizeof(BQuantDesc));
    if (e == cudaSuccess) e = up(dqAt, dq.data(), dq.size() * sizeof(BQuantDesc));
    if (e == cudaSuccess) e = up(encAt, encHost.data(), b->enc.bytes);
    if (e == cudaSuccess) e = up(encLPAt, encLPHost.data(), b->encLP.bytes);
    if (e == cudaSuccess) e = up(decAt, decHost.data(), b->dec.bytes);
    if (e == cudaSuccess) e = pinnedAlloc(reinterpret_cast<void**>(&b->hostPlan), sizeof(void*) * count * kTabRing);
    for (unsigned r = 0; r < kTabRing && e == cudaSuccess; ++r)
        e = cudaEventCreateWithFlags(&b->tabEvent[r], cudaEventDisableTiming);
    if (e == cudaSuccess) e = pinnedAlloc(reinterpret_cast<void**>(&b->hostExt), 2 * sizeof(u64) * count);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->extEvent, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) { cc_volume_batch_destroy(b); return cudaFail(e, "volume batch set-up"); }
    b->flHost = fl;
    b->izHost = iz;
    b->qdHost = qd;
    b->dqHost = dq;
    b->fwdLevel.resize(L);
    b->fwdRows.resize(L); b->invRows.resize(L); b->fwdY.resize(L); b->fwdZ.resize(L); b->invZ.resize(L); b->invY.resize(L);
    auto mapPtr = [&](size_t m) { return reinterpret_cast<const u32*>(base + mapAt[m]); };
    for (u32 l = 0; l < L; ++l) {
        b->fwdLevel[l] = {reinterpret_cast<const BLevelDesc*>(base + flAt[l]), mapPtr(flMap[l]), u32(fl[l].size()), flC[l]};
        b->fwdRows[l] = {reinterpret_cast<const BRowDesc*>(base + frAt[l]), mapPtr(frMap[l]), u32(fr[l].size()), frC[l]};
        b->invRows[l] = {reinterpret_cast<const BRowDesc*>(base + irAt[l]), mapPtr(irMap[l]), u32(ir[l].size()), irC[l]};
        b->fwdY[l] = {reinterpret_cast<const BColDesc*>(base + fyAt[l]), mapPtr(fyMap[l]), u32(fy[l].size()), fyC[l]};
        b->fwdZ[l] = {reinterpret_cast<const BColDesc*>(base + fzAt[l]), mapPtr(fzMap[l]), u32(fz[l].size()), fzC[l]};
        b->invZ[l] = {reinterpret_cast<const BColDesc*>(base + izAt[l]), mapPtr(izMap[l]), u32(iz[l].size()), izC[l]};
        b->invY[l] = {reinterpret_cast<const BColDesc*>(base + iyAt[l]), mapPtr(iyMap[l]), u32(iy[l].size()), iyC[l]};
    }
    b->quant = {reinterpret_cast<const BQuantDesc*>(base + qAt), mapPtr(qMap), u32(qd.size()), qC};
    b->dequantLP = {reinterpret_cast<const BQuantDesc*>(base + dqAt), mapPtr(dqMap), u32(dq.size()), dqC};
    // prefixes by volume
    auto prefix = [&](auto& li, const auto& host, u32 perVolume) {
        li.descEnd.resize(count);
        li.ctaEnd.resize(count);
        for (u32 v = 0; v < count; ++v) {
            const u32 e = (v + 1) * perVolume;
            li.descEnd[v] = e;
            li.ctaEnd[v] = e < host.size() ? host[e].ctaOff : li.ctas;
        }
    };
    for (u32 l = 0; l < L; ++l) {
        prefix(b->fwdLevel[l], fl[l], 1);
        prefix(b->fwdRows[l], fr[l], 1);
        prefix(b->invRows[l], ir[l], 1);
        prefix(b->fwdY[l], fy[l], 1);
        prefix(b->fwdZ[l], fz[l], 1);
        prefix(b->invZ[l], iz[l], 1);
        prefix(b->invY[l], iy[l], 1);
    }
    prefix(b->quant, qd, 1 + 7 * L);
    prefix(b->dequantLP, dq, 1);
    {
        const u32 cb = I->codingBlockSize;
        u32 S = 0, T = 0, tiles = 0, blocks = 0, nRl = 0, nH = 0, rlB = 0, hB = 0;
        u32 hS = 0, hT = 0, hTiles = 0, hBlocks = 0, lTiles = 0, lBlocks = 0;
        for (u32 v = 0; v < count; ++v) {
            for (u32 st = firstStream[v]; st < firstStream[v + 1]; ++st) {
                const EncStream& e = es[st];
                const u32 nb = u32(ceilDiv(e.n, cb)), nt = u32(ceilDiv(e.n, kRleTile));
                ++S;
                tiles += nt;
                if (e.kind == KIND_RLHUFF) {
                    T += 2; blocks += 2 * nb; ++nRl; rlB += nb;
                    ++hS; hT += 2; hTiles += nt; hBlocks += 2 * nb;
                } else {
                    T += 1; blocks += nb; ++nH; hB += nb;
                    lTiles += nt; lBlocks += nb;
                }
            }
            b->encS.push_back(hS);
            b->encT.push_back(hT);
            b->encTiles.push_back(hTiles);
            b->encBlocks.push_back(hBlocks);
            b->lpTiles.push_back(lTiles);
            b->lpBlocks.push_back(lBlocks);
            b->decS.push_back(S);
            b->decT.push_back(T);
            b->decRl.push_back(nRl);
            b->decH.push_back(nH);
            b->decRlBlocks.push_back(rlB);
            b->decHBlocks.push_back(hB);
            b->symEnd.push_back(symOff[v] + sl[v].total);
        }
    }
    b->active = count;
    *out = b;
    return CC_OK;
}

void cc_volume_batch_destroy(cc_volume_batch* b) {
    if (!b) return;
    DeviceGuard deviceGuard(b->I ? b->I->device : -1);
    cudaDeviceSynchronize();
    for (auto& kv : b->gCompress) cudaGraphExecDestroy(kv.second);
    for (auto& kv : b->gDecompress) cudaGraphExecDestroy(kv.second);
    if (b->captureStream) cudaStreamDestroy(b->captureStream);
    if (b->sideStream) cudaStreamDestroy(b->sideStream);
    if (b->evFork) cudaEventDestroy(b->evFork);
    if (b->evJoin) cudaEventDestroy(b->evJoin);
    for (cudaEvent_t ev : b->tabEvent)
        if (ev) cudaEventDestroy(ev);
    if (b->hostPlan) cudaFreeHost(b->hostPlan);
    if (b->hostExt) cudaFreeHost(b->hostExt);
    if (b->extEvent) cudaEventDestroy(b->extEvent);
    if (b->mem) cudaFree(b->mem);
    if (b->ILP) cc_destroy_instance(b->ILP);
    if (b->I) cc_destroy_instance(b->I);
    delete b;
}

int cc_volume_batch_set_active(cc_volume_batch* b, uint32_t active) {
    if (!b || active == 0 || active > b->count) { setError("cc_volume_batch_set_active: active must be 1..count"); return CC_ERR_INVALID_ARGUMENT; }
    b->active = active;
    return CC_OK;
}

int cc_volume_batch_set_stream(cc_volume_batch* b, void* stream) {
    if (!b) { setError("cc_volume_batch_set_stream: null batch"); return CC_ERR_INVALID_ARGUMENT; }
    b->ownStream = static_cast<cudaStream_t>(stream);
    b->hasOwnStream = true;
    return CC_OK;
}

int cc_volume_batch_use_graph(cc_volume_batch* b, int enable) {
    if (!b) { setError("cc_volume_batch_use_graph: null batch"); return CC_ERR_INVALID_ARGUMENT; }
    b->useGraph = enable != 0;
    return CC_OK;
}

int cc_volume_batch_compress(cc_volume_batch* b, const float* const* dVolumes) {
    if (!b || !dVolumes) { setError("cc_volume_batch_compress: null argument"); return CC_ERR_INVALID_ARGUMENT; }
    DeviceGuard deviceGuard(b->I->device);
    b->I->stream = b->hasOwnStream ? b->ownStream : b->user->stream;
    b->I->timing = b->user->timing;
    b->ILP->timing = b->user->timing;
    int rc = uploadTable(b, reinterpret_cast<const void* const*>(dVolumes), b->inTab);
    if (rc) return rc;
    return runMaybeGraph(b, batchEnqueueCompress, b->gCompress, b->launchesCompress);
}

int cc_volume_batch_decompress(cc_volume_batch* b, float* const* dVolumes) {
    if (!b || !dVolumes) { setError("cc_volume_batch_decompress: null argument"); return CC_ERR_INVALID_ARGUMENT; }
    DeviceGuard deviceGuard(b->I->device);
    b->I->stream = b->hasOwnStream ? b->ownStream : b->user->stream;
    b->I->timing = b->user->timing;
    int rc = uploadTable(b, reinterpret_cast<const void* const*>(dVolumes), b->outTab);
    if (rc) return rc;
    return runMaybeGraph(b, batchEnqueueDecompress, b->gDecompress, b->launchesDecompress);
}

int cc_volume_batch_stream(const cc_volume_batch* b, const uint32_t** dWords, const uint64_t** dWordOffsets,
                           const uint64_t** dBitSizes, uint64_t* capacityWords) {
    if (!b) { setError("cc_volume_batch_stream: null batch"); return CC_ERR_INVALID_ARGUMENT; }
    if (dWords) *dWords = b->words;
    if (dWordOffsets) *dWordOffsets = b->wordOff;
    if (dBitSizes) *dBitSizes = b->bitSize;
    if (capacityWords) *capacityWords = b->wordsCap;
    return CC_OK;
}

int cc_volume_batch_read_stream(cc_volume_batch* b, uint32_t v, uint32_t* dst, uint64_t capacityWords,
                                uint64_t* bitSize) {
    if (!b || !bitSize || v >= b->count) { setError("cc_volume_batch_read_stream: bad argument"); return CC_ERR_INVALID_ARGUMENT; }
    DeviceGuard deviceGuard(b->I->device);
    u64 ext[2] = {0, 0};
    CC_TRY_CUDA(cudaMemcpyAsync(&ext[0], b->wordOff + v, sizeof(u64), cudaMemcpyDeviceToHost, b->I->stream), "read offset");
    CC_TRY_CUDA(cudaMemcpyAsync(&ext[1], b->bitSize + v, sizeof(u64), cudaMemcpyDeviceToHost, b->I->stream), "read size");
    CC_TRY_CUDA(cudaStreamSynchronize(b->I->stream), "read stream");
    *bitSize = ext[1];
    const u64 words = ceilDiv(ext[1], 32);
    if (!dst) return CC_OK;
    if (words > capacityWords) { setError("cc_volume_batch_read_stream: need %llu words", (unsigned long long)words); return CC_ERR_CAPACITY; }
    CC_TRY_CUDA(cudaMemcpy(dst, b->words + ext[0], words * 4, cudaMemcpyDefault), "copy stream");
    return CC_OK;
}

// Device address of page-locked host memory (CC_ERR_INVALID_ARGUMENT if the
// memory is not page-locked).
static int hostDevicePointer(const void* h, void** d, const char* what) {
    cudaPointerAttributes a{};
    if (!h || cudaPointerGetAttributes(&a, h) != cudaSuccess || a.type != cudaMemoryTypeHost) {
        cudaGetLastError();
        setError("%s: host buffers must be page-locked (cudaHostAlloc / cudaHostRegister)", what);
        return CC_ERR_INVALID_ARGUMENT;
    }
    *d = a.devicePointer ? a.devicePointer : const_cast<void*>(h);
    return CC_OK;
}

int cc_volume_batch_download_streams(cc_volume_batch* b, uint32_t* hWords, uint64_t capacityWords, uint64_t* hExt) {
    const char* what = "cc_volume_batch_download_streams";
    if (!b || !b->active) { setError("%s: bad argument", what); return CC_ERR_INVALID_ARGUMENT; }
    DeviceGuard deviceGuard(b->I->device);
    void *dW = nullptr, *dE = nullptr;
    int rc = hostDevicePointer(hWords, &dW, what);
    if (!rc) rc = hostDevicePointer(hExt, &dE, what);
    if (rc) return rc;
    cudaStream_t st = b->hasOwnStream ? b->ownStream : b->user->stream;
    b->I->stream = st;
    const bool vec = (reinterpret_cast<uintptr_t>(dW) & 15) == 0;
    const unsigned g = 148 * 4;
    if (vec) k_streamsToHost<true><<<g, 256, 0, st>>>(b->words, b->wordOff, b->bitSize, b->active, static_cast<u32*>(dW), capacityWords, static_cast<u64*>(dE), b->I->errors);
    else k_streamsToHost<false><<<g, 256, 0, st>>>(b->words, b->wordOff, b->bitSize, b->active, static_cast<u32*>(dW), capacityWords, static_cast<u64*>(dE), b->I->errors);
    countLaunch();
    CC_TRY_CUDA(cudaGetLastError(), what);
    return CC_OK;
}

int cc_volume_batch_upload_streams(cc_volume_batch* b, const uint32_t* hWords, const uint64_t* hExt) {
    const char* what = "cc_volume_batch_upload_streams";
    if (!b || !b->active) { setError("%s: bad argument", what); return CC_ERR_INVALID_ARGUMENT; }
    DeviceGuard deviceGuard(b->I->device);
    void *dW = nullptr, *dE = nullptr;
    int rc = hostDevicePointer(hWords, &dW, what);
    if (!rc) rc = hostDevicePointer(hExt, &dE, what);
    if (rc) return rc;
    cudaStream_t st = b->hasOwnStream ? b->ownStream : b->user->stream;
    b->I->stream = st;
    const bool vec = (reinterpret_cast<uintptr_t>(dW) & 15) == 0;
    const unsigned g = 148 * 4;
    if (vec) k_streamsFromHost<true><<<g, 256, 0, st>>>(static_cast<const u32*>(dW), static_cast<const u64*>(dE), b->active, b->words, b->wordOff, b->bitSize, b->wordsCap, b->I->errors + 4);
    else k_streamsFromHost<false><<<g, 256, 0, st>>>(static_cast<const u32*>(dW), static_cast<const u64*>(dE), b->active, b->words, b->wordOff, b->bitSize, b->wordsCap, b->I->errors + 4);
    countLaunch();
    CC_TRY_CUDA(cudaGetLastError(), what);
    return CC_OK;
}

int cc_volume_batch_load_streams(cc_volume_batch* b, const uint32_t* const* words, const uint64_t* bitSizes) {
    if (!b || !words || !bitSizes) { setError("cc_volume_batch_load_streams: null argument"); return CC_ERR_INVALID_ARGUMENT; }
    DeviceGuard deviceGuard(b->I->device);
    cudaStream_t st = b->hasOwnStream ? b->ownStream : b->user->stream;
    b->I->stream = st;
    cudaEventSynchronize(b->extEvent);   // the previous load has read the pinned offsets
    u64 at = 0;
    for (u32 v = 0; v < b->active; ++v) {
        const u64 nw = ceilDiv(bitSizes[v], 32);
        if (at + nw > b->wordsCap) { setError("cc_volume_batch_load_streams: streams exceed the batch buffer (%llu words)", (unsigned long long)b->wordsCap); return CC_ERR_CAPACITY; }
        b->hostExt[v] = at;
        b->hostExt[b->active + v] = bitSizes[v];
        if (nw) CC_TRY_CUDA(cudaMemcpyAsync(b->words + at, words[v], nw * 4, cudaMemcpyDefault, st), "load stream");
        at += nw;
    }
    CC_TRY_CUDA(cudaMemcpyAsync(b->wordOff, b->hostExt, sizeof(u64) * b->active, cudaMemcpyHostToDevice, st), "load offsets");
    CC_TRY_CUDA(cudaMemcpyAsync(b->bitSize, b->hostExt + b->active, sizeof(u64) * b->active, cudaMemcpyHostToDevice, st), "load sizes");
    cudaEventRecord(b->extEvent, st);
    return CC_OK;
}

int cc_volume_batch_status(cc_volume_batch* b) {
    if (!b) return CC_ERR_INVALID_ARGUMENT;
    u32 flags[8] = {}, lp = 0;
    CC_TRY_CUDA(cudaMemcpyAsync(flags, b->I->errors, sizeof(flags), cudaMemcpyDeviceToHost, b->I->stream), "batch status");
    CC_TRY_CUDA(cudaMemcpyAsync(&lp, b->ILP->errors, sizeof(lp), cudaMemcpyDeviceToHost, b->I->stream), "batch status");
    CC_TRY_CUDA(cudaStreamSynchronize(b->I->stream), "batch status");
    if (lp) return deviceErrorStatus(lp, "batch compress (lowpass streams)");
    if (flags[0]) return deviceErrorStatus(flags[0], "batch compress");
    return deviceErrorStatus(flags[4], "batch decompress");
}

// Resolves and folds the batch's internal timing sections into the user
// instance (cc_timing_* report both); the lowpass encode's own sections
// (on the side stream) get the prefix "lp.".
void cc_volume_batch_collect_timings(cc_volume_batch* b) {
    if (!b) return;
    b->I->resolveTimings();
    for (auto& kv : b->I->timings) {
        auto& acc = b->user->timings[kv.first];
        acc.first += kv.second.first;
        acc.second += kv.second.second;
    }
    b->I->timings.clear();
    b->ILP->resolveTimings();
    for (auto& kv : b->ILP->timings) {
        auto& acc = b->user->timings[std::string("lp.") + kv.first];
        acc.first += kv.second.first;
        acc.second += kv.second.second;
    }
    b->ILP->timings.clear();
}

}  // extern "C"
