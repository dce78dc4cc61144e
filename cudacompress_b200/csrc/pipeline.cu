// pipeline.cu - whole-codec entry points: the lossy volume codecs
// (examples CompressVolume.cpp:312-856: float, with doRLEOnlyOnLvl0, quantize-
// first, and their multi-channel decoders) and the lossless 2D heightfield codec
// (one level = CompressHeightfield.cpp:82-216 band layout, levels chained as
// compressVolumeLossless, CompressVolume.cpp:234-309).  Device-resident input
// and device-resident 32-bit-word bit stream.
//
// Volume stream: LP band (step q0/2^(L-1)) encodeHuff, then for level
// L-1 .. 0 the 7 highpass bands (index x+2y+4z, step q0/2^level) encodeRLHuff.
// Heightfield stream: LP encodeHuff, then levels L-1 .. 0, 3 bands each
// (index x+2y) encodeRLHuff, every level starting word aligned.
#include <cstring>
#include <vector>

#include "batch.cuh"

namespace ccb {

namespace {

struct Bump {
    char* base;
    size_t off = 0;
    template <class T>
    T* take(u64 n) {
        off = alignUp(off, 256);
        T* p = reinterpret_cast<T*>(base + off);
        off += n * sizeof(T);
        return p;
    }
};

u64 cube(u64 a, u64 b, u64 c) { return a * b * c; }

}  // namespace

// Encodes the groups back to back into dWords (word aligned segments; the
// reference's BitStream is word aligned at every group start here), batching
// as many groups per device call as the instance's symbol and stream budget
// allows.  A batch whose histograms exceed the instance's table capacity is
// redone one group per call (the capacity every instance guarantees).
int encodeGroups(cc_instance* I, const std::vector<EncStream>& streams, const std::vector<EncGroup>& groups,
                 u32* dWords, u64 cap, u64* wordsOut, std::vector<u64>* groupStart) {
    if (groupStart) groupStart->assign(groups.size() + 1, 0);
    // word range of group k of the batch just encoded at word `base`
    auto record = [&](size_t k, u32 batchFirst, u64 base) {
        if (!groupStart) return;
        const SegmentLayout& a = I->lastLayout[groups[k].first - batchFirst];
        const SegmentLayout& b = I->lastLayout[groups[k].first + groups[k].count - 1 - batchFirst];
        (*groupStart)[k] = base + a.startWord;
        (*groupStart)[k + 1] = base + b.startWord + b.words;
    };
    u64 at = 0;
    size_t g = 0;
    while (g < groups.size()) {
        // greedy batch [g, h)
        size_t h = g;
        u64 compact = 0, tiles = 0, blocks = 0, nStreams = 0;
        while (h < groups.size()) {
            u64 c2 = compact, t2 = tiles, b2 = blocks;
            for (u32 i = 0; i < groups[h].count; ++i) {
                const EncStream& e = streams[groups[h].first + i];
                const u64 nb = ceilDiv(e.n, I->codingBlockSize);
                if (e.kind == KIND_RLHUFF) c2 += e.n;
                t2 += ceilDiv(e.n, kRleTile);
                b2 += e.kind == KIND_RLHUFF ? 2 * nb : nb;
            }
            const u64 s2 = nStreams + groups[h].count;
            const bool fits = s2 <= I->capStreams && c2 <= I->capCompact && t2 <= I->capTiles && b2 <= I->capBlocks;
            if (!fits && h > g) break;
            compact = c2; tiles = t2; blocks = b2; nStreams = s2;
            ++h;
            if (!fits) break;   // a single group that does not fit reports the error below
        }
        const u32 first = groups[g].first;
        const u32 count = groups[h - 1].first + groups[h - 1].count - first;
        std::vector<EncStream> batch(streams.begin() + first, streams.begin() + first + count);
        for (EncStream& e : batch) e.groupFirst -= first;
        u64 words = 0;
        int rc = encodeDevice(I, batch.data(), count, EncOutput{dWords + at, cap - at}, false, &words);
        if (rc == CC_ERR_CAPACITY && h - g > 1) {
            for (size_t k = g; k < h; ++k) {
                std::vector<EncStream> one(streams.begin() + groups[k].first,
                                           streams.begin() + groups[k].first + groups[k].count);
                for (EncStream& e : one) e.groupFirst -= groups[k].first;
                if ((rc = encodeDevice(I, one.data(), groups[k].count, EncOutput{dWords + at, cap - at}, false, &words)))
                    return rc;
                record(k, groups[k].first, at);
                at += words;
            }
        } else if (rc) {
            return rc;
        } else {
            for (size_t k = g; k < h; ++k) record(k, first, at);
            at += words;
        }
        g = h;
    }
    *wordsOut = at;
    return CC_OK;
}

}  // namespace ccb

// ---------------------------------------------------------------------------
// Lossy volume codecs.  Stream: LP band encodeHuff, then for level L-1 .. 0
// the 7 highpass bands (index x+2y+4z) encodeRLHuff - encodeHuff above level
// 0 with CC_VOLUME_RLE_ONLY_LEVEL0 (doRLEOnlyOnLvl0, CompressVolume.cpp:
// 389-395, 491-495).  Float codec: float DWT + deadzone quantization with
// step q0/2^level (CompressVolume.cpp:312-516).  Quant-first codec: uniform
// quantization to short, integer DWT, symbolize (CompressVolume.cpp:651-856).
// ---------------------------------------------------------------------------
namespace ccb {
namespace {

bool volumeSizesOk(u32 nx, u32 ny, u32 nz, u32 levels, const char* what) {
    const u32 f = levels ? 1u << levels : 0u;
    if (levels == 0 || levels > 12 || nx % f || ny % f || nz % f || (nx >> (levels - 1)) < 8 ||
        (ny >> (levels - 1)) < 8 || (nz >> (levels - 1)) < 8) {
        setError("%s: sizes must be divisible by 2^levels with coarsest level >= 8", what);
        return false;
    }
    return true;
}

// Symbol layout of one volume: LP, then levels L-1 .. 0 with 7 bands each.
struct VolumeSymbols {
    u64 lp = 0, total = 0;
    std::vector<u64> level;   // first band of level l
    std::vector<u64> band;    // band size of level l
};

VolumeSymbols volumeSymbols(u32 nx, u32 ny, u32 nz, u32 L) {
    VolumeSymbols v;
    v.level.assign(L, 0);
    v.band.assign(L, 0);
    v.lp = cube(nx >> L, ny >> L, nz >> L);
    u64 at = v.lp;
    for (int l = int(L) - 1; l >= 0; --l) {
        v.level[l] = at;
        v.band[l] = cube(nx >> (l + 1), ny >> (l + 1), nz >> (l + 1));
        at += 7 * v.band[l];
    }
    v.total = at;
    return v;
}

// Entropy coding of one volume's symbols (layout volumeSymbols) into dWords.
int encodeVolumeSymbols(cc_instance* I, const u16* syms, const VolumeSymbols& vs, u32 L, bool rleOnly, u32* dWords,
                        u64 cap, u32* bitSize, const char* what) {
    std::vector<EncStream> es;
    std::vector<EncGroup> groups;
    es.push_back(EncStream{syms, u32(vs.lp), 0, 0, 1, KIND_HUFF});
    groups.push_back(EncGroup{0, 1});
    for (int l = int(L) - 1; l >= 0; --l) {
        const u32 first = u32(es.size());
        const u32 kind = (rleOnly && l > 0) ? KIND_HUFF : KIND_RLHUFF;
        for (u32 i = 0; i < 7; ++i)
            es.push_back(EncStream{syms + vs.level[l] + i * vs.band[l], u32(vs.band[l]), 0, first, 7, kind});
        groups.push_back(EncGroup{first, 7});
    }
    u64 at = 0;
    int rc = encodeGroups(I, es, groups, dWords, cap, &at);
    if (rc) return rc;
    CC_TRY_CUDA(cudaStreamSynchronize(I->stream), what);
    if (at * 32 > 0xffffffffull) { setError("%s: stream exceeds 2^32 bits", what); return CC_ERR_CAPACITY; }
    *bitSize = u32(at * 32);
    return CC_OK;
}

// Decodes `count` volume streams of the same sizes (device words) into their
// symbols (volume c at syms + c * vs.total): all LP streams in one decode
// call, then each level's bands of all volumes in one call
// (decompressVolumeFloatMultiChannel, CompressVolume.cpp:518-648).
int decodeVolumeSymbols(cc_instance* I, const u32* const* dWords, const u32* bitSizes, u32 count, u32 L, bool rleOnly,
                        const VolumeSymbols& vs, u16* syms, const char* what) {
    cudaStream_t st = I->stream;
    if (u64(count) * 7 > I->streamCountMax || vs.band.empty() || vs.band[0] > I->elemCountPerStreamMax) {
        setError("%s: instance needs >= %u streams of >= %llu symbols", what, count * 7,
                 (unsigned long long)(vs.band.empty() ? 0 : vs.band[0]));
        return CC_ERR_CAPACITY;
    }
    // the bit stream walk happens on the host
    std::vector<std::vector<u32>> host(count);
    for (u32 c = 0; c < count; ++c) {
        const u64 words = ceilDiv(u64(bitSizes[c]), 32);
        if (words > I->hostWordsMax) { setError("%s: stream larger than instance staging", what); return CC_ERR_CAPACITY; }
        host[c].resize(words);
        CC_TRY_CUDA(cudaMemcpyAsync(I->hostWords, dWords[c], words * 4, cudaMemcpyDeviceToHost, st), "download stream");
        CC_TRY_CUDA(cudaStreamSynchronize(st), "download stream");
        std::memcpy(host[c].data(), I->hostWords, words * 4);
    }
    std::vector<const u32*> hw(count);
    std::vector<u32> pos(count, 0), bsIndex(7 * count);
    for (u32 c = 0; c < count; ++c) hw[c] = host[c].data();
    std::vector<void*> outs(7 * count);
    for (u32 c = 0; c < count; ++c) { outs[c] = syms + c * vs.total; bsIndex[c] = c; }
    int rc = decodeDevice(I, KIND_HUFF, hw.data(), bitSizes, pos.data(), count, bsIndex.data(), outs.data(), count,
                          u32(vs.lp));
    if (rc) return rc;
    for (u32 c = 0; c < count; ++c) pos[c] = u32(alignUp(pos[c], 32));
    for (int l = int(L) - 1; l >= 0; --l) {
        const bool huff = rleOnly && l > 0;
        for (u32 c = 0; c < count; ++c) {
            u16* first = syms + c * vs.total + vs.level[l];
            for (u32 i = 0; i < 7; ++i) {
                outs[c * 7 + i] = first + i * vs.band[l];
                bsIndex[c * 7 + i] = c;
            }
        }
        rc = decodeDevice(I, huff ? KIND_HUFF : KIND_RLHUFF, hw.data(), bitSizes, pos.data(), count, bsIndex.data(),
                          outs.data(), 7 * count, u32(vs.band[l]));
        if (rc) return rc;
        for (u32 c = 0; c < count; ++c) pos[c] = u32(alignUp(pos[c], 32));
    }
    return CC_OK;
}

// compressVolumeFloat and decompressVolumeFloat(MultiChannel) run through a
// volume batch of the call's volumes (csrc/batch.cu: the fused forward
// levels, both encodes at once, one device-side walk and decode of all
// streams, the batched inverse passes, CUDA graphs) that the instance keeps
// for later calls of the same volume count, sizes and levels; a call with
// other quantization steps patches the batch's steps.  Making a batch costs
// 10-20 ms (allocations, plans, graph capture), so a shape gets one only on
// its fifth consecutive call: calls that change shape every time, or every
// compress / decompress pair (bricks of many sizes), stay on the
// level-by-level path.  The batch
// writes and reads the same stream format bit-identically.  kNoBatch: no
// batch for this call (sizes outside the batch's limits, or a shape not yet
// repeated), nothing done - the caller runs the level-by-level path.
constexpr int kNoBatch = 1 << 20;
constexpr u32 kPlainBatchRun = 5;   // consecutive calls of a shape before it gets a batch

int plainBatchFor(cc_instance* I, u32 count, u32 nx, u32 ny, u32 nz, u32 L, const float* q, const char* what,
                  cc_volume_batch** out) {
    // the instance's declared capacities bound the call, as on the level path
    if (u64(count) * 7 > I->streamCountMax || cube(nx / 2, ny / 2, nz / 2) > I->elemCountPerStreamMax) {
        setError("%s: instance needs >= %u streams of >= %llu symbols", what, count * 7,
                 (unsigned long long)cube(nx / 2, ny / 2, nz / 2));
        return CC_ERR_CAPACITY;
    }
    if (L > 8 || cube(nx, ny, nz) >= (u64(1) << 31)) return kNoBatch;
    for (u32 c = 0; c < count; ++c)
        if (!(q[c] > 0.0f)) { setError("%s: volume %u: quantization step must be > 0", what, c); return CC_ERR_INVALID_ARGUMENT; }
    const u32 key[5] = {count, nx, ny, nz, L};
    if (std::memcmp(key, I->plainSeenKey, sizeof(key)) == 0) {
        ++I->plainSeenRun;
    } else {
        std::memcpy(I->plainSeenKey, key, sizeof(key));
        I->plainSeenRun = 1;
    }
    cc_instance::PlainBatch* slot = nullptr;
    for (auto& pb : I->plainBatch)
        if (pb.b && std::memcmp(key, pb.key, sizeof(key)) == 0) slot = &pb;
    if (!slot) {
        if (I->plainSeenRun < kPlainBatchRun) return kNoBatch;
        slot = &I->plainBatch[0];
        for (auto& pb : I->plainBatch)
            if (!pb.b || pb.used < slot->used) slot = &pb;   // an empty slot, else the least recently used
        if (slot->b) cc_volume_batch_destroy(slot->b);
        slot->b = nullptr;
        std::vector<u32> sizes(3 * size_t(count));
        for (u32 c = 0; c < count; ++c) { sizes[3 * c] = nx; sizes[3 * c + 1] = ny; sizes[3 * c + 2] = nz; }
        cc_volume_batch* b = nullptr;
        const int rc = cc_volume_batch_create(I, count, sizes.data(), L, q, &b);
        if (rc) return rc;
        slot->b = b;
        std::memcpy(slot->key, key, sizeof(key));
    }
    slot->used = ++I->plainCalls;
    // with timing on, the calls run launch by launch so that every section is
    // recorded (a graph replay records none)
    cc_volume_batch_use_graph(slot->b, I->timing ? 0 : 1);
    int rc = cc_volume_batch_set_stream(slot->b, I->stream);
    if (!rc) rc = batchSetQuantSteps(slot->b, q);
    *out = slot->b;
    return rc;
}

int compressVolumeFloatBatched(cc_instance* I, const float* vol, u32 nx, u32 ny, u32 nz, u32 L, float q0,
                               u32* dWords, u64 cap, u32* bitSize, const char* what) {
    cc_volume_batch* b = nullptr;
    int rc = plainBatchFor(I, 1, nx, ny, nz, L, &q0, what, &b);
    if (rc) return rc;
    const float* vols[1] = {vol};
    rc = cc_volume_batch_compress(b, vols);
    if (!rc) rc = batchStatusOf(b, false);   // synchronizes the stream
    if (I->timing) cc_volume_batch_collect_timings(b);   // the batch's sections into the instance's
    u64 bits = 0;
    if (!rc) rc = cc_volume_batch_read_stream(b, 0, dWords, cap, &bits);
    if (!rc && bits > 0xffffffffull) { setError("%s: stream exceeds 2^32 bits", what); rc = CC_ERR_CAPACITY; }
    if (!rc) *bitSize = u32(bits);
    return rc;
}

int decompressVolumeFloatBatched(cc_instance* I, const cc_volume_channel* ch, u32 count, u32 nx, u32 ny, u32 nz,
                                 u32 L, const char* what) {
    std::vector<float> q(count);
    for (u32 c = 0; c < count; ++c) q[c] = ch[c].quant_step;
    cc_volume_batch* b = nullptr;
    int rc = plainBatchFor(I, count, nx, ny, nz, L, q.data(), what, &b);
    if (rc) return rc;
    std::vector<const u32*> words(count);
    std::vector<u64> bits(count);
    std::vector<float*> outs(count);
    for (u32 c = 0; c < count; ++c) { words[c] = ch[c].d_words; bits[c] = ch[c].bit_size; outs[c] = ch[c].d_volume; }
    rc = cc_volume_batch_load_streams(b, words.data(), bits.data());
    if (!rc) rc = cc_volume_batch_decompress(b, outs.data());
    if (!rc) rc = batchStatusOf(b, true);   // synchronizes the stream
    if (I->timing) cc_volume_batch_collect_timings(b);   // the batch's sections into the instance's
    return rc;
}

// ---- float codec ----
int compressVolumeFloat(cc_instance* I, const float* vol, u32 nx, u32 ny, u32 nz, u32 L, float q0, bool rleOnly,
                        u32* dWords, u64 cap, u32* bitSize) {
    const char* what = "compressVolumeFloat";
    if (!I || !vol || !dWords || !bitSize) { setError("%s: bad argument", what); return CC_ERR_INVALID_ARGUMENT; }
    if (!volumeSizesOk(nx, ny, nz, L, what)) return CC_ERR_INVALID_ARGUMENT;
    if (I->symBytes != 2) { setError("%s: needs a 16-bit-symbol instance", what); return CC_ERR_INVALID_ARGUMENT; }
    const u64 band0 = cube(nx / 2, ny / 2, nz / 2);
    if (I->streamCountMax < 7 || I->elemCountPerStreamMax < band0) {
        setError("%s: instance needs >= 7 streams of >= %llu symbols", what, (unsigned long long)band0);
        return CC_ERR_CAPACITY;
    }
    DeviceGuard deviceGuard(I->device);
    if (!rleOnly) {
        const int rc = compressVolumeFloatBatched(I, vol, nx, ny, nz, L, q0, dWords, cap, bitSize, what);
        if (rc != kNoBatch) return rc;
    }
    cudaStream_t st = I->stream;
    const u64 N0 = cube(nx, ny, nz);
    const VolumeSymbols vs = volumeSymbols(nx, ny, nz, L);
    Bump b{nullptr};
    b.take<float>(N0);
    b.take<float>(N0);
    for (u32 l = 0; l < L; ++l) b.take<float>(cube(nx >> l, ny >> l, nz >> l));
    b.take<u16>(vs.total + 1024);
    int rc = ensurePipelineWork(I, b.off + 1024);
    if (rc) return rc;
    Bump w{I->pipeWork};
    float* t1 = w.take<float>(N0);
    float* t2 = w.take<float>(N0);
    std::vector<float*> coef(L);
    for (u32 l = 0; l < L; ++l) coef[l] = w.take<float>(cube(nx >> l, ny >> l, nz >> l));
    u16* syms = w.take<u16>(vs.total + 1024);
    // forward transforms: level l reads the LLL corner of level l-1
    for (u32 l = 0; l < L; ++l) {
        const int sx = int(nx >> l), sy = int(ny >> l), sz = int(nz >> l);
        const float* src = l == 0 ? vol : coef[l - 1];
        const int sr = l == 0 ? 0 : int(nx >> (l - 1));
        const int ss = l == 0 ? 0 : int((nx >> (l - 1)) * (ny >> (l - 1)));
        { SectionTimer t(I, "pipe.dwt_forward", st); rc = cc_dwt_float_forward(coef[l], t2, t1, src, sx, sy, sz, 1, 0, 0, sr, ss, st); }
        if (rc) return rc;
    }
    // deadzone quantization: LP (step q0/2^(L-1)), then levels coarse -> fine, bands 1..7 (step q0/2^l)
    const u32 lx = nx >> L, ly = ny >> L, lz = nz >> L;
    rc = cc_quantize_to_symbols(syms, 2, coef[L - 1], lx, ly, lz, q0 / float(1u << (L - 1)), nx >> (L - 1),
                                (nx >> (L - 1)) * (ny >> (L - 1)), 0, st);
    if (rc) return rc;
    for (int l = int(L) - 1; l >= 0; --l) {
        const u32 sx = nx >> l, sy = ny >> l, sz = nz >> l;
        const u32 hx = sx / 2, hy = sy / 2, hz = sz / 2;
        for (u32 bi = 1; bi < 8; ++bi) {
            const u32 x = bi % 2, y = (bi / 2) % 2, z = bi / 4;
            const float* src = coef[l] + u64(z) * hz * sx * sy + u64(y) * hy * sx + u64(x) * hx;
            SectionTimer t(I, "pipe.quantize", st);
            rc = cc_quantize_to_symbols(syms + vs.level[l] + (bi - 1) * vs.band[l], 2, src, hx, hy, hz,
                                        q0 / float(1u << l), sx, sx * sy, 0, st);
            if (rc) return rc;
        }
    }
    return encodeVolumeSymbols(I, syms, vs, L, rleOnly, dWords, cap, bitSize, what);
}

int decompressVolumeFloat(cc_instance* I, const cc_volume_channel* ch, u32 count, u32 nx, u32 ny, u32 nz, u32 L,
                          bool rleOnly, const char* what) {
    if (!I || !ch || count == 0) { setError("%s: bad argument", what); return CC_ERR_INVALID_ARGUMENT; }
    for (u32 c = 0; c < count; ++c)
        if (!ch[c].d_volume || !ch[c].d_words) { setError("%s: channel %u: null pointer", what, c); return CC_ERR_INVALID_ARGUMENT; }
    if (!volumeSizesOk(nx, ny, nz, L, what)) return CC_ERR_INVALID_ARGUMENT;
    if (I->symBytes != 2) { setError("%s: needs a 16-bit-symbol instance", what); return CC_ERR_INVALID_ARGUMENT; }
    DeviceGuard deviceGuard(I->device);
    if (!rleOnly) {
        const int rc = decompressVolumeFloatBatched(I, ch, count, nx, ny, nz, L, what);
        if (rc != kNoBatch) return rc;
    }
    cudaStream_t st = I->stream;
    const u64 N0 = cube(nx, ny, nz);
    const VolumeSymbols vs = volumeSymbols(nx, ny, nz, L);
    Bump b{nullptr};
    b.take<float>(N0);
    b.take<float>(N0);
    b.take<float>(N0);
    b.take<u16>(vs.total * count + 1024);
    b.take<void*>(8 * L);
    int rc = ensurePipelineWork(I, b.off + 1024);
    if (rc) return rc;
    Bump w{I->pipeWork};
    float* t1 = w.take<float>(N0);
    float* t2 = w.take<float>(N0);
    float* cur = w.take<float>(N0);
    u16* syms = w.take<u16>(vs.total * count + 1024);
    void** dPtrs = w.take<void*>(8 * L);
    std::vector<const u32*> words(count);
    std::vector<u32> bits(count);
    for (u32 c = 0; c < count; ++c) { words[c] = ch[c].d_words; bits[c] = ch[c].bit_size; }
    if ((rc = decodeVolumeSymbols(I, words.data(), bits.data(), count, L, rleOnly, vs, syms, what))) return rc;
    std::vector<void*> hostPtrs(8 * L);
    for (u32 c = 0; c < count; ++c) {
        const u16* s = syms + c * vs.total;
        const float q0 = ch[c].quant_step;
        for (u32 l = 0; l < L; ++l)
            for (u32 i = 0; i < 7; ++i) hostPtrs[l * 8 + i] = const_cast<u16*>(s + vs.level[l] + i * vs.band[l]);
        CC_TRY_CUDA(cudaMemcpyAsync(dPtrs, hostPtrs.data(), hostPtrs.size() * sizeof(void*), cudaMemcpyHostToDevice, st),
                    "upload band pointers");
        rc = cc_unquantize_from_symbols(cur, s, 2, nx >> L, ny >> L, nz >> L, q0 / float(1u << (L - 1)), 0, 0, 0, st);
        if (rc) return rc;
        // level l: lowpass `cur` (dense) + 7 bands -> dense level volume, written
        // back over `cur` (the first pass has consumed it by then) or into the output
        for (int l = int(L) - 1; l >= 0; --l) {
            const int sx = int(nx >> l), sy = int(ny >> l), sz = int(nz >> l);
            SectionTimer tInv(I, "pipe.dwt_inverse", st);
            rc = cc_dwt_float_inverse_from_symbols(l == 0 ? ch[c].d_volume : cur, t2, t1, cur, dPtrs + l * 8, 2,
                                                   q0 / float(1u << l), sx, sy, sz, 1, 0, 0, sx / 2,
                                                   (sx / 2) * (sy / 2), st);
            if (rc) return rc;
        }
    }
    CC_TRY_CUDA(cudaStreamSynchronize(st), what);
    return cc_decode_status(I);
}

// ---- quant-first codec ----
int compressVolumeQuantFirst(cc_instance* I, const float* vol, u32 nx, u32 ny, u32 nz, u32 L, float step,
                             bool rleOnly, u32* dWords, u64 cap, u32* bitSize) {
    const char* what = "compressVolumeFloatQuantFirst";
    if (!I || !vol || !dWords || !bitSize) { setError("%s: bad argument", what); return CC_ERR_INVALID_ARGUMENT; }
    if (!volumeSizesOk(nx, ny, nz, L, what)) return CC_ERR_INVALID_ARGUMENT;
    if (I->symBytes != 2) { setError("%s: needs a 16-bit-symbol instance", what); return CC_ERR_INVALID_ARGUMENT; }
    const u64 band0 = cube(nx / 2, ny / 2, nz / 2);
    if (I->streamCountMax < 7 || I->elemCountPerStreamMax < band0) {
        setError("%s: instance needs >= 7 streams of >= %llu symbols", what, (unsigned long long)band0);
        return CC_ERR_CAPACITY;
    }
    DeviceGuard deviceGuard(I->device);
    cudaStream_t st = I->stream;
    const u64 N0 = cube(nx, ny, nz);
    const VolumeSymbols vs = volumeSymbols(nx, ny, nz, L);
    Bump b{nullptr};
    b.take<i16>(N0);
    b.take<i16>(N0);
    for (u32 l = 0; l < L; ++l) b.take<i16>(cube(nx >> l, ny >> l, nz >> l));
    b.take<u16>(vs.total + 1024);
    int rc = ensurePipelineWork(I, b.off + 1024);
    if (rc) return rc;
    Bump w{I->pipeWork};
    i16* q = w.take<i16>(N0);
    i16* buf = w.take<i16>(N0);
    std::vector<i16*> coef(L);
    for (u32 l = 0; l < L; ++l) coef[l] = w.take<i16>(cube(nx >> l, ny >> l, nz >> l));
    u16* syms = w.take<u16>(vs.total + 1024);
    // uniform quantization (quantizeToShort, QUANTIZE_UNIFORM), then the integer DWT level by level
    if ((rc = cc_quantize_to_short(q, vol, nx, ny, nz, step, 0, 0, 1, st))) return rc;
    for (u32 l = 0; l < L; ++l) {
        const int sx = int(nx >> l), sy = int(ny >> l), sz = int(nz >> l);
        const i16* src = l == 0 ? q : coef[l - 1];
        const int sr = l == 0 ? int(nx) : int(nx >> (l - 1));
        const int ss = l == 0 ? int(nx * ny) : int((nx >> (l - 1)) * (ny >> (l - 1)));
        if ((rc = cc_dwt_int_forward(coef[l], buf, src, sx, sy, sz, sx, sx * sy, sr, ss, st))) return rc;
    }
    // symbolize: LP (the LLL corner of the coarsest level), then levels coarse -> fine, bands 1..7
    const u32 lsx = nx >> (L - 1), lsy = ny >> (L - 1);
    if ((rc = cc_symbolize(syms, coef[L - 1], nx >> L, ny >> L, nz >> L, lsx, lsx * lsy, st))) return rc;
    for (int l = int(L) - 1; l >= 0; --l) {
        const u32 sx = nx >> l, sy = ny >> l, sz = nz >> l;
        const u32 hx = sx / 2, hy = sy / 2, hz = sz / 2;
        for (u32 bi = 1; bi < 8; ++bi) {
            const u32 x = bi % 2, y = (bi / 2) % 2, z = bi / 4;
            const i16* src = coef[l] + u64(z) * hz * sx * sy + u64(y) * hy * sx + u64(x) * hx;
            if ((rc = cc_symbolize(syms + vs.level[l] + (bi - 1) * vs.band[l], src, hx, hy, hz, sx, sx * sy, st)))
                return rc;
        }
    }
    return encodeVolumeSymbols(I, syms, vs, L, rleOnly, dWords, cap, bitSize, what);
}

// The inverse levels run coarse -> fine in every case; each level's inverse
// writes straight into the lowpass corner of the next finer level.  (The
// reference's decoder, CompressVolume.cpp:840-846, starts its inverse from
// buffer numLevels % 2 while the coarsest level's data is in buffer 0, so for
// odd level counts it reads the other buffer; the streams are unaffected.)
int decompressVolumeQuantFirst(cc_instance* I, const cc_volume_channel* ch, u32 count, u32 nx, u32 ny, u32 nz, u32 L,
                               bool rleOnly, const char* what) {
    if (!I || !ch || count == 0) { setError("%s: bad argument", what); return CC_ERR_INVALID_ARGUMENT; }
    for (u32 c = 0; c < count; ++c)
        if (!ch[c].d_volume || !ch[c].d_words) { setError("%s: channel %u: null pointer", what, c); return CC_ERR_INVALID_ARGUMENT; }
    if (!volumeSizesOk(nx, ny, nz, L, what)) return CC_ERR_INVALID_ARGUMENT;
    if (I->symBytes != 2) { setError("%s: needs a 16-bit-symbol instance", what); return CC_ERR_INVALID_ARGUMENT; }
    DeviceGuard deviceGuard(I->device);
    cudaStream_t st = I->stream;
    const u64 N0 = cube(nx, ny, nz);
    const VolumeSymbols vs = volumeSymbols(nx, ny, nz, L);
    Bump b{nullptr};
    b.take<i16>(N0);
    b.take<i16>(N0);
    for (u32 l = 0; l < L; ++l) b.take<i16>(cube(nx >> l, ny >> l, nz >> l));
    b.take<u16>(vs.total * count + 1024);
    int rc = ensurePipelineWork(I, b.off + 1024);
    if (rc) return rc;
    Bump w{I->pipeWork};
    i16* rec = w.take<i16>(N0);
    i16* buf = w.take<i16>(N0);
    std::vector<i16*> coef(L);
    for (u32 l = 0; l < L; ++l) coef[l] = w.take<i16>(cube(nx >> l, ny >> l, nz >> l));
    u16* syms = w.take<u16>(vs.total * count + 1024);
    std::vector<const u32*> words(count);
    std::vector<u32> bits(count);
    for (u32 c = 0; c < count; ++c) { words[c] = ch[c].d_words; bits[c] = ch[c].bit_size; }
    if ((rc = decodeVolumeSymbols(I, words.data(), bits.data(), count, L, rleOnly, vs, syms, what))) return rc;
    for (u32 c = 0; c < count; ++c) {
        const u16* s = syms + c * vs.total;
        // level L-1's lowpass into its LLL corner
        const u32 lsx = nx >> (L - 1), lsy = ny >> (L - 1);
        if ((rc = cc_unsymbolize(coef[L - 1], s, nx >> L, ny >> L, nz >> L, lsx, lsx * lsy, st))) return rc;
        for (int l = int(L) - 1; l >= 0; --l) {
            // level l's bands go in after the level l+1 inverse: that inverse
            // (dwtIntInverse, DWTInt.cu:222-229) uses the first elements of its
            // destination - this level's array - as scratch with its own pitches
            const u32 sx = nx >> l, sy = ny >> l, sz = nz >> l;
            const u32 hx = sx / 2, hy = sy / 2, hz = sz / 2;
            for (u32 bi = 1; bi < 8; ++bi) {
                const u32 x = bi % 2, y = (bi / 2) % 2, z = bi / 4;
                i16* dst = coef[l] + u64(z) * hz * sx * sy + u64(y) * hy * sx + u64(x) * hx;
                if ((rc = cc_unsymbolize(dst, s + vs.level[l] + (bi - 1) * vs.band[l], hx, hy, hz, sx, sx * sy, st)))
                    return rc;
            }
            i16* dst = l == 0 ? rec : coef[l - 1];
            const int dr = l == 0 ? int(nx) : int(nx >> (l - 1));
            const int ds = l == 0 ? int(nx * ny) : int((nx >> (l - 1)) * (ny >> (l - 1)));
            if ((rc = cc_dwt_int_inverse(dst, buf, coef[l], int(sx), int(sy), int(sz), dr, ds, int(sx), int(sx * sy), st)))
                return rc;
        }
        if ((rc = cc_unquantize_from_short(ch[c].d_volume, rec, nx, ny, nz, ch[c].quant_step, 0, 0, 1, st))) return rc;
    }
    CC_TRY_CUDA(cudaStreamSynchronize(st), what);
    return cc_decode_status(I);
}

}  // namespace
}  // namespace ccb

using namespace ccb;

extern "C" {

int cc_compress_volume_float(cc_instance* I, const float* vol, uint32_t nx, uint32_t ny, uint32_t nz, uint32_t levels,
                             float q0, uint32_t* dWords, uint64_t cap, uint32_t* bitSize) {
    return compressVolumeFloat(I, vol, nx, ny, nz, levels, q0, false, dWords, cap, bitSize);
}

int cc_compress_volume_float_ex(cc_instance* I, const float* vol, uint32_t nx, uint32_t ny, uint32_t nz,
                                uint32_t levels, float q0, uint32_t flags, uint32_t* dWords, uint64_t cap,
                                uint32_t* bitSize) {
    if (flags & ~uint32_t(CC_VOLUME_RLE_ONLY_LEVEL0)) { setError("compressVolumeFloat: unknown flags 0x%x", flags); return CC_ERR_INVALID_ARGUMENT; }
    return compressVolumeFloat(I, vol, nx, ny, nz, levels, q0, flags & CC_VOLUME_RLE_ONLY_LEVEL0, dWords, cap, bitSize);
}

int cc_decompress_volume_float(cc_instance* I, float* out, uint32_t nx, uint32_t ny, uint32_t nz, uint32_t levels,
                               float q0, const uint32_t* dWords, uint32_t bitSize) {
    const cc_volume_channel ch{out, dWords, bitSize, q0};
    return decompressVolumeFloat(I, &ch, 1, nx, ny, nz, levels, false, "decompressVolumeFloat");
}

int cc_decompress_volume_float_ex(cc_instance* I, float* out, uint32_t nx, uint32_t ny, uint32_t nz,
                                  uint32_t levels, float q0, uint32_t flags, const uint32_t* dWords,
                                  uint32_t bitSize) {
    if (flags & ~uint32_t(CC_VOLUME_RLE_ONLY_LEVEL0)) { setError("decompressVolumeFloat: unknown flags 0x%x", flags); return CC_ERR_INVALID_ARGUMENT; }
    const cc_volume_channel ch{out, dWords, bitSize, q0};
    return decompressVolumeFloat(I, &ch, 1, nx, ny, nz, levels, flags & CC_VOLUME_RLE_ONLY_LEVEL0,
                                 "decompressVolumeFloat");
}

int cc_decompress_volume_float_multichannel(cc_instance* I, const cc_volume_channel* channels, uint32_t count,
                                            uint32_t nx, uint32_t ny, uint32_t nz, uint32_t levels, uint32_t flags) {
    if (flags & ~uint32_t(CC_VOLUME_RLE_ONLY_LEVEL0)) { setError("decompressVolumeFloatMultiChannel: unknown flags 0x%x", flags); return CC_ERR_INVALID_ARGUMENT; }
    return decompressVolumeFloat(I, channels, count, nx, ny, nz, levels, flags & CC_VOLUME_RLE_ONLY_LEVEL0,
                                 "decompressVolumeFloatMultiChannel");
}

int cc_compress_volume_float_quant_first(cc_instance* I, const float* vol, uint32_t nx, uint32_t ny, uint32_t nz,
                                         uint32_t levels, float step, uint32_t flags, uint32_t* dWords,
                                         uint64_t cap, uint32_t* bitSize) {
    if (flags & ~uint32_t(CC_VOLUME_RLE_ONLY_LEVEL0)) { setError("compressVolumeFloatQuantFirst: unknown flags 0x%x", flags); return CC_ERR_INVALID_ARGUMENT; }
    return compressVolumeQuantFirst(I, vol, nx, ny, nz, levels, step, flags & CC_VOLUME_RLE_ONLY_LEVEL0, dWords, cap,
                                    bitSize);
}

int cc_decompress_volume_float_quant_first(cc_instance* I, float* out, uint32_t nx, uint32_t ny, uint32_t nz,
                                           uint32_t levels, float step, uint32_t flags, const uint32_t* dWords,
                                           uint32_t bitSize) {
    if (flags & ~uint32_t(CC_VOLUME_RLE_ONLY_LEVEL0)) { setError("decompressVolumeFloatQuantFirst: unknown flags 0x%x", flags); return CC_ERR_INVALID_ARGUMENT; }
    const cc_volume_channel ch{out, dWords, bitSize, step};
    return decompressVolumeQuantFirst(I, &ch, 1, nx, ny, nz, levels, flags & CC_VOLUME_RLE_ONLY_LEVEL0,
                                      "decompressVolumeFloatQuantFirst");
}

int cc_decompress_volume_float_quant_first_multichannel(cc_instance* I, const cc_volume_channel* channels,
                                                        uint32_t count, uint32_t nx, uint32_t ny, uint32_t nz,
                                                        uint32_t levels, uint32_t flags) {
    if (flags & ~uint32_t(CC_VOLUME_RLE_ONLY_LEVEL0)) { setError("decompressVolumeFloatQuantFirstMultiChannel: unknown flags 0x%x", flags); return CC_ERR_INVALID_ARGUMENT; }
    return decompressVolumeQuantFirst(I, channels, count, nx, ny, nz, levels, flags & CC_VOLUME_RLE_ONLY_LEVEL0,
                                      "decompressVolumeFloatQuantFirstMultiChannel");
}

int cc_compress_heightfield(cc_instance* I, const int16_t* img, uint32_t nx, uint32_t ny, uint32_t levels,
                            uint32_t* dWords, uint64_t cap, uint32_t* bitSize) {
    if (!I || !img || !dWords || !bitSize || levels == 0) { setError("compressHeightfield: bad argument"); return CC_ERR_INVALID_ARGUMENT; }
    const u32 f = 1u << levels;
    if (nx % f || ny % f || (nx >> (levels - 1)) < 8 || (ny >> (levels - 1)) < 8) {
        setError("compressHeightfield: sizes must be divisible by 2^levels with coarsest level >= 8");
        return CC_ERR_INVALID_ARGUMENT;
    }
    if (I->symBytes != 2) { setError("compressHeightfield: needs a 16-bit-symbol instance"); return CC_ERR_INVALID_ARGUMENT; }
    const u64 band0 = u64(nx / 2) * (ny / 2);
    if (I->streamCountMax < 3 || I->elemCountPerStreamMax < band0) {
        setError("compressHeightfield: instance needs >= 3 streams of >= %llu symbols", (unsigned long long)band0);
        return CC_ERR_CAPACITY;
    }
    DeviceGuard deviceGuard(I->device);
    cudaStream_t st = I->stream;
    const u64 N0 = u64(nx) * ny;
    Bump b{nullptr};
    b.take<i16>(N0);
    b.take<i16>(N0);
    b.take<i16>(N0);
    b.take<u16>(N0 + 1024);
    int rc = ensurePipelineWork(I, b.off + 1024);
    if (rc) return rc;
    Bump w{I->pipeWork};
    i16* coefA = w.take<i16>(N0);
    i16* coefB = w.take<i16>(N0);
    i16* tmp = w.take<i16>(N0);
    u16* syms = w.take<u16>(N0 + 1024);
    // level l: transform the (dense) lowpass of level l-1
    std::vector<i16*> coef(levels);
    const i16* src = img;
    u16* next = syms;
    std::vector<std::vector<u16*>> bands(levels, std::vector<u16*>(3));
    for (u32 l = 0; l < levels; ++l) {
        const u32 sx = nx >> l, sy = ny >> l;
        i16* dst = (l % 2 == 0) ? coefA : coefB;
        rc = cc_dwt_int_forward(dst, tmp, src, int(sx), int(sy), 1, 0, 0, int(l == 0 ? nx : (nx >> (l - 1))), 0, st);
        if (rc) return rc;
        const u32 hx = sx / 2, hy = sy / 2;
        for (u32 bi = 1; bi < 4; ++bi) {
            const u32 x = bi % 2, y = bi / 2;
            rc = cc_symbolize(next, dst + u64(y) * hy * sx + u64(x) * hx, hx, hy, 1, sx, 0, st);
            if (rc) return rc;
            bands[l][bi - 1] = next;
            next += u64(hx) * hy;
        }
        coef[l] = dst;
        src = dst;   // LL corner, row pitch sx (passed above as the next level's source pitch)
    }
    const u32 L = levels;
    const u32 lx = nx >> L, ly = ny >> L;
    u16* lp = next;
    rc = cc_symbolize(lp, coef[L - 1], lx, ly, 1, nx >> (L - 1), 0, st);
    if (rc) return rc;
    std::vector<EncStream> es;
    std::vector<EncGroup> groups;
    es.push_back(EncStream{lp, lx * ly, 0, 0, 1, KIND_HUFF});
    groups.push_back(EncGroup{0, 1});
    for (int l = int(L) - 1; l >= 0; --l) {
        const u32 n = (nx >> (l + 1)) * (ny >> (l + 1));
        const u32 first = u32(es.size());
        for (u32 i = 0; i < 3; ++i) es.push_back(EncStream{bands[l][i], n, 0, first, 3, KIND_RLHUFF});
        groups.push_back(EncGroup{first, 3});
    }
    u64 at = 0;
    if ((rc = encodeGroups(I, es, groups, dWords, cap, &at))) return rc;
    CC_TRY_CUDA(cudaStreamSynchronize(st), "compressHeightfield");
    if (at * 32 > 0xffffffffull) { setError("compressHeightfield: stream exceeds 2^32 bits"); return CC_ERR_CAPACITY; }
    *bitSize = u32(at * 32);
    return CC_OK;
}

// The heightfield decode one level at a time with a host walk of the stream:
// for instances too small to decode every level in one call.
static int decompressHeightfieldPerLevel(cc_instance* I, int16_t* out, uint32_t nx, uint32_t ny, uint32_t levels,
                                         const uint32_t* dWords, uint32_t bitSize) {
    if (!I || !out || !dWords || levels == 0) { setError("decompressHeightfield: bad argument"); return CC_ERR_INVALID_ARGUMENT; }
    if (I->symBytes != 2) { setError("decompressHeightfield: needs a 16-bit-symbol instance"); return CC_ERR_INVALID_ARGUMENT; }
    DeviceGuard deviceGuard(I->device);
    cudaStream_t st = I->stream;
    const u64 words = ceilDiv(bitSize, 32);
    if (words > I->hostWordsMax) { setError("decompressHeightfield: stream larger than instance staging"); return CC_ERR_CAPACITY; }
    const u64 N0 = u64(nx) * ny;
    Bump b{nullptr};
    b.take<i16>(N0);
    b.take<i16>(N0);
    b.take<i16>(N0);
    b.take<u16>(N0 + 1024);
    int rc = ensurePipelineWork(I, b.off + 1024);
    if (rc) return rc;
    Bump w{I->pipeWork};
    i16* cur = w.take<i16>(N0);
    i16* coef = w.take<i16>(N0);
    i16* tmp = w.take<i16>(N0);
    u16* syms = w.take<u16>(N0 + 1024);
    CC_TRY_CUDA(cudaMemcpyAsync(I->hostWords, dWords, words * 4, cudaMemcpyDeviceToHost, st), "download stream");
    CC_TRY_CUDA(cudaStreamSynchronize(st), "download stream");
    std::vector<u32> host(I->hostWords, I->hostWords + words);
    const u32* hw = host.data();
    u32 pos = 0;
    const u32 L = levels;
    const u32 lx = nx >> L, ly = ny >> L;
    void* outs[3] = {syms};
    if ((rc = decodeDevice(I, KIND_HUFF, &hw, &bitSize, &pos, 1, nullptr, outs, 1, lx * ly))) return rc;
    pos = u32(alignUp(pos, 32));
    rc = cc_unsymbolize(cur, syms, lx, ly, 1, 0, 0, st);
    if (rc) return rc;
    for (int l = int(L) - 1; l >= 0; --l) {
        const u32 sx = nx >> l, sy = ny >> l, hx = sx / 2, hy = sy / 2;
        const u64 bandN = u64(hx) * hy;
        for (u32 i = 0; i < 3; ++i) outs[i] = syms + i * bandN;
        if ((rc = decodeDevice(I, KIND_RLHUFF, &hw, &bitSize, &pos, 1, nullptr, outs, 3, u32(bandN)))) return rc;
        pos = u32(alignUp(pos, 32));
        // assemble [LL | HL ; LH | HH] of this level then invert
        CC_TRY_CUDA(cudaMemcpy2DAsync(coef, sx * sizeof(i16), cur, hx * sizeof(i16), hx * sizeof(i16), hy,
                                      cudaMemcpyDeviceToDevice, st), "place lowpass");
        for (u32 bi = 1; bi < 4; ++bi) {
            const u32 x = bi % 2, y = bi / 2;
            rc = cc_unsymbolize(coef + u64(y) * hy * sx + u64(x) * hx, static_cast<u16*>(outs[bi - 1]), hx, hy, 1, sx, 0, st);
            if (rc) return rc;
        }
        rc = cc_dwt_int_inverse(l == 0 ? out : cur, tmp, coef, int(sx), int(sy), 1, 0, 0, 0, 0, st);
        if (rc) return rc;
    }
    CC_TRY_CUDA(cudaStreamSynchronize(st), "decompressHeightfield");
    return cc_decode_status(I);
}

int cc_decompress_heightfield(cc_instance* I, int16_t* out, uint32_t nx, uint32_t ny, uint32_t levels,
                              const uint32_t* dWords, uint32_t bitSize) {
    if (!I || !out || !dWords || levels == 0) { setError("decompressHeightfield: bad argument"); return CC_ERR_INVALID_ARGUMENT; }
    if (I->symBytes != 2) { setError("decompressHeightfield: needs a 16-bit-symbol instance"); return CC_ERR_INVALID_ARGUMENT; }
    const u32 f = 1u << levels;
    if (nx % f || ny % f || (nx >> (levels - 1)) < 8 || (ny >> (levels - 1)) < 8) {
        setError("decompressHeightfield: sizes must be divisible by 2^levels with coarsest level >= 8");
        return CC_ERR_INVALID_ARGUMENT;
    }
    DeviceGuard deviceGuard(I->device);
    cudaStream_t st = I->stream;
    const u64 N0 = u64(nx) * ny;
    Bump b{nullptr};
    b.take<i16>(N0);
    b.take<i16>(N0);
    b.take<i16>(N0);
    b.take<u16>(N0 + 1024);
    int rc = ensurePipelineWork(I, b.off + 1024);
    if (rc) return rc;
    Bump w{I->pipeWork};
    i16* cur = w.take<i16>(N0);
    i16* coef = w.take<i16>(N0);
    i16* tmp = w.take<i16>(N0);
    u16* syms = w.take<u16>(N0 + 1024);
    // every stream of every level in one device-walked decode: the LP stream
    // (Huff), then per level coarse -> fine its 3 bands (RLHuff); the symbols
    // in the layout LP | level L-1 bands | ... | level 0 bands
    const u32 L = levels;
    const u32 lx = nx >> L, ly = ny >> L;
    std::vector<DecStreamSpec> ds;
    std::vector<u16*> bandAt(L);
    u64 at = u64(lx) * ly;
    ds.push_back(DecStreamSpec{KIND_HUFF, lx * ly, syms, 0});
    for (int l = int(L) - 1; l >= 0; --l) {
        const u64 bandN = u64(nx >> (l + 1)) * (ny >> (l + 1));
        bandAt[l] = syms + at;
        for (u32 i = 0; i < 3; ++i) ds.push_back(DecStreamSpec{KIND_RLHUFF, u32(bandN), syms + at + i * bandN, 0});
        at += 3 * bandN;
    }
    const DecSourceSpec src{dWords, bitSize, 0};
    char* slot = I->takeRingSlot();
    DecPlan dp;
    rc = decodePrepare(I, ds.data(), u32(ds.size()), &src, 1, slot, I->hostRingBytes, dp);
    if (rc == CC_ERR_CAPACITY) return decompressHeightfieldPerLevel(I, out, nx, ny, levels, dWords, bitSize);
    if (rc) return rc;
    dp.dev = I->dPlan;
    CC_TRY_CUDA(cudaMemcpyAsync(I->dPlan, slot, dp.bytes, cudaMemcpyHostToDevice, st), "upload plan");
    cudaEventRecord(I->ringEvent[(I->ringNext + cc_instance::kRing - 1) % cc_instance::kRing], st);
    if ((rc = decodeLaunch(I, dp))) return rc;
    rc = cc_unsymbolize(cur, syms, lx, ly, 1, 0, 0, st);
    if (rc) return rc;
    for (int l = int(L) - 1; l >= 0; --l) {
        const u32 sx = nx >> l, sy = ny >> l, hx = sx / 2, hy = sy / 2;
        const u64 bandN = u64(hx) * hy;
        // assemble [LL | HL ; LH | HH] of this level then invert
        CC_TRY_CUDA(cudaMemcpy2DAsync(coef, sx * sizeof(i16), cur, hx * sizeof(i16), hx * sizeof(i16), hy,
                                      cudaMemcpyDeviceToDevice, st), "place lowpass");
        for (u32 bi = 1; bi < 4; ++bi) {
            const u32 x = bi % 2, y = bi / 2;
            rc = cc_unsymbolize(coef + u64(y) * hy * sx + u64(x) * hx, bandAt[l] + (bi - 1) * bandN, hx, hy, 1, sx, 0, st);
            if (rc) return rc;
        }
        rc = cc_dwt_int_inverse(l == 0 ? out : cur, tmp, coef, int(sx), int(sy), 1, 0, 0, 0, 0, st);
        if (rc) return rc;
    }
    CC_TRY_CUDA(cudaStreamSynchronize(st), "decompressHeightfield");
    return cc_decode_status(I);
}

}  // extern "C"
