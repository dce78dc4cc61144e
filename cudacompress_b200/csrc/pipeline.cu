// pipeline.cu - whole-codec entry points: the lossy volume codec
// (examples CompressVolume.cpp:312-516) and the lossless 2D heightfield codec
// (one level = CompressHeightfield.cpp:82-216 band layout, levels chained as
// compressVolumeLossless, CompressVolume.cpp:234-309).  Device-resident input
// and device-resident 32-bit-word bit stream.
//
// Volume stream: LP band (step q0/2^(L-1)) encodeHuff, then for level
// L-1 .. 0 the 7 highpass bands (index x+2y+4z, step q0/2^level) encodeRLHuff.
// Heightfield stream: LP encodeHuff, then levels L-1 .. 0, 3 bands each
// (index x+2y) encodeRLHuff, every level starting word aligned.
#include <cstring>

#include "capi_internal.cuh"

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

// One reference encode call of a pipeline: `count` streams from `first`.
struct EncGroup {
    u32 first, count;
};

// Encodes the groups back to back into dWords (word aligned segments; the
// reference's BitStream is word aligned at every group start here), batching
// as many groups per device call as the instance's symbol and stream budget
// allows.  A batch whose histograms exceed the instance's table capacity is
// redone one group per call (the capacity every instance guarantees).
static int encodeGroups(cc_instance* I, const std::vector<EncStream>& streams, const std::vector<EncGroup>& groups,
                        u32* dWords, u64 cap, u64* wordsOut) {
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
                at += words;
            }
        } else if (rc) {
            return rc;
        } else {
            at += words;
        }
        g = h;
    }
    *wordsOut = at;
    return CC_OK;
}

}  // namespace ccb

using namespace ccb;

extern "C" {

int cc_compress_volume_float(cc_instance* I, const float* vol, uint32_t nx, uint32_t ny, uint32_t nz, uint32_t levels,
                             float q0, uint32_t* dWords, uint64_t cap, uint32_t* bitSize) {
    if (!I || !vol || !dWords || !bitSize || levels == 0) { setError("compressVolumeFloat: bad argument"); return CC_ERR_INVALID_ARGUMENT; }
    const u32 f = 1u << levels;
    if (nx % f || ny % f || nz % f || (nx >> (levels - 1)) < 8 || (ny >> (levels - 1)) < 8 || (nz >> (levels - 1)) < 8) {
        setError("compressVolumeFloat: sizes must be divisible by 2^levels with coarsest level >= 8");
        return CC_ERR_INVALID_ARGUMENT;
    }
    if (I->symBytes != 2) { setError("compressVolumeFloat: needs a 16-bit-symbol instance"); return CC_ERR_INVALID_ARGUMENT; }
    const u64 band0 = cube(nx / 2, ny / 2, nz / 2);
    if (I->streamCountMax < 7 || I->elemCountPerStreamMax < band0) {
        setError("compressVolumeFloat: instance needs >= 7 streams of >= %llu symbols", (unsigned long long)band0);
        return CC_ERR_CAPACITY;
    }
    cudaSetDevice(I->device);
    cudaStream_t st = I->stream;
    const u64 N0 = cube(nx, ny, nz);
    // workspace: two DWT buffers, per-level coefficients, symbols
    Bump b{nullptr};
    b.take<float>(N0);
    b.take<float>(N0);
    for (u32 l = 0; l < levels; ++l) b.take<float>(cube(nx >> l, ny >> l, nz >> l));
    b.take<u16>(N0 + 1024);
    int rc = ensurePipelineWork(I, b.off + 1024);
    if (rc) return rc;
    Bump w{I->pipeWork};
    float* t1 = w.take<float>(N0);
    float* t2 = w.take<float>(N0);
    std::vector<float*> coef(levels);
    for (u32 l = 0; l < levels; ++l) coef[l] = w.take<float>(cube(nx >> l, ny >> l, nz >> l));
    u16* syms = w.take<u16>(N0 + 1024);
    // forward transforms: level l reads the LLL corner of level l-1
    for (u32 l = 0; l < levels; ++l) {
        const int sx = int(nx >> l), sy = int(ny >> l), sz = int(nz >> l);
        const float* src = l == 0 ? vol : coef[l - 1];
        const int sr = l == 0 ? 0 : int(nx >> (l - 1));
        const int ss = l == 0 ? 0 : int((nx >> (l - 1)) * (ny >> (l - 1)));
        { SectionTimer t(I, "pipe.dwt_forward", st); rc = cc_dwt_float_forward(coef[l], t2, t1, src, sx, sy, sz, 1, 0, 0, sr, ss, st); }
        if (rc) return rc;
    }
    // quantize: LP then levels coarse -> fine, bands 1..7
    const u32 L = levels;
    const u32 lx = nx >> L, ly = ny >> L, lz = nz >> L;
    u16* lp = syms;
    rc = cc_quantize_to_symbols(lp, 2, coef[L - 1], lx, ly, lz, q0 / float(1u << (L - 1)), nx >> (L - 1),
                                (nx >> (L - 1)) * (ny >> (L - 1)), 0, st);
    if (rc) return rc;
    u16* next = lp + cube(lx, ly, lz);
    std::vector<std::vector<u16*>> bands(L, std::vector<u16*>(7));
    for (int l = int(L) - 1; l >= 0; --l) {
        const u32 sx = nx >> l, sy = ny >> l, sz = nz >> l;
        const u32 hx = sx / 2, hy = sy / 2, hz = sz / 2;
        const float step = q0 / float(1u << l);
        for (u32 bi = 1; bi < 8; ++bi) {
            const u32 x = bi % 2, y = (bi / 2) % 2, z = bi / 4;
            const float* src = coef[l] + u64(z) * hz * sx * sy + u64(y) * hy * sx + u64(x) * hx;
            { SectionTimer t(I, "pipe.quantize", st); rc = cc_quantize_to_symbols(next, 2, src, hx, hy, hz, step, sx, sx * sy, 0, st); }
            if (rc) return rc;
            bands[l][bi - 1] = next;
            next += cube(hx, hy, hz);
        }
    }
    // entropy coding in stream order: LP (encodeHuff), then levels coarse -> fine (encodeRLHuff of 7 bands)
    std::vector<EncStream> es;
    std::vector<EncGroup> groups;
    es.push_back(EncStream{lp, u32(cube(lx, ly, lz)), 0, 0, 1, KIND_HUFF});
    groups.push_back(EncGroup{0, 1});
    for (int l = int(L) - 1; l >= 0; --l) {
        const u32 first = u32(es.size());
        for (u32 i = 0; i < 7; ++i)
            es.push_back(EncStream{bands[l][i], u32(cube(nx >> (l + 1), ny >> (l + 1), nz >> (l + 1))), 0, first, 7, KIND_RLHUFF});
        groups.push_back(EncGroup{first, 7});
    }
    u64 at = 0;
    if ((rc = encodeGroups(I, es, groups, dWords, cap, &at))) return rc;
    CC_TRY_CUDA(cudaStreamSynchronize(st), "compressVolumeFloat");
    if (at * 32 > 0xffffffffull) { setError("compressVolumeFloat: stream exceeds 2^32 bits"); return CC_ERR_CAPACITY; }
    *bitSize = u32(at * 32);
    return CC_OK;
}

int cc_decompress_volume_float(cc_instance* I, float* out, uint32_t nx, uint32_t ny, uint32_t nz, uint32_t levels,
                               float q0, const uint32_t* dWords, uint32_t bitSize) {
    if (!I || !out || !dWords || levels == 0) { setError("decompressVolumeFloat: bad argument"); return CC_ERR_INVALID_ARGUMENT; }
    const u32 f = 1u << levels;
    if (nx % f || ny % f || nz % f) { setError("decompressVolumeFloat: sizes must be divisible by 2^levels"); return CC_ERR_INVALID_ARGUMENT; }
    if (I->symBytes != 2) { setError("decompressVolumeFloat: needs a 16-bit-symbol instance"); return CC_ERR_INVALID_ARGUMENT; }
    cudaSetDevice(I->device);
    cudaStream_t st = I->stream;
    const u64 words = ceilDiv(bitSize, 32);
    if (words > I->hostWordsMax) { setError("decompressVolumeFloat: stream larger than instance staging"); return CC_ERR_CAPACITY; }
    const u64 N0 = cube(nx, ny, nz);
    Bump b{nullptr};
    b.take<float>(N0);
    b.take<float>(N0);
    b.take<float>(N0);
    b.take<u16>(N0 + 1024);
    b.take<void*>(8 * levels);
    int rc = ensurePipelineWork(I, b.off + 1024);
    if (rc) return rc;
    Bump w{I->pipeWork};
    float* t1 = w.take<float>(N0);
    float* t2 = w.take<float>(N0);
    float* cur = w.take<float>(N0);
    u16* syms = w.take<u16>(N0 + 1024);
    void** dPtrs = w.take<void*>(8 * levels);
    // the bit stream walk happens on the host
    CC_TRY_CUDA(cudaMemcpyAsync(I->hostWords, dWords, words * 4, cudaMemcpyDeviceToHost, st), "download stream");
    CC_TRY_CUDA(cudaStreamSynchronize(st), "download stream");
    std::vector<u32> host(I->hostWords, I->hostWords + words);
    const u32* hw = host.data();
    u32 pos = 0;
    const u32 L = levels;
    const u32 lx = nx >> L, ly = ny >> L, lz = nz >> L;
    u16* lp = syms;
    void* outs[7] = {lp};
    if ((rc = decodeDevice(I, KIND_HUFF, &hw, &bitSize, &pos, 1, nullptr, outs, 1, u32(cube(lx, ly, lz))))) return rc;
    pos = u32(alignUp(pos, 32));
    rc = cc_unquantize_from_symbols(cur, lp, 2, lx, ly, lz, q0 / float(1u << (L - 1)), 0, 0, 0, st);
    if (rc) return rc;
    u16* next = lp + cube(lx, ly, lz);
    std::vector<void*> hostPtrs(8 * L);
    for (int l = int(L) - 1; l >= 0; --l) {
        const u32 hx = nx >> (l + 1), hy = ny >> (l + 1), hz = nz >> (l + 1);
        const u64 bandN = cube(hx, hy, hz);
        for (u32 i = 0; i < 7; ++i) outs[i] = next + i * bandN;
        CC_TRY_CUDA(cudaMemsetAsync(next, 0, 7 * bandN * sizeof(u16), st), "zero bands");
        if ((rc = decodeDevice(I, KIND_RLHUFF, &hw, &bitSize, &pos, 1, nullptr, outs, 7, u32(bandN)))) return rc;
        for (u32 i = 0; i < 7; ++i) hostPtrs[l * 8 + i] = outs[i];
        next += 7 * bandN;
    }
    CC_TRY_CUDA(cudaMemcpyAsync(dPtrs, hostPtrs.data(), hostPtrs.size() * sizeof(void*), cudaMemcpyHostToDevice, st), "upload band pointers");
    // level l: lowpass `cur` (dense) + 7 bands -> dense level volume, written
    // back over `cur` (the first pass has consumed it by then) or into `out`
    for (int l = int(L) - 1; l >= 0; --l) {
        const int sx = int(nx >> l), sy = int(ny >> l), sz = int(nz >> l);
        SectionTimer tInv(I, "pipe.dwt_inverse", st);
        rc = cc_dwt_float_inverse_from_symbols(l == 0 ? out : cur, t2, t1, cur, dPtrs + l * 8, 2, q0 / float(1u << l),
                                               sx, sy, sz, 1, 0, 0, sx / 2, (sx / 2) * (sy / 2), st);
        if (rc) return rc;
    }
    CC_TRY_CUDA(cudaStreamSynchronize(st), "decompressVolumeFloat");
    return cc_decode_status(I);
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
    cudaSetDevice(I->device);
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

int cc_decompress_heightfield(cc_instance* I, int16_t* out, uint32_t nx, uint32_t ny, uint32_t levels,
                              const uint32_t* dWords, uint32_t bitSize) {
    if (!I || !out || !dWords || levels == 0) { setError("decompressHeightfield: bad argument"); return CC_ERR_INVALID_ARGUMENT; }
    if (I->symBytes != 2) { setError("decompressHeightfield: needs a 16-bit-symbol instance"); return CC_ERR_INVALID_ARGUMENT; }
    cudaSetDevice(I->device);
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
        CC_TRY_CUDA(cudaMemsetAsync(syms, 0, 3 * bandN * sizeof(u16), st), "zero bands");
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

}  // extern "C"
