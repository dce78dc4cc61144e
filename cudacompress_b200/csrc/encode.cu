// encode.cu - device entropy encoder: zero-run RLE, histograms, Huffman table
// construction, codeword packing and bit-stream assembly, all on the GPU.
// Replaces encodeRLHuff / encodeHuff (Encode.cpp:207-471, :648-790) and the
// Tier-0 pieces they call (RunLength.cu:82-188, Histogram.cu:109-289,
// HuffmanTable.cu:385-596, Huffman.cu:73-187, PackInc.cu:210-219).
//
// Launch sequence of one call (no host round trip until the result is read):
//   RLHuff: rleSummary -> rleScan -> rleWrite(+histograms) ->
//   Huff:   histPlain ->
//   both:   tableBuild -> blockBits -> blockScan -> layout -> pack -> headers
#include <cstring>

#include "capi_internal.cuh"
#include "huffman_build.cuh"

namespace ccb {

struct EncParams {
    int kind;
    u32 S;
    u32 cb;
    u32 log2Max;
    u32 bins;
    u32 symBytes;
    const EncStream* streams;
    char* compact;
    char* zc;
    u64 nStride;
    RunSum* tiles;
    TileStart* tileStart;
    u32 tilesMax;
    u32* hist;
    uint2* enc;
    TableMeta* meta;
    u32* headers;
    u32 hdrWordsMax;
    u32* blockBits;
    u32* blockOff;
    u32 blocksMax;
    SegmentLayout* layout;
    u32* out;
    u64 outWordsMax;
    u32* counts;
    u32* errors;
    u64* totals;
    u64* leafWork;
    u32* parentWork;
    u32* orderWork;
    u32* leafSymWork;
    u32 leavesMax;
    u32 heapCap;      // leaves that fit the shared-memory heap of tableBuild
};

constexpr u32 kSmemSymBins = 4096;

__device__ __forceinline__ u32 numTables(const EncParams& p) { return p.kind == KIND_RLHUFF ? 2 * p.S : p.S; }

template <class Sym>
__device__ __forceinline__ const Sym* tableInput(const EncParams& p, u32 t, u32& count) {
    if (p.kind == KIND_RLHUFF) {
        u32 s = t < p.S ? t : t - p.S;
        count = p.counts[s];
        return reinterpret_cast<const Sym*>(t < p.S ? p.compact : p.zc) + u64(s) * p.nStride;
    }
    count = p.streams[t].n;
    return reinterpret_cast<const Sym*>(p.streams[t].in);
}

// Loads kRlePerThread symbols starting at `base` (zero beyond n).
template <class Sym>
__device__ __forceinline__ void loadSyms(const Sym* in, u32 base, u32 n, u32 (&v)[kRlePerThread]) {
    const bool vec = ((reinterpret_cast<uintptr_t>(in) & 15u) == 0) && base + kRlePerThread <= n;
    if (vec) {
        if (sizeof(Sym) == 2) {
            uint4 q = *reinterpret_cast<const uint4*>(in + base);
            u32 w[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
            for (int i = 0; i < 4; ++i) { v[2 * i] = w[i] & 0xFFFFu; v[2 * i + 1] = w[i] >> 16; }
        } else {
            uint4 a = *reinterpret_cast<const uint4*>(in + base);
            uint4 b = *reinterpret_cast<const uint4*>(in + base + 4);
            v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w; v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
        }
    } else {
#pragma unroll
        for (u32 i = 0; i < kRlePerThread; ++i) v[i] = (base + i < n) ? u32(in[base + i]) : 0u;
    }
}

__device__ __forceinline__ RunSum shflRun(RunSum r, int delta, bool up) {
    RunSum t;
    if (up) {
        t.cnt = __shfl_up_sync(0xffffffffu, r.cnt, delta);
        t.ext = __shfl_up_sync(0xffffffffu, r.ext, delta);
        t.firstP1 = __shfl_up_sync(0xffffffffu, r.firstP1, delta);
        t.lastP1 = __shfl_up_sync(0xffffffffu, r.lastP1, delta);
    } else {
        t.cnt = __shfl_down_sync(0xffffffffu, r.cnt, delta);
        t.ext = __shfl_down_sync(0xffffffffu, r.ext, delta);
        t.firstP1 = __shfl_down_sync(0xffffffffu, r.firstP1, delta);
        t.lastP1 = __shfl_down_sync(0xffffffffu, r.lastP1, delta);
    }
    return t;
}

// Order-preserving block scan of RunSum (256 threads); returns the exclusive
// prefix of the calling thread; *total receives the block aggregate.
__device__ RunSum blockScanRun(RunSum r, RunSum* smem /*[9]*/, RunSum* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    RunSum inc = r;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        RunSum t = shflRun(inc, o, true);
        if (lane >= o) inc = runCombine(t, inc);
    }
    if (lane == 31) smem[warp] = inc;
    __syncthreads();
    if (threadIdx.x == 0) {
        RunSum acc{0, 0, 0, 0};
        for (int w = 0; w < int(kRleThreads / 32); ++w) {
            RunSum x = smem[w];
            smem[w] = acc;
            acc = runCombine(acc, x);
        }
        smem[8] = acc;
    }
    __syncthreads();
    RunSum exclLane = shflRun(inc, 1, true);
    if (lane == 0) exclLane = RunSum{0, 0, 0, 0};
    RunSum res = runCombine(smem[warp], exclLane);
    if (total) *total = smem[8];
    __syncthreads();
    return res;
}

__device__ __forceinline__ RunSum threadRun(const u32 (&v)[kRlePerThread], u32 base, u32 n) {
    RunSum r{0, 0, 0, 0};
#pragma unroll
    for (u32 i = 0; i < kRlePerThread; ++i) {
        if (base + i < n && v[i] != 0) {
            u32 q = base + i + 1;
            if (r.cnt == 0) r.firstP1 = q;
            else r.ext += (q - r.lastP1 - 1) / 256u;
            r.lastP1 = q;
            r.cnt++;
        }
    }
    return r;
}

// ---------------------------------------------------------------------------
// Run-length encode (RunLength.cu:82-188 semantics: each nonzero symbol with
// the count of zeros before it; runs of 256+ zeros emit (0, 255) entries;
// trailing zeros dropped).
// ---------------------------------------------------------------------------
template <class Sym>
__global__ void __launch_bounds__(kRleThreads) k_rleSummary(EncParams p) {
    __shared__ RunSum smem[9];
    const u32 s = blockIdx.y, tile = blockIdx.x;
    const u32 n = p.streams[s].n;
    if (tile * kRleTile >= n) return;
    const Sym* in = reinterpret_cast<const Sym*>(p.streams[s].in);
    const u32 base = tile * kRleTile + threadIdx.x * kRlePerThread;
    u32 v[kRlePerThread];
    loadSyms(in, base, n, v);
    RunSum r = threadRun(v, base, n), total;
    blockScanRun(r, smem, &total);
    if (threadIdx.x == 0) p.tiles[u64(s) * p.tilesMax + tile] = total;
}

// One block per stream: scans the tile summaries.
__global__ void __launch_bounds__(1024) k_rleScan(EncParams p) {
    __shared__ RunSum warpTot[32];
    __shared__ RunSum carry;
    const u32 s = blockIdx.x;
    const u32 n = p.streams[s].n;
    const u32 tiles = u32(ceilDiv(n, kRleTile));
    RunSum* T = p.tiles + u64(s) * p.tilesMax;
    TileStart* TS = p.tileStart + u64(s) * p.tilesMax;
    if (threadIdx.x == 0) carry = RunSum{0, 0, 0, 0};
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (u32 base = 0; base < tiles; base += 1024) {
        u32 i = base + threadIdx.x;
        RunSum r = i < tiles ? T[i] : RunSum{0, 0, 0, 0};
        RunSum inc = r;
        for (int o = 1; o < 32; o <<= 1) {
            RunSum t = shflRun(inc, o, true);
            if (lane >= o) inc = runCombine(t, inc);
        }
        if (lane == 31) warpTot[warp] = inc;
        __syncthreads();
        if (threadIdx.x == 0) {
            RunSum acc = carry;
            for (int w = 0; w < 32; ++w) {
                RunSum x = warpTot[w];
                warpTot[w] = acc;
                acc = runCombine(acc, x);
            }
            carry = acc;
        }
        __syncthreads();
        RunSum ex = shflRun(inc, 1, true);
        if (lane == 0) ex = RunSum{0, 0, 0, 0};
        RunSum E = runCombine(warpTot[warp], ex);
        if (i < tiles) {
            TileStart ts;
            ts.prevP1 = E.cnt ? E.lastP1 : 0u;
            ts.out = E.cnt ? E.cnt + E.ext + (E.firstP1 - 1u) / 256u : 0u;
            TS[i] = ts;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        RunSum E = carry;
        p.counts[s] = E.cnt ? E.cnt + E.ext + (E.firstP1 - 1u) / 256u : 0u;
    }
}

// Writes the compact symbols and zero counts and accumulates both histograms.
template <class Sym>
__global__ void __launch_bounds__(kRleThreads) k_rleWrite(EncParams p) {
    __shared__ RunSum smem[9];
    __shared__ u32 hSym[kSmemSymBins];
    __shared__ u32 hZc[256];
    __shared__ u32 extraTotal;
    const u32 s = blockIdx.y, tile = blockIdx.x;
    const u32 n = p.streams[s].n;
    if (tile * kRleTile >= n) return;
    const u32 smemBins = min(p.bins, kSmemSymBins);
    for (u32 i = threadIdx.x; i < smemBins; i += kRleThreads) hSym[i] = 0;
    hZc[threadIdx.x] = 0;
    if (threadIdx.x == 0) extraTotal = 0;
    const Sym* in = reinterpret_cast<const Sym*>(p.streams[s].in);
    const u32 base = tile * kRleTile + threadIdx.x * kRlePerThread;
    u32 v[kRlePerThread];
    loadSyms(in, base, n, v);
    RunSum r = threadRun(v, base, n);
    RunSum E = blockScanRun(r, smem, nullptr);   // includes __syncthreads (smem hist zeroed)
    const TileStart ts = p.tileStart[u64(s) * p.tilesMax + tile];
    u32 prevP1 = E.cnt ? E.lastP1 : ts.prevP1;
    u32 outPos = ts.out + (E.cnt ? E.cnt + E.ext + (E.firstP1 - ts.prevP1 - 1u) / 256u : 0u);
    Sym* comp = reinterpret_cast<Sym*>(p.compact) + u64(s) * p.nStride;
    Sym* zcs = reinterpret_cast<Sym*>(p.zc) + u64(s) * p.nStride;
    u32* gSym = p.hist + u64(s) * p.bins;
    u32* gZc = p.hist + u64(p.S + s) * p.bins;
    u32 extras = 0;
    bool rangeErr = false;
#pragma unroll
    for (u32 i = 0; i < kRlePerThread; ++i) {
        const bool nz = base + i < n && v[i] != 0;
        u32 z = 0;
        if (nz) {
            const u32 q = base + i + 1;
            z = q - prevP1 - 1;
            const u32 e = z / 256u;
            for (u32 k = 0; k < e; ++k) {
                comp[outPos] = Sym(0);
                zcs[outPos] = Sym(255);
                ++outPos;
            }
            extras += e;
            comp[outPos] = Sym(v[i]);
            zcs[outPos] = Sym(z & 255u);
            ++outPos;
            prevP1 = q;
        }
        const u32 sym = v[i];
        const bool inRange = sym < p.bins;
        rangeErr |= nz && !inRange;
        const bool toSmem = nz && inRange && sym < smemBins;
        aggregatedIncrement(hSym, toSmem ? sym : 0u, toSmem);
        if (nz && inRange && !toSmem) atomicAdd(gSym + sym, 1u);
        const bool zcOk = (z & 255u) < p.bins;
        rangeErr |= nz && !zcOk;
        aggregatedIncrement(hZc, z & 255u, nz && zcOk);
    }
    if (rangeErr) atomicOr(p.errors, DEV_ERR_SYMBOL_RANGE);
    u32 e = warpSum(extras);
    if ((threadIdx.x & 31) == 0 && e) atomicAdd(&extraTotal, e);
    __syncthreads();
    if (threadIdx.x == 0 && extraTotal) {
        hSym[0] += extraTotal;
        if (p.bins > 255u) hZc[255] += extraTotal;
        else atomicOr(p.errors, DEV_ERR_SYMBOL_RANGE);
    }
    __syncthreads();
    for (u32 i = threadIdx.x; i < smemBins; i += kRleThreads)
        if (hSym[i]) atomicAdd(gSym + i, hSym[i]);
    if (threadIdx.x < p.bins && hZc[threadIdx.x]) atomicAdd(gZc + threadIdx.x, hZc[threadIdx.x]);
}

// encodeHuff histogram (no run-length stage).
template <class Sym>
__global__ void __launch_bounds__(kRleThreads) k_histPlain(EncParams p) {
    __shared__ u32 hSym[kSmemSymBins];
    const u32 s = blockIdx.y, tile = blockIdx.x;
    const u32 n = p.streams[s].n;
    if (tile * kRleTile >= n) return;
    const u32 smemBins = min(p.bins, kSmemSymBins);
    for (u32 i = threadIdx.x; i < smemBins; i += kRleThreads) hSym[i] = 0;
    __syncthreads();
    const Sym* in = reinterpret_cast<const Sym*>(p.streams[s].in);
    const u32 base = tile * kRleTile + threadIdx.x * kRlePerThread;
    u32 v[kRlePerThread];
    loadSyms(in, base, n, v);
    u32* gSym = p.hist + u64(s) * p.bins;
    bool rangeErr = false;
#pragma unroll
    for (u32 i = 0; i < kRlePerThread; ++i) {
        const bool valid = base + i < n;
        const bool inRange = v[i] < p.bins;
        rangeErr |= valid && !inRange;
        const bool toSmem = valid && inRange && v[i] < smemBins;
        aggregatedIncrement(hSym, toSmem ? v[i] : 0u, toSmem);
        if (valid && inRange && !toSmem) atomicAdd(gSym + v[i], 1u);
    }
    if (rangeErr) atomicOr(p.errors, DEV_ERR_SYMBOL_RANGE);
    __syncthreads();
    for (u32 i = threadIdx.x; i < smemBins; i += kRleThreads)
        if (hSym[i]) atomicAdd(gSym + i, hSym[i]);
}

// ---------------------------------------------------------------------------
// Table construction: one block per table.  Leaf gathering, depths, canonical
// codes and serialization are block parallel; the heap merge and the sort
// run in thread 0 with the tie-breaking of huffman_build.cuh.
// ---------------------------------------------------------------------------
constexpr u32 kBuildThreads = 256;

__device__ __forceinline__ void putBits(u32* words, u32 pos, u32 value, u32 count) {
    // MSB-first, count <= 32, words pre-zeroed; atomics because neighbouring
    // fields written by other threads share words.
    if (count == 0) return;
    value &= count == 32 ? 0xffffffffu : ((1u << count) - 1u);
    const u32 w = pos >> 5, b = pos & 31u;
    const int shift = int(32 - b) - int(count);
    if (shift >= 0) {
        atomicOr(words + w, value << shift);
    } else {
        atomicOr(words + w, value >> (-shift));
        atomicOr(words + w + 1, value << (32 + shift));
    }
}

__global__ void __launch_bounds__(kBuildThreads) k_tableBuild(EncParams p) {
    extern __shared__ __align__(16) unsigned char dyn[];
    if (*(volatile u32*)p.errors) return;
    __shared__ u32 sScan[40];
    __shared__ u32 sMax, sL, sMaxLen, sAllEmpty;
    __shared__ u32 lenCount[32], firstIndex[33], firstCode[33];
    const u32 t = blockIdx.x;
    const u32 S = p.S;
    u32 count;
    // every table's input is u16 or u32; only the count is needed here
    if (p.kind == KIND_RLHUFF) count = p.counts[t < S ? t : t - S];
    else count = p.streams[t].n;
    u32* hist = p.hist + u64(t) * p.bins;
    const bool isZc = p.kind == KIND_RLHUFF && t >= S;

    // 1. largest present symbol
    const u32 sIdx = t < S ? t : t - S;
    const EncStream es = p.streams[sIdx];
    if (threadIdx.x == 0) { sMax = 0; sAllEmpty = 1; }
    __syncthreads();
    if (p.kind == KIND_RLHUFF)
        for (u32 s = es.groupFirst + threadIdx.x; s < es.groupFirst + es.groupSize; s += kBuildThreads)
            if (p.counts[s]) atomicAnd(&sAllEmpty, 0u);
    u32 localMax = 0;
    bool any = false;
    const u32 scanBins = isZc ? min(256u, p.bins) : p.bins;
    for (u32 b = threadIdx.x; b < scanBins; b += kBuildThreads)
        if (hist[b]) { localMax = b; any = true; }
    if (any) atomicMax(&sMax, localMax);
    __syncthreads();
    u32 symbolMax = count ? sMax : 0u;
    // Histogram.cu:117-121: with every stream of the call empty the reference
    // builds its tables from stale arena words; for zero-count table i that
    // word is the low half of a device pointer when 2+2i < S (nonzero), else
    // the all-zero run-length scan output.
    const bool quirkLeaf = isZc && sAllEmpty && (2u + 2u * (sIdx - es.groupFirst) < es.groupSize);
    // 2. leaves in symbol order
    const bool smemHeap = true;
    u32 L;
    u32* leafSym = p.leafSymWork + u64(t) * p.leavesMax;
    u64* heapG = p.leafWork + u64(t) * p.leavesMax;
    u32* parent = p.parentWork + u64(t) * 2 * p.leavesMax;
    u32* orderG = p.orderWork + u64(t) * p.leavesMax;
    if (quirkLeaf) {
        if (threadIdx.x == 0) { leafSym[0] = 0; heapG[0] = (u64(1) << 32) | 0u; sL = 1; }
        __syncthreads();
        L = 1;
    } else if (count == 0) {
        L = 0;
    } else {
        const u32 nb = symbolMax + 1;
        const u32 per = (nb + kBuildThreads - 1) / kBuildThreads;
        const u32 b0 = threadIdx.x * per, b1 = min(nb, b0 + per);
        u32 c = 0;
        for (u32 b = b0; b < b1; ++b) c += hist[b] ? 1u : 0u;
        u32 tot;
        u32 off = blockExclusiveSum<kBuildThreads>(c, sScan, &tot);
        L = tot;
        if (L > p.leavesMax) {
            if (threadIdx.x == 0) atomicOr(p.errors, DEV_ERR_TABLE_CAPACITY);
            return;
        }
        const bool quirk65535 = p.symBytes == 2 && p.bins == 65536u && symbolMax == 65535u;
        for (u32 b = b0; b < b1; ++b) {
            u32 h = hist[b];
            if (h) {
                if (quirk65535 && b == 65535u) h += count & 1u;   // HistogramKernels.cui:165,200 padding word
                leafSym[off] = b;
                heapG[off] = (u64(h) << 32) | off;
                ++off;
            }
        }
        __syncthreads();
    }
    const bool inSmem = smemHeap && L <= p.heapCap;
    u64* heap = inSmem ? reinterpret_cast<u64*>(dyn) : heapG;
    u32* order = inSmem ? reinterpret_cast<u32*>(dyn + sizeof(u64) * p.heapCap) : orderG;
    if (inSmem)
        for (u32 i = threadIdx.x; i < L; i += kBuildThreads) heap[i] = heapG[i];
    __syncthreads();
    // 3. tree, depths and sort (thread 0)
    if (threadIdx.x == 0) {
        u32 maxLen = 0;
        if (L >= 1) {
            hb::buildTree(heap, parent, int(L));
            // depths in place over the parent links
            const int nodes = int(2 * L - 1);
            parent[nodes - 1] = 0;
            for (int id = nodes - 2; id >= 0; --id) {
                u32 d = parent[parent[id]] + 1u;
                parent[id] = d > 255u ? 255u : d;
            }
            for (u32 i = 0; i < L; ++i) {
                u32 d = parent[i];
                maxLen = max(maxLen, d);
                order[i] = (min(d, 31u) << 27) | i;
            }
            if (maxLen <= 31) hb::introsort(order, int(L), hb::LenLess());
        }
        sMaxLen = maxLen;
        for (int l = 0; l < 32; ++l) lenCount[l] = 0;
    }
    __syncthreads();
    const u32 maxLen = sMaxLen;
    if (maxLen > 31) {
        if (threadIdx.x == 0) atomicOr(p.errors, DEV_ERR_CODEWORD_TOO_LONG);
        return;
    }
    // 4. canonical codes (HuffmanTable.cu:551-593)
    for (u32 k = threadIdx.x; k < L; k += kBuildThreads) {
        u32 len = order[k] >> 27;
        if (len) atomicAdd(&lenCount[len - 1], 1u);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        u32 idx = 0, code = 0;
        for (u32 l = 1; l <= 32; ++l) {
            firstIndex[l] = idx;
            firstCode[l] = code;
            u32 c = l <= 31 ? lenCount[l - 1] : 0u;
            idx += c;
            code = (code + c) << 1;
        }
    }
    __syncthreads();
    uint2* enc = p.enc + u64(t) * p.bins;
    for (u32 k = threadIdx.x; k < L; k += kBuildThreads) {
        u32 len = order[k] >> 27;
        u32 sym = leafSym[order[k] & hb::kLeafMask];
        u32 code = len ? firstCode[len] + (k - firstIndex[len]) : 0u;
        enc[sym] = make_uint2(code, len);
    }
    // 5. serialized table (HuffmanTable.cu:470-485)
    const bool longSym = p.log2Max > 16;
    const u32 symbolBits = requiredBits(symbolMax);
    const u32 fixedBits = 5 + maxLen * p.log2Max + p.log2Max + (longSym ? 5u : 4u);
    const u32 headerBits = fixedBits + L * symbolBits;
    u32* hdr = p.headers + u64(t) * p.hdrWordsMax;
    const u32 hdrWords = u32(ceilDiv(headerBits, 32));
    if (hdrWords > p.hdrWordsMax) {
        if (threadIdx.x == 0) atomicOr(p.errors, DEV_ERR_TABLE_CAPACITY);
        return;
    }
    for (u32 w = threadIdx.x; w < hdrWords; w += kBuildThreads) hdr[w] = 0;
    __syncthreads();
    if (threadIdx.x == 0) {
        u32 pos = 0;
        putBits(hdr, pos, maxLen, 5); pos += 5;
        for (u32 l = 0; l < maxLen; ++l) { putBits(hdr, pos, lenCount[l], p.log2Max); pos += p.log2Max; }
        putBits(hdr, pos, L, p.log2Max); pos += p.log2Max;
        putBits(hdr, pos, symbolBits, longSym ? 5 : 4);
    }
    for (u32 k = threadIdx.x; k < L; k += kBuildThreads)
        putBits(hdr, fixedBits + k * symbolBits, leafSym[order[k] & hb::kLeafMask], symbolBits);
    if (threadIdx.x == 0) {
        TableMeta m;
        m.count = count;
        m.symbolMax = symbolMax;
        m.leaves = L;
        m.maxLen = maxLen;
        m.headerBits = headerBits;
        m.codeBits = 0;
        m.blocks = u32(ceilDiv(count, p.cb));
        m.pad = 0;
        p.meta[t] = m;
    }
}

// ---------------------------------------------------------------------------
// Huffman encode (Huffman.cu:73-187): per coding block bit totals, per table
// scan to block offsets, then packing.
// ---------------------------------------------------------------------------
constexpr u32 kPackWarps = 8;

template <class Sym>
__global__ void __launch_bounds__(kPackWarps * 32) k_blockBits(EncParams p) {
    if (*(volatile u32*)p.errors) return;
    const u32 t = blockIdx.y;
    const u32 b = blockIdx.x * kPackWarps + (threadIdx.x >> 5);
    const u32 lane = threadIdx.x & 31;
    u32 count;
    const Sym* in = tableInput<Sym>(p, t, count);
    const u32 blocks = u32(ceilDiv(count, p.cb));
    if (b >= blocks) return;
    const uint2* enc = p.enc + u64(t) * p.bins;
    const u32 i0 = b * p.cb, i1 = min(count, i0 + p.cb);
    u32 bits = 0;
    for (u32 i = i0 + lane; i < i1; i += 32) bits += enc[min(u32(in[i]), p.bins - 1u)].y;
    bits = warpSum(bits);
    if (lane == 0) p.blockBits[u64(t) * p.blocksMax + b] = bits;
}

__global__ void __launch_bounds__(1024) k_blockScan(EncParams p) {
    if (*(volatile u32*)p.errors) return;
    __shared__ u32 scratch[40];
    __shared__ u32 carry;
    const u32 t = blockIdx.x;
    const TableMeta m = p.meta[t];
    const u32 blocks = m.blocks;
    const u32* bb = p.blockBits + u64(t) * p.blocksMax;
    u32* bo = p.blockOff + u64(t) * p.blocksMax;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (u32 base = 0; base < blocks; base += 1024) {
        u32 i = base + threadIdx.x;
        u32 v = i < blocks ? bb[i] : 0u;
        u32 tot;
        u32 ex = blockExclusiveSum<1024>(v, scratch, &tot);
        if (i < blocks) bo[i] = carry + ex;
        __syncthreads();
        if (threadIdx.x == 0) carry += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) p.meta[t].codeBits = carry;
}

// Segment layout per stream and exclusive scan over streams (one block).
__global__ void __launch_bounds__(1024) k_layout(EncParams p) {
    if (*(volatile u32*)p.errors) return;
    __shared__ u32 scratch[40];
    __shared__ unsigned long long carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (u32 base = 0; base < p.S; base += 1024) {
        const u32 s = base + threadIdx.x;
        SegmentLayout L{};
        u32 words = 0;
        if (s < p.S) {
            if (p.kind == KIND_RLHUFF) {
                const TableMeta ms = p.meta[s], mz = p.meta[p.S + s];
                const u32 offW = u32(ceilDiv(ceilDiv(p.counts[s], p.cb), 2));
                L.countWord = 0;
                L.hdrWord[0] = 1;
                L.cwWord[0] = L.hdrWord[0] + u32(ceilDiv(ms.headerBits, 32)) + 1;
                L.offWord[0] = L.cwWord[0] + u32(ceilDiv(ms.codeBits, 32));
                L.hdrWord[1] = L.offWord[0] + offW;
                L.cwWord[1] = L.hdrWord[1] + u32(ceilDiv(mz.headerBits, 32)) + 1;
                L.offWord[1] = L.cwWord[1] + u32(ceilDiv(mz.codeBits, 32));
                words = L.offWord[1] + offW;
                L.startBit = 0;
            } else {
                const TableMeta ms = p.meta[s];
                const u32 r = p.streams[s].startBit;
                const u32 offW = u32(ceilDiv(ceilDiv(p.streams[s].n, p.cb), 2));
                L.hdrWord[0] = 0;
                L.cwWord[0] = u32(ceilDiv(r + ms.headerBits, 32)) + 1;
                L.offWord[0] = L.cwWord[0] + u32(ceilDiv(ms.codeBits, 32));
                words = L.offWord[0] + offW;
                L.startBit = r;
            }
            L.words = words;
            L.bitLength = words * 32u;
        }
        // 64-bit carry across chunks; within a chunk a 32-bit scan suffices
        u32 tot;
        u32 ex = blockExclusiveSum<1024>(words, scratch, &tot);
        if (s < p.S) {
            L.startWord = carry + ex;
            p.layout[s] = L;
        }
        __syncthreads();
        if (threadIdx.x == 0) carry += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        p.totals[0] = carry;
        if (carry > p.outWordsMax) atomicOr(p.errors, DEV_ERR_TABLE_CAPACITY);
    }
}

// Or the part of codeword `code` (len bits at absolute bit `pos`) that falls
// in words [wLo, wHi) into win[] (win[0] = word wLo).
__device__ __forceinline__ void orCodeword(u32* win, u32 wLo, u32 wHi, u32 pos, u32 code, u32 len) {
    if (len == 0) return;
    const u32 w0 = pos >> 5;
    const int shift = int(32 - (pos & 31u)) - int(len);
    if (shift >= 0) {
        if (w0 >= wLo && w0 < wHi) atomicOr(win + (w0 - wLo), code << shift);
    } else {
        if (w0 >= wLo && w0 < wHi) atomicOr(win + (w0 - wLo), code >> (-shift));
        if (w0 + 1 >= wLo && w0 + 1 < wHi) atomicOr(win + (w0 + 1 - wLo), code << (32 + shift));
    }
}

// Each warp writes the output words whose first bit lies in its coding block
// (gather ownership: no atomics on global memory, no pre-zeroing); the bits
// of the last owned word that belong to the next block are recomputed from
// that block's first symbols.
template <class Sym>
__global__ void __launch_bounds__(kPackWarps * 32) k_pack(EncParams p) {
    extern __shared__ u32 winAll[];
    if (*(volatile u32*)p.errors) return;
    const u32 t = blockIdx.y;
    const u32 warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const u32 b = blockIdx.x * kPackWarps + warp;
    const u32 winWords = p.cb + 2;
    u32* win = winAll + warp * winWords;
    u32 count;
    const Sym* in = tableInput<Sym>(p, t, count);
    const TableMeta m = p.meta[t];
    if (b >= m.blocks) return;
    const u32* bo = p.blockOff + u64(t) * p.blocksMax;
    const u32 off0 = bo[b];
    const u32 off1 = (b + 1 < m.blocks) ? bo[b + 1] : m.codeBits;
    const u32 wLo = (off0 + 31) >> 5, wHi = (off1 + 31) >> 5;
    if (wLo >= wHi) return;
    for (u32 w = lane; w < wHi - wLo; w += 32) win[w] = 0;
    __syncwarp();
    const uint2* enc = p.enc + u64(t) * p.bins;
    const u32 i0 = b * p.cb;
    const u32 per = p.cb / 32;
    const u32 j0 = i0 + lane * per;
    uint2 cw[8];
    u32 lsum = 0;
    for (u32 k = 0; k < per; ++k) {
        const u32 j = j0 + k;
        cw[k] = j < count ? enc[min(u32(in[j]), p.bins - 1u)] : make_uint2(0, 0);
        lsum += cw[k].y;
    }
    u32 pos = off0 + warpInclusiveSum(lsum) - lsum;
    for (u32 k = 0; k < per; ++k) {
        orCodeword(win, wLo, wHi, pos, cw[k].x, cw[k].y);
        pos += cw[k].y;
    }
    // bits of the next block inside the last owned word
    if (b + 1 < m.blocks && (wHi << 5) > off1) {
        const u32 j = (b + 1) * p.cb + lane;
        uint2 c = j < count ? enc[min(u32(in[j]), p.bins - 1u)] : make_uint2(0, 0);
        u32 q = off1 + warpInclusiveSum(c.y) - c.y;
        if (q < (wHi << 5)) orCodeword(win, wLo, wHi, q, c.x, c.y);
    }
    __syncwarp();
    const u32 s = p.kind == KIND_RLHUFF ? (t < p.S ? t : t - p.S) : t;
    const u32 which = (p.kind == KIND_RLHUFF && t >= p.S) ? 1u : 0u;
    const SegmentLayout L = p.layout[s];
    u32* dst = p.out + L.startWord + L.cwWord[which];
    for (u32 w = lane; w < wHi - wLo; w += 32) dst[wLo + w] = win[w];
}

// Count words, table headers, codeword bit counts and offset increments.
__global__ void __launch_bounds__(128) k_headers(EncParams p) {
    if (*(volatile u32*)p.errors) return;
    const u32 s = blockIdx.x;
    const SegmentLayout L = p.layout[s];
    u32* seg = p.out + L.startWord;
    const u32 parts = p.kind == KIND_RLHUFF ? 2u : 1u;
    if (p.kind == KIND_RLHUFF && threadIdx.x == 0) seg[L.countWord] = p.counts[s];
    for (u32 part = 0; part < parts; ++part) {
        const u32 t = part == 0 ? s : p.S + s;
        const TableMeta m = p.meta[t];
        const u32* hdr = p.headers + u64(t) * p.hdrWordsMax;
        const u32 r = part == 0 ? L.startBit : 0u;
        const u32 hw = u32(ceilDiv(r + m.headerBits, 32));
        u32* dst = seg + L.hdrWord[part];
        const u32 srcWords = u32(ceilDiv(m.headerBits, 32));
        for (u32 w = threadIdx.x; w < hw; w += blockDim.x) {
            u32 v;
            if (r == 0) {
                v = hdr[w];
            } else {
                const u32 hi = (w >= 1 && w - 1 < srcWords) ? hdr[w - 1] : 0u;
                const u32 lo = w < srcWords ? hdr[w] : 0u;
                v = (hi << (32 - r)) | (lo >> r);
            }
            dst[w] = v;
        }
        if (threadIdx.x == 0) seg[L.cwWord[part] - 1] = m.codeBits;
        // offsets: u16 increments, two per word, first in the low half (LE memcpy)
        const u32 nOff = m.blocks;
        const u32* bo = p.blockOff + u64(t) * p.blocksMax;
        u32* od = seg + L.offWord[part];
        for (u32 w = threadIdx.x; w < (nOff + 1) / 2; w += blockDim.x) {
            const u32 k0 = 2 * w, k1 = 2 * w + 1;
            const u32 a = k0 == 0 ? bo[0] : bo[k0] - bo[k0 - 1];
            const u32 b = k1 < nOff ? bo[k1] - bo[k1 - 1] : 0u;
            od[w] = (a & 0xFFFFu) | ((b & 0xFFFFu) << 16);
        }
    }
}

// ---------------------------------------------------------------------------
// Host orchestration.
// ---------------------------------------------------------------------------
static EncParams makeParams(cc_instance* I, int kind, u32 S) {
    EncParams p{};
    p.kind = kind;
    p.S = S;
    p.cb = I->codingBlockSize;
    p.log2Max = I->log2Max;
    p.bins = I->bins;
    p.symBytes = I->symBytes;
    p.streams = I->dStreams;
    p.compact = static_cast<char*>(I->compact);
    p.zc = static_cast<char*>(I->zc);
    p.nStride = I->elemCountPerStreamMax;
    p.tiles = I->tiles;
    p.tileStart = I->tileStart;
    p.tilesMax = I->tilesMax;
    p.hist = I->hist;
    p.enc = I->enc;
    p.meta = I->meta;
    p.headers = I->headers;
    p.hdrWordsMax = I->hdrWordsMax;
    p.blockBits = I->blockBits;
    p.blockOff = I->blockOff;
    p.blocksMax = I->blocksMax;
    p.layout = I->layout;
    p.out = I->out;
    p.outWordsMax = I->outWordsMax;
    p.counts = I->counts;
    p.errors = I->errors;
    p.totals = I->totals;
    p.leafWork = I->leafWork;
    p.parentWork = I->parentWork;
    p.orderWork = I->orderWork;
    p.leafSymWork = I->leafSymWork;
    p.leavesMax = I->leavesMax;
    p.heapCap = std::min<u32>(I->leavesMax, 12288u);
    return p;
}

template <class Sym>
static int launchEncode(cc_instance* I, const EncParams& p, u32 nMax) {
    cudaStream_t st = I->stream;
    const u32 T = p.kind == KIND_RLHUFF ? 2 * p.S : p.S;
    const u32 tiles = std::max<u32>(1u, u32(ceilDiv(nMax, kRleTile)));
    CC_TRY_CUDA(cudaMemsetAsync(I->errors, 0, 8 * sizeof(u32), st), "memset errors");
    CC_TRY_CUDA(cudaMemsetAsync(I->hist, 0, u64(T) * I->bins * sizeof(u32), st), "memset histograms");
    dim3 gTiles(tiles, p.S);
    if (p.kind == KIND_RLHUFF) {
        { SectionTimer t(I, "enc.rle_summary", st); k_rleSummary<Sym><<<gTiles, kRleThreads, 0, st>>>(p); countLaunch(); }
        { SectionTimer t(I, "enc.rle_scan", st); k_rleScan<<<p.S, 1024, 0, st>>>(p); countLaunch(); }
        { SectionTimer t(I, "enc.rle_write_hist", st); k_rleWrite<Sym><<<gTiles, kRleThreads, 0, st>>>(p); countLaunch(); }
    } else {
        { SectionTimer t(I, "enc.histogram", st); k_histPlain<Sym><<<gTiles, kRleThreads, 0, st>>>(p); countLaunch(); }
    }
    const size_t buildSmem = size_t(p.heapCap) * (sizeof(u64) + sizeof(u32));
    CC_TRY_CUDA(cudaFuncSetAttribute(k_tableBuild, cudaFuncAttributeMaxDynamicSharedMemorySize, int(buildSmem) > 0 ? int(buildSmem) : 1), "tableBuild smem");
    { SectionTimer t(I, "enc.table_build", st); k_tableBuild<<<T, kBuildThreads, buildSmem, st>>>(p); countLaunch(); }
    const u32 blocks = std::max<u32>(1u, u32(ceilDiv(nMax, p.cb)));
    dim3 gBlocks(u32(ceilDiv(blocks, kPackWarps)), T);
    { SectionTimer t(I, "enc.block_bits", st); k_blockBits<Sym><<<gBlocks, kPackWarps * 32, 0, st>>>(p); countLaunch(); }
    { SectionTimer t(I, "enc.block_scan", st); k_blockScan<<<T, 1024, 0, st>>>(p); countLaunch(); }
    { SectionTimer t(I, "enc.layout", st); k_layout<<<1, 1024, 0, st>>>(p); countLaunch(); }
    const size_t packSmem = size_t(kPackWarps) * (p.cb + 2) * sizeof(u32);
    { SectionTimer t(I, "enc.pack", st); k_pack<Sym><<<gBlocks, kPackWarps * 32, packSmem, st>>>(p); countLaunch(); }
    { SectionTimer t(I, "enc.headers", st); k_headers<<<p.S, 128, 0, st>>>(p); countLaunch(); }
    CC_TRY_CUDA(cudaGetLastError(), "encode launch");
    return CC_OK;
}

int encodeDevice(cc_instance* I, int kind, const EncStream* streams, u32 S, bool download, u64* totalWords) {
    if (totalWords) *totalWords = 0;
    if (S == 0) { I->lastLayout.clear(); return CC_OK; }
    if (S > I->streamCountMax) { setError("stream count %u exceeds instance limit %u", S, I->streamCountMax); return CC_ERR_CAPACITY; }
    u32 nMax = 0;
    for (u32 i = 0; i < S; ++i) {
        if (streams[i].n > I->elemCountPerStreamMax) {
            setError("symbol count %u exceeds instance limit %u", streams[i].n, I->elemCountPerStreamMax);
            return CC_ERR_CAPACITY;
        }
        nMax = std::max(nMax, streams[i].n);
    }
    cudaStream_t st = I->stream;
    char* slot = I->takeRingSlot();
    std::memcpy(slot, streams, sizeof(EncStream) * S);
    CC_TRY_CUDA(cudaMemcpyAsync(I->dStreams, slot, sizeof(EncStream) * S, cudaMemcpyHostToDevice, st), "upload streams");
    cudaEventRecord(I->ringEvent[(I->ringNext + cc_instance::kRing - 1) % cc_instance::kRing], st);
    EncParams p = makeParams(I, kind, S);
    int rc = I->symBytes == 2 ? launchEncode<u16>(I, p, nMax) : launchEncode<u32>(I, p, nMax);
    if (rc) return rc;
    // results: layout, total words, error flags
    char* down = I->hostDown;
    CC_TRY_CUDA(cudaMemcpyAsync(down, I->layout, sizeof(SegmentLayout) * S, cudaMemcpyDeviceToHost, st), "download layout");
    char* tail = down + alignUp(sizeof(SegmentLayout) * S, 64);
    CC_TRY_CUDA(cudaMemcpyAsync(tail, I->totals, sizeof(u64), cudaMemcpyDeviceToHost, st), "download totals");
    CC_TRY_CUDA(cudaMemcpyAsync(tail + 64, I->errors, sizeof(u32), cudaMemcpyDeviceToHost, st), "download errors");
    CC_TRY_CUDA(cudaStreamSynchronize(st), "encode");
    u32 flags = *reinterpret_cast<u32*>(tail + 64);
    if (flags) return deviceErrorStatus(flags, "encode");
    u64 total = *reinterpret_cast<u64*>(tail);
    I->lastLayout.assign(reinterpret_cast<SegmentLayout*>(down), reinterpret_cast<SegmentLayout*>(down) + S);
    if (totalWords) *totalWords = total;
    if (download && total) {
        CC_TRY_CUDA(cudaMemcpyAsync(I->hostWords, I->out, total * 4, cudaMemcpyDeviceToHost, st), "download words");
        CC_TRY_CUDA(cudaStreamSynchronize(st), "download words");
    }
    return CC_OK;
}

}  // namespace ccb

using namespace ccb;

extern "C" {

int cc_encode(cc_instance* I, int kind, int symbolBytes, const void* const* dStreams, uint32_t S, uint32_t n,
              const uint32_t* startBits) {
    if (!I || (S && !dStreams)) { setError("cc_encode: null argument"); return CC_ERR_INVALID_ARGUMENT; }
    if (kind != KIND_RLHUFF && kind != KIND_HUFF) { setError("cc_encode: bad kind %d", kind); return CC_ERR_INVALID_ARGUMENT; }
    if (u32(symbolBytes) != I->symBytes) {
        setError("cc_encode: %d-byte symbols need an instance with log2HuffmanDistinctSymbolCountMax %s 16",
                 symbolBytes, symbolBytes == 2 ? "<=" : ">");
        return CC_ERR_INVALID_ARGUMENT;
    }
    cudaSetDevice(I->device);
    std::vector<EncStream> st(S);
    for (u32 i = 0; i < S; ++i) {
        st[i].in = dStreams[i];
        st[i].n = n;
        st[i].startBit = (kind == KIND_HUFF && startBits) ? (startBits[i] & 31u) : 0u;
        st[i].groupFirst = 0;
        st[i].groupSize = S;
    }
    return encodeDevice(I, kind, st.data(), S, true);
}

int cc_encoded_segment(const cc_instance* I, uint32_t i, const uint32_t** words, uint32_t* wordCount,
                       uint32_t* startBit, uint32_t* bitLength) {
    if (!I || i >= I->lastLayout.size()) { setError("cc_encoded_segment: index out of range"); return CC_ERR_INVALID_ARGUMENT; }
    const SegmentLayout& L = I->lastLayout[i];
    if (words) *words = I->hostWords + L.startWord;
    if (wordCount) *wordCount = L.words;
    if (startBit) *startBit = L.startBit;
    if (bitLength) *bitLength = L.bitLength;
    return CC_OK;
}

// Appends the segments to a word buffer with BitStream::write* semantics
// (BitStream.h:377-480): RLHuff segments start at the next word boundary,
// Huff segments at the current bit; bits before the position are kept.
int cc_encode_to_buffer(cc_instance* I, int kind, int symbolBytes, const void* const* dStreams, uint32_t S,
                        uint32_t n, uint32_t* words, uint32_t capacity, uint32_t* bitSize, uint32_t* bitPos) {
    if (!bitSize || !bitPos) { setError("cc_encode_to_buffer: null size/position"); return CC_ERR_INVALID_ARGUMENT; }
    u32 pos = *bitPos;
    std::vector<u32> sb(S, 0);
    if (S) sb[0] = pos & 31u;
    int rc = cc_encode(I, kind, symbolBytes, dStreams, S, n, sb.data());
    if (rc) return rc;
    u64 end = pos;
    for (u32 i = 0; i < S; ++i) {
        const SegmentLayout& L = I->lastLayout[i];
        u64 w0 = kind == KIND_RLHUFF ? ceilDiv(end, 32) : end / 32;
        end = w0 * 32 + L.bitLength;
    }
    u64 needWords = ceilDiv(std::max<u64>(end, *bitSize), 32);
    if (needWords > capacity) {
        *bitSize = u32(std::max<u64>(end, *bitSize));
        setError("cc_encode_to_buffer: need %llu words, capacity %u", (unsigned long long)needWords, capacity);
        return CC_ERR_CAPACITY;
    }
    u32 oldWords = u32(ceilDiv(*bitSize, 32));
    for (u64 w = oldWords; w < needWords; ++w) words[w] = 0;
    u64 cur = pos;
    for (u32 i = 0; i < S; ++i) {
        const SegmentLayout& L = I->lastLayout[i];
        const u32* src = I->hostWords + L.startWord;
        u64 w0 = kind == KIND_RLHUFF ? ceilDiv(cur, 32) : cur / 32;
        u32 r = kind == KIND_RLHUFF ? 0u : u32(cur & 31u);
        u32 keep = r ? (0xffffffffu << (32 - r)) : 0u;
        words[w0] = (words[w0] & keep) | (src[0] & ~keep);
        std::memcpy(words + w0 + 1, src + 1, size_t(L.words - 1) * 4);
        cur = w0 * 32 + L.bitLength;
    }
    *bitPos = u32(cur);
    *bitSize = u32(std::max<u64>(cur, *bitSize));
    return CC_OK;
}

}  // extern "C"
