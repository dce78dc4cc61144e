// encode.cu - device entropy encoder: zero-run RLE, histograms, Huffman table
// construction, codeword packing and bit-stream assembly, all on the GPU.
// Replaces encodeRLHuff / encodeHuff (Encode.cpp:207-471, :648-790) and the
// Tier-0 pieces they call (RunLength.cu:82-188, Histogram.cu:109-289,
// HuffmanTable.cu:385-596, Huffman.cu:73-187, PackInc.cu:210-219).
//
// One call codes a batch of streams of any sizes and of both kinds (a whole
// volume: the lowpass band with encodeHuff and every level's bands with
// encodeRLHuff, or many bricks).  Work is flattened: run-length tiles and
// coding blocks are numbered across all streams and found back by binary
// search over the per-stream / per-table offsets, so one launch of each
// kernel covers the batch and all Huffman tables are built concurrently.
// Launch sequence (no host round trip until the result is read):
//   summary -> scan -> histPlan -> zeroHist -> write(+histograms)
//   -> tableBuild -> blockBits -> blockScan -> layout -> pack -> headers
#include <cstring>

#include "capi_internal.cuh"
#include "table_build.cuh"

namespace ccb {

struct EncParams {
    u32 S, T;
    u32 totalTiles, totalBlocks;
    u32 cb, log2Max, bins, symBytes;
    const EncStreamDev* streams;
    const EncTableDev* tables;
    char* compact;
    char* zc;
    RunSum* tiles;
    TileStart* tileStart;
    u32* streamMax;
    u32* counts;
    u32* hist;
    uint2* enc;
    TableMeta* meta;
    u32* headers;
    u32* blockBits;
    u32* blockOff;
    u32* blockTable;  // [used blocks] table of each coding block in use (k_usedBlocks)
    u32* runTable;    // [runs] table of each run of coding blocks (k_usedBlocks)
    u32* tileStream;  // [totalTiles] stream of each run-length tile (k_lookupMaps)
    SegmentLayout* layout;
    u32* out;
    u64 outWordsMax;
    u64 capHist, capLeaves, capHdr;
    u32* errors;
    u64* totals;
    u64* leafWork;
    u32* parentWork;
    u32* orderWork;
    u32* leafSymWork;
    u32* tierTables;  // [4][T]: the tables of each leaf-count tier (k_leafTiers); counts in totals[4..7]
    u64* planPart;    // [8 per chunk]: sums of each plan chunk (k_histPlan)
    u32 heapCap;      // leaves that fit the shared-memory builder of tableBuild
    u32 buildLo, buildHi;   // k_tableBuild builds the tables with buildLo <= leaves <= buildHi
    u32 buildTier;    // k_tableBuild: kBuildEach (table blockIdx.x) or the tier whose list its CTAs walk
};


// Error flag of the call, read once per block and shared so that every
// thread of the block takes the same branch.
__device__ __forceinline__ bool blockFailed(const EncParams& p) {
    __shared__ u32 sFailed;
    if (threadIdx.x == 0) sFailed = *reinterpret_cast<volatile const u32*>(p.errors);
    __syncthreads();
    return sFailed != 0;
}
__device__ __forceinline__ bool warpFailed(const EncParams& p) {
    return __any_sync(0xffffffffu, *reinterpret_cast<volatile const u32*>(p.errors) != 0);
}

// Stream owning run-length tile `tile`: one load from the map k_lookupMaps
// writes at the start of a call.
__device__ __forceinline__ u32 streamOfTile(const EncParams& p, u32 tile) { return p.tileStream[tile]; }

// Input symbols of table t and their count.
template <class Sym>
__device__ __forceinline__ const Sym* tableInput(const EncParams& p, const EncTableDev& td, u32& count) {
    const EncStreamDev& sd = p.streams[td.stream];
    if (sd.kind == KIND_RLHUFF) {
        count = p.counts[td.stream];
        return reinterpret_cast<const Sym*>(td.which ? p.zc : p.compact) + sd.compactOff;
    }
    count = sd.n;
    return reinterpret_cast<const Sym*>(sd.in);
}

// Run-length tiles: kRleWarps warps x 32 groups x 32 symbols.  Warp w
// covers symbols [w * 1024, (w + 1) * 1024) of the tile; group k of it is 32
// consecutive symbols, symbol k * 32 + i held by lane i.  A ballot gives a
// group's nonzero mask, kept by lane k, so a warp describes its 1024
// symbols with one mask per lane and the run-length bookkeeping is warp
// scans over the groups.  Positions are kept +1 so that 0 means "no
// nonzero".
constexpr u32 kRleWarps = kRleThreads / 32;
static_assert(kRleTile == kRleWarps * 1024, "a tile is 32 groups of 32 symbols per warp");

template <class Sym>
struct WarpSyms {
    u32 x[16];      // this lane's symbol of groups 2j (low half) and 2j + 1 (high half); u16 symbols
    u32 y[32];      // 32-bit symbols (Sym = u32)
    __device__ __forceinline__ u32 at(u32 k) const {   // k a compile-time constant after unrolling
        return sizeof(Sym) == 2 ? (x[k >> 1] >> (16 * (k & 1))) & 0xFFFFu : y[k];
    }
};

// Group data of lane k of the calling warp (its group k).
struct GroupRuns {
    u32 mask, cnt, firstP1, lastP1;
};

// Loads the warp's 1024 symbols from stream position wbase (zero beyond n)
// and returns lane k's group k mask data; maxSym receives the warp's largest
// symbol.
template <class Sym>
__device__ __forceinline__ GroupRuns loadGroups(const Sym* in, u32 wbase, u32 n, WarpSyms<Sym>& v, u32& maxSym) {
    const u32 lane = threadIdx.x & 31u;
#pragma unroll
    for (u32 k = 0; k < 32; ++k) {
        const u32 pos = wbase + 32u * k + lane;
        const u32 x = pos < n ? u32(in[pos]) : 0u;
        if (sizeof(Sym) == 2) {
            if (k & 1) v.x[k >> 1] |= x << 16;
            else v.x[k >> 1] = x;
        } else {
            v.y[k] = x;
        }
    }
    GroupRuns g{0u, 0u, 0u, 0u};
    u32 m = 0;
#pragma unroll
    for (u32 k = 0; k < 32; ++k) {
        const u32 x = v.at(k);
        m = max(m, x);
        const u32 b = __ballot_sync(0xffffffffu, x != 0u);
        if (lane == k) g.mask = b;
    }
    maxSym = __reduce_max_sync(0xffffffffu, m);
    const u32 gb = wbase + 32u * lane;
    g.cnt = __popc(g.mask);
    g.firstP1 = g.mask ? gb + u32(__ffs(g.mask)) : 0u;
    g.lastP1 = g.mask ? gb + 32u - u32(__clz(g.mask)) : 0u;
    return g;
}

// Exclusive max-scan of lastP1 over the warp's lanes (0 for lane 0).
__device__ __forceinline__ u32 warpExclusiveMax(u32 v) {
    const u32 lane = threadIdx.x & 31u;
#pragma unroll
    for (u32 d = 1; d < 32; d <<= 1) {
        const u32 t = __shfl_up_sync(0xffffffffu, v, d);
        if (lane >= d) v = max(v, t);
    }
    const u32 e = __shfl_up_sync(0xffffffffu, v, 1);
    return lane ? e : 0u;
}

__device__ __forceinline__ RunSum shflUpRun(RunSum r, int delta) {
    RunSum t;
    t.cnt = __shfl_up_sync(0xffffffffu, r.cnt, delta);
    t.ext = __shfl_up_sync(0xffffffffu, r.ext, delta);
    t.firstP1 = __shfl_up_sync(0xffffffffu, r.firstP1, delta);
    t.lastP1 = __shfl_up_sync(0xffffffffu, r.lastP1, delta);
    return t;
}

__device__ __forceinline__ RunSum warpInclusiveRun(RunSum r) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        RunSum t = shflUpRun(r, o);
        if (lane >= o) r = runCombine(t, r);
    }
    return r;
}

// The call's tile map: CTA s writes the stream index over its tiles (the
// prefix layout of the call's descriptors).
__global__ void __launch_bounds__(256) k_lookupMaps(EncParams p) {
    const u32 i = blockIdx.x;
    const EncStreamDev& sd = p.streams[i];
    const u32 tiles = u32(ceilDiv(sd.n, kRleTile));
    for (u32 k = threadIdx.x; k < tiles; k += 256) p.tileStream[sd.tileOff + k] = i;
}

// The coding blocks in use (those holding symbols after the run-length
// step), listed table by table: warp t writes t over its meta.blocks entries
// from meta.actOff (k_histPlan).  The block-level kernels walk this list
// instead of every block a table could have.
__global__ void __launch_bounds__(256) k_usedBlocks(EncParams p) {
    if (warpFailed(p)) return;
    const u32 t = blockIdx.x * 8u + (threadIdx.x >> 5), lane = threadIdx.x & 31u;   // a warp per table
    if (t >= p.T) return;
    const TableMeta& m = p.meta[t];
    for (u32 k = lane; k < m.blocks; k += 32) p.blockTable[m.actOff + k] = t;
    const u32 runs = u32(ceilDiv(m.blocks, kRunSymbols / p.cb));
    for (u32 k = lane; k < runs; k += 32) p.runTable[m.runOff + k] = t;
}

// ---------------------------------------------------------------------------
// Run-length encode (RunLength.cu:82-188 semantics: each nonzero symbol with
// the count of zeros before it; runs of 256+ zeros emit (0, 255) entries;
// trailing zeros dropped).
// Pass 1: per tile, the run summary (RLHuff) and the largest symbol, from
// the warps' group masks.
// ---------------------------------------------------------------------------
template <class Sym>
__global__ void __launch_bounds__(kRleThreads) k_summary(EncParams p) {
    __shared__ RunSum sRun[kRleWarps];
    __shared__ u32 sStream, sMaxSym;
    const u32 tile = blockIdx.x;
    const u32 lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) { sStream = streamOfTile(p, tile); sMaxSym = 0; }
    __syncthreads();
    const u32 s = sStream;
    const EncStreamDev sd = p.streams[s];
    const u32 n = sd.n;
    const Sym* in = reinterpret_cast<const Sym*>(sd.in);
    const u32 wbase = (tile - sd.tileOff) * kRleTile + warp * 1024u;
    WarpSyms<Sym> v;
    u32 m;
    const GroupRuns g = loadGroups(in, wbase, n, v, m);
    if (lane == 0 && m) atomicMax(&sMaxSym, m);
    if (sd.kind == KIND_RLHUFF) {
        // the warp's summary: (0, 255) entries of the gaps whose previous
        // nonzero lies in the warp
        const u32 prevW = warpExclusiveMax(g.lastP1);
        const u32 e = (g.mask && prevW) ? (g.firstP1 - prevW - 1u) / 256u : 0u;
        RunSum w;
        w.cnt = __reduce_add_sync(0xffffffffu, g.cnt);
        w.ext = __reduce_add_sync(0xffffffffu, e);
        w.firstP1 = __reduce_min_sync(0xffffffffu, g.mask ? g.firstP1 : 0xFFFFFFFFu);
        w.lastP1 = __reduce_max_sync(0xffffffffu, g.lastP1);
        if (!w.cnt) w.firstP1 = 0;
        if (lane == 0) sRun[warp] = w;
        __syncthreads();
        if (threadIdx.x == 0) {
            RunSum acc{0, 0, 0, 0};
#pragma unroll
            for (u32 k = 0; k < kRleWarps; ++k) acc = runCombine(acc, sRun[k]);
            p.tiles[tile] = acc;
        }
    } else {
        __syncthreads();
    }
    if (threadIdx.x == 0 && sMaxSym) atomicMax(p.streamMax + s, sMaxSym);
}

constexpr u32 kScanWarps = 8;   // warps (streams or tables) per CTA of the per-unit scans

// Pass 2: the scan of each stream's tile summaries, a warp per stream.
__global__ void __launch_bounds__(kScanWarps * 32) k_scan(EncParams p) {
    const u32 s = blockIdx.x * kScanWarps + (threadIdx.x >> 5);
    if (s >= p.S) return;
    const u32 lane = threadIdx.x & 31u;
    const EncStreamDev sd = p.streams[s];
    if (sd.kind != KIND_RLHUFF) {
        if (lane == 0) p.counts[s] = sd.n;
        return;
    }
    const u32 tiles = u32(ceilDiv(sd.n, kRleTile));
    const RunSum* T = p.tiles + sd.tileOff;
    TileStart* TS = p.tileStart + sd.tileOff;
    RunSum carry{0, 0, 0, 0};
    for (u32 base = 0; base < tiles; base += 32) {
        const u32 i = base + lane;
        const RunSum inc = warpInclusiveRun(i < tiles ? T[i] : RunSum{0, 0, 0, 0});
        RunSum ex = shflUpRun(inc, 1);
        if (lane == 0) ex = RunSum{0, 0, 0, 0};
        const RunSum E = runCombine(carry, ex);
        if (i < tiles) {
            TileStart ts;
            ts.prevP1 = E.cnt ? E.lastP1 : 0u;
            ts.out = E.cnt ? E.cnt + E.ext + (E.firstP1 - 1u) / 256u : 0u;
            TS[i] = ts;
        }
        RunSum last;
        last.cnt = __shfl_sync(0xffffffffu, inc.cnt, 31);
        last.ext = __shfl_sync(0xffffffffu, inc.ext, 31);
        last.firstP1 = __shfl_sync(0xffffffffu, inc.firstP1, 31);
        last.lastP1 = __shfl_sync(0xffffffffu, inc.lastP1, 31);
        carry = runCombine(carry, last);
    }
    if (lane == 0) p.counts[s] = carry.cnt ? carry.cnt + carry.ext + (carry.firstP1 - 1u) / 256u : 0u;
}

// Table builders by leaf count (k_leafTiers sorts the tables, k_tableBuild
// builds them): the heap merge is a latency-bound chain on one thread, so a
// smaller table gets a smaller CTA and heap and more of them share an SM.
//   tier 0: up to 256 leaves, a warp, 5 KB of heap (32 per SM)
//   tier 1: up to 1024 leaves, 64 threads, 20 KB (11 per SM)
//   tier 2: up to 2048 leaves, 256 threads, 41 KB (5 per SM)
//   tier 3: more, 256 threads, the full heap (one per SM)
constexpr u32 kTinyLeaves = 256;
constexpr u32 kSmallLeaves = 1024;
constexpr u32 kBuildSplitLeaves = 2048;
constexpr int kTinySegs = int(kTinyLeaves / 17u) + 1;    // sort segments longer than 16 keys
constexpr int kSmallSegs = int(kSmallLeaves / 17u) + 1;
constexpr u32 kBuildEach = 0xFFFFFFFFu;                  // buildTier: one table per CTA
constexpr u32 kTierMinTables = 64;                       // calls of more tables use the tiers

// Pass 3: histogram / builder / header offsets of every table, sized from
// the largest symbol of its stream.  A symbol outside the instance's
// 2^log2Max range fails the call (HuffmanTable.cu:411-419).  CTA b plans the
// kPlanChunk tables of chunk b, four consecutive per thread with their loads
// in flight together: their offsets within the chunk, and the chunk's sums
// (planPart); with more than one chunk, k_histPlanCarry adds the sums of the
// chunks before each one - every CTA's work independent, so a call of 10^5
// tables takes two short launches instead of a loop on one SM.
constexpr u32 kPlanPer = 4;
static_assert(kPlanChunk == 1024 * kPlanPer, "a plan chunk is one 1024-thread CTA's tables");

// The call's totals from the offsets' grand sums c[2..6] (bins, leaves,
// header words, coding blocks, runs), and the capacity check.
__device__ __forceinline__ void planTotals(const EncParams& p, const unsigned long long (&c)[7]) {
    p.totals[2] = c[5];
    p.totals[3] = c[6];
    for (u32 k = 4; k < 8; ++k) p.totals[k] = 0;   // the tier lists' counts (k_leafTiers)
    p.totals[1] = c[2];
    if (c[2] > p.capHist || c[3] > p.capLeaves || c[4] > p.capHdr) atomicOr(p.errors, DEV_ERR_TABLE_CAPACITY);
}

__global__ void __launch_bounds__(1024) k_histPlan(EncParams p) {
    __shared__ u32 scratch[33 * 7];
    const u32 t0 = blockIdx.x * kPlanChunk + threadIdx.x * kPlanPer;
    // per table: (unused), (unused), bins, leaves, header words, blocks, runs
    u32 v[kPlanPer][7];
    TableMeta m[kPlanPer];
#pragma unroll
    for (u32 j = 0; j < kPlanPer; ++j) {
        const u32 t = t0 + j;
        m[j] = TableMeta{};
        u32 hs = 0, ls = 0, ws = 0;
        if (t < p.T) {
            const EncTableDev td = p.tables[t];
            const u32 smax = p.streamMax[td.stream];
            const u32 count = p.counts[td.stream];
            if (td.which == 0 && smax >= p.bins) atomicOr(p.errors, DEV_ERR_SYMBOL_RANGE);
            hs = td.which ? min(256u, p.bins) : min(smax, p.bins - 1u) + 1u;
            ls = min(hs, count + 1u);
            ws = headerWordsFor(ls, p.log2Max);
            m[j].count = count;
            m[j].histSize = hs;
            m[j].blocks = u32(ceilDiv(count, p.cb));
        }
        v[j][0] = 0;
        v[j][1] = 0;
        v[j][2] = hs;
        v[j][3] = ls;
        v[j][4] = ws;
        v[j][5] = m[j].blocks;
        v[j][6] = u32(ceilDiv(m[j].blocks, kRunSymbols / p.cb));
    }
    u32 sum[7], ex[7], tot[7];
#pragma unroll
    for (u32 k = 0; k < 7; ++k) {
        sum[k] = 0;
#pragma unroll
        for (u32 j = 0; j < kPlanPer; ++j) sum[k] += v[j][k];
    }
    blockExclusiveSumN<1024, 7>(sum, ex, tot, scratch);
    unsigned long long at[7];
#pragma unroll
    for (u32 k = 0; k < 7; ++k) at[k] = ex[k];
#pragma unroll
    for (u32 j = 0; j < kPlanPer; ++j) {
        const u32 t = t0 + j;
        if (t < p.T) {
            m[j].histOff = at[2];
            m[j].leafOff = at[3];
            m[j].hdrOff = at[4];
            m[j].actOff = u32(at[5]);
            m[j].runOff = u32(at[6]);
            p.meta[t] = m[j];
        }
#pragma unroll
        for (u32 k = 0; k < 7; ++k) at[k] += v[j][k];
    }
    if (threadIdx.x == 0) {
        if (gridDim.x == 1) {
            unsigned long long c[7];
#pragma unroll
            for (u32 k = 0; k < 7; ++k) c[k] = tot[k];
            planTotals(p, c);
        } else {
#pragma unroll
            for (u32 k = 0; k < 7; ++k) p.planPart[u64(blockIdx.x) * 8 + k] = tot[k];
        }
    }
}

// Chunk b = blockIdx.x + 1 of a plan of more than one chunk: the sums of
// chunks 0 .. b-1 (a warp over planPart) added to its tables' offsets; the
// last chunk's CTA forms the call's totals.
__global__ void __launch_bounds__(1024) k_histPlanCarry(EncParams p) {
    __shared__ unsigned long long sC[7];
    const u32 b = blockIdx.x + 1;
    if (threadIdx.x < 32) {
        unsigned long long c[7] = {0, 0, 0, 0, 0, 0, 0};
        for (u32 i = threadIdx.x; i < b; i += 32)
#pragma unroll
            for (u32 k = 2; k < 7; ++k) c[k] += p.planPart[u64(i) * 8 + k];
#pragma unroll
        for (u32 k = 2; k < 7; ++k)
#pragma unroll
            for (u32 o = 16; o > 0; o >>= 1) c[k] += __shfl_xor_sync(0xffffffffu, c[k], o);
        if (threadIdx.x == 0)
#pragma unroll
            for (u32 k = 0; k < 7; ++k) sC[k] = c[k];
    }
    __syncthreads();
    const u32 t0 = b * kPlanChunk + threadIdx.x * kPlanPer;
#pragma unroll
    for (u32 j = 0; j < kPlanPer; ++j) {
        const u32 t = t0 + j;
        if (t < p.T) {
            TableMeta& m = p.meta[t];
            m.histOff += sC[2];
            m.leafOff += sC[3];
            m.hdrOff += sC[4];
            m.actOff += u32(sC[5]);
            m.runOff += u32(sC[6]);
        }
    }
    if (b == gridDim.x && threadIdx.x == 0) {
        unsigned long long c[7];
#pragma unroll
        for (u32 k = 0; k < 7; ++k) c[k] = sC[k] + p.planPart[u64(b) * 8 + k];
        planTotals(p, c);
    }
}

__global__ void __launch_bounds__(256) k_zeroHist(EncParams p) {
    if (*reinterpret_cast<volatile const u32*>(p.errors)) return;   // no barriers in this kernel
    const u64 total = p.totals[1];
    for (u64 i = u64(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += u64(gridDim.x) * blockDim.x) p.hist[i] = 0;
}

// The leaf count of every table (the nonzero bins of its histogram; a warp
// per table) and the tier list it goes on (tierTables, counts totals[4..7]).
// A table whose histogram is empty (its stream has no symbols) goes on tier
// 0, the only builder that may then give it a leaf.
__global__ void __launch_bounds__(256) k_leafTiers(EncParams p) {
    if (warpFailed(p)) return;
    const u32 t = blockIdx.x * 8u + (threadIdx.x >> 5), lane = threadIdx.x & 31u;
    if (t >= p.T) return;
    const TableMeta m = p.meta[t];
    const u32* h = p.hist + m.histOff;
    u32 c = 0;
    for (u32 b = lane; b < m.histSize; b += 32) c += h[b] ? 1u : 0u;
    c = __reduce_add_sync(0xffffffffu, c);
    if (lane == 0) {
        const u32 tier = c <= kTinyLeaves ? 0u : c <= kSmallLeaves ? 1u : c <= kBuildSplitLeaves ? 2u : 3u;
        const u32 pos = u32(atomicAdd(reinterpret_cast<unsigned long long*>(p.totals + 4 + tier), 1ull));
        p.tierTables[u64(tier) * p.T + pos] = t;
    }
}

// Pass 4: compact symbols + zero counts (RLHuff) and both histograms, or the
// plain histogram of a Huff stream.  Symbol bins below kWriteSymBins are
// counted in shared memory.
//
// RLHuff: a tile's run-length entries form one contiguous range of the
// stream's compact arrays.  Group k of a warp starts its entries after the
// entries of the tile's groups before it (a warp scan of the groups' counts
// plus their (0, 255) entries, and a block combine over the warps); inside a
// group a nonzero's rank is the popcount of the mask below its lane, and its
// zero count the distance to the set bit below it (or to the nonzero before
// the group).  Entries are staged in shared memory at their positions within
// the tile, then copied out with consecutive threads on consecutive entries.
// Both histograms are counted over the staged entries: the eight most
// frequent keys of each (zero counts 0..7, symbols 1..8) in per-lane
// counters, the others with shared-memory atomics.  The stage (dynamic
// shared memory) holds a whole tile's entries for 16-bit symbols - up to one
// per symbol, plus the (0, 255) entries of zero runs inside the tile - so
// only a tile that a zero run of millions of symbols ends in writes its
// entries directly (and counts them with warp-aggregated atomics).
constexpr u32 kWriteSymBins = 4096;   // symbol bins counted in shared memory by k_write

template <class Sym>
constexpr u32 writeStage() { return sizeof(Sym) == 2 ? kRleTile + kRleTile / 256u : kRleTile / 2u; }
template <class Sym>
constexpr size_t writeSmem() { return 2 * sizeof(Sym) * size_t(writeStage<Sym>()); }

template <class Sym>
__global__ void __launch_bounds__(kRleThreads) k_write(EncParams p) {
    constexpr u32 kStage = writeStage<Sym>();
    extern __shared__ __align__(16) unsigned char dynWrite[];
    __shared__ u32 sLast[kRleWarps], sEnt[kRleWarps];
    __shared__ u32 hSym[kWriteSymBins];
    __shared__ u32 hZc[256];
    Sym* const sComp = reinterpret_cast<Sym*>(dynWrite);
    Sym* const sZcs = sComp + kStage;
    __shared__ u32 sStream;
    const u32 lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) sStream = streamOfTile(p, blockIdx.x);
    if (blockFailed(p)) return;   // synchronizes (sStream visible)
    const u32 tile = blockIdx.x;
    const u32 s = sStream;
    const EncStreamDev sd = p.streams[s];
    const u32 n = sd.n;
    const TableMeta mS = p.meta[sd.tableFirst];
    const u32 smemBins = min(mS.histSize, kWriteSymBins);
    for (u32 i = threadIdx.x; i < smemBins; i += kRleThreads) hSym[i] = 0;
    hZc[threadIdx.x] = 0;
    const Sym* in = reinterpret_cast<const Sym*>(sd.in);
    const u32 wbase = (tile - sd.tileOff) * kRleTile + warp * 1024u;
    WarpSyms<Sym> v;
    u32 mUnused;
    const GroupRuns g = loadGroups(in, wbase, n, v, mUnused);
    u32* gSym = p.hist + mS.histOff;
    if (sd.kind != KIND_RLHUFF) {
        __syncthreads();
#pragma unroll
        for (u32 k = 0; k < 32; ++k) {
            const u32 x = v.at(k);
            const bool valid = wbase + 32u * k + lane < n;
            const bool toSmem = valid && x < smemBins;
            aggregatedIncrement(hSym, toSmem ? x : 0u, toSmem);
            if (valid && !toSmem && x < mS.histSize) atomicAdd(gSym + x, 1u);
        }
        __syncthreads();
        for (u32 i = threadIdx.x; i < smemBins; i += kRleThreads)
            if (hSym[i]) atomicAdd(gSym + i, hSym[i]);
        return;
    }
    const TableMeta mZ = p.meta[sd.tableFirst + 1];
    u32* gZc = p.hist + mZ.histOff;
    // the nonzero before each group: in the warp, in the warps before, or
    // before the tile
    const u32 lastW = __reduce_max_sync(0xffffffffu, g.lastP1);
    if (lane == 0) sLast[warp] = lastW;
    __syncthreads();   // also orders the histogram zeroing
    u32 lastBefore = 0;
#pragma unroll
    for (u32 w = 0; w < kRleWarps; ++w)
        if (w < warp) lastBefore = max(lastBefore, sLast[w]);
    const TileStart ts = p.tileStart[tile];
    u32 prev = max(warpExclusiveMax(g.lastP1), lastBefore);
    if (!prev) prev = ts.prevP1;
    const u32 e = g.mask ? (g.firstP1 - prev - 1u) / 256u : 0u;   // (0, 255) entries before the group
    const u32 ent = g.cnt + e;
    const u32 entIncl = warpInclusiveSum(ent);
    if (lane == 31) sEnt[warp] = entIncl;
    __syncthreads();
    u32 warpOut = 0, entries = 0;
#pragma unroll
    for (u32 w = 0; w < kRleWarps; ++w) {
        const u32 x = sEnt[w];
        if (w < warp) warpOut += x;
        entries += x;
    }
    const u32 groupOut = warpOut + entIncl - ent;
    Sym* comp = reinterpret_cast<Sym*>(p.compact) + sd.compactOff + ts.out;
    Sym* zcs = reinterpret_cast<Sym*>(p.zc) + sd.compactOff + ts.out;
    const bool staged = entries <= kStage;                // block-uniform
    Sym* oc = staged ? sComp : comp;
    Sym* oz = staged ? sZcs : zcs;
    {
#pragma unroll
        for (u32 k = 0; k < 32; ++k) {
            const u32 mk = __shfl_sync(0xffffffffu, g.mask, k);
            if (mk == 0u) continue;                           // warp-uniform
            const u32 ok = __shfl_sync(0xffffffffu, groupOut, k);
            const u32 ek = __shfl_sync(0xffffffffu, e, k);
            const u32 pk = __shfl_sync(0xffffffffu, prev, k);
            for (u32 t = lane; t < ek; t += 32) {
                oc[ok + t] = Sym(0);
                oz[ok + t] = Sym(255);
            }
            if ((mk >> lane) & 1u) {
                const u32 below = mk & ((1u << lane) - 1u);
                const u32 gb = wbase + 32u * k;
                const u32 q = gb + lane + 1u;
                const u32 pp = below ? gb + 32u - u32(__clz(below)) : pk;
                const u32 o = ok + ek + u32(__popc(below));
                oc[o] = Sym(v.at(k));
                oz[o] = Sym((q - pp - 1u) & 255u);
            }
        }
    }
    __syncthreads();
    // histograms (and the copy-out of a staged tile)
    const Sym* hc = staged ? sComp : comp;
    const Sym* hz = staged ? sZcs : zcs;
    const bool fast = staged && mZ.histSize == 256u && smemBins > 8u;   // block-uniform
    // the eight most frequent keys of each histogram (zero counts 0..7,
    // symbols 1..8) in per-lane 8-bit counters, four keys per register (at
    // most ceil(kStage / kRleThreads) = 33 entries per lane), added once per
    // warp at the end; integer ALU work only
    u32 z03 = 0, z47 = 0, s03 = 0, s47 = 0;
    bool rangeErr = false;
    for (u32 j0 = 0; j0 < entries; j0 += kRleThreads) {
        const u32 j = j0 + threadIdx.x;
        const bool act = j < entries;
        const u32 sym = act ? u32(hc[j]) : 0u;
        const u32 zc = act ? u32(hz[j]) : 0u;
        if (act && staged) {
            comp[j] = Sym(sym);
            zcs[j] = Sym(zc);
        }
        if (fast) {
            if (act) {
                const u32 zi = 1u << ((zc & 3u) << 3);
                if (zc < 4u) z03 += zi;
                else if (zc < 8u) z47 += zi;
                else atomicAdd(hZc + zc, 1u);
                const u32 k = sym - 1u;            // keys 1..8 -> 0..7
                const u32 si = 1u << ((k & 3u) << 3);
                if (k < 4u) s03 += si;
                else if (k < 8u) s47 += si;
                else if (sym < smemBins) atomicAdd(hSym + sym, 1u);
                else if (sym < mS.histSize) atomicAdd(gSym + sym, 1u);
            }
        } else {
            const bool toSmem = act && sym < smemBins;
            aggregatedIncrement(hSym, toSmem ? sym : 0u, toSmem);
            if (act && !toSmem && sym < mS.histSize) atomicAdd(gSym + sym, 1u);
            const bool zcOk = zc < mZ.histSize;
            rangeErr |= act && !zcOk;
            aggregatedIncrement(hZc, zc, act && zcOk);
        }
    }
    if (fast) {
        // widen to 16-bit fields (keys k, k + 2 per register) and sum over the warp
        u32 a[8] = {z03 & 0x00FF00FFu, (z03 >> 8) & 0x00FF00FFu, z47 & 0x00FF00FFu, (z47 >> 8) & 0x00FF00FFu,
                    s03 & 0x00FF00FFu, (s03 >> 8) & 0x00FF00FFu, s47 & 0x00FF00FFu, (s47 >> 8) & 0x00FF00FFu};
#pragma unroll
        for (u32 o = 16; o > 0; o >>= 1)
#pragma unroll
            for (u32 i = 0; i < 8; ++i) a[i] += __shfl_xor_sync(0xffffffffu, a[i], o);
        if (lane == 0) {
            // a[0]: keys 0, 2; a[1]: 1, 3; a[2]: 4, 6; a[3]: 5, 7 (zero counts); a[4..7] the same for symbols - 1
            const u32 key[4] = {0u, 1u, 4u, 5u};
#pragma unroll
            for (u32 i = 0; i < 4; ++i) {
                const u32 zl = a[i] & 0xFFFFu, zh = a[i] >> 16, sl = a[4 + i] & 0xFFFFu, sh = a[4 + i] >> 16;
                if (zl) atomicAdd(hZc + key[i], zl);
                if (zh) atomicAdd(hZc + key[i] + 2u, zh);
                if (sl) atomicAdd(hSym + key[i] + 1u, sl);
                if (sh) atomicAdd(hSym + key[i] + 3u, sh);
            }
        }
    }
    if (rangeErr) atomicOr(p.errors, DEV_ERR_SYMBOL_RANGE);
    __syncthreads();
    for (u32 i = threadIdx.x; i < smemBins; i += kRleThreads)
        if (hSym[i]) atomicAdd(gSym + i, hSym[i]);
    if (threadIdx.x < mZ.histSize && hZc[threadIdx.x]) atomicAdd(gZc + threadIdx.x, hZc[threadIdx.x]);
}

// ---------------------------------------------------------------------------
// Table construction: one block per table, all tables of the call at once.
// Leaf gathering, depths, the sort (an exact warp-parallel replay of
// std::sort), canonical codes and serialization are block parallel; the heap
// merge runs in one thread on shared memory (table_build.cuh).  Tables with
// more leaves than the shared-memory builder holds run sequentially on
// global memory (huffman_build.cuh).
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

// Builds table t (all kThreads threads of the block; returns uniformly).
// kSegs: the sort's segment queue (segments longer than 16 keys in a round:
// at most heapCap / 17).
template <u32 kThreads, int kSegs>
__device__ void buildTable(const EncParams& p, u32 t) {
    extern __shared__ __align__(16) unsigned char dyn[];
    __shared__ u32 sScan[40];
    __shared__ u32 sMax, sMaxLen, sAllEmpty;
    __shared__ u32 lenCount[32], firstIndex[33], firstCode[33];
    __shared__ tb::Seg sSegA[kSegs], sSegB[kSegs];
    __shared__ int sSegCount[4];
    if (threadIdx.x == 0) { sMax = 0; sAllEmpty = 1; }
    if (blockFailed(p)) return;
    const EncTableDev td = p.tables[t];
    const EncStreamDev es = p.streams[td.stream];
    TableMeta meta = p.meta[t];
    const u32 count = meta.count;
    const u32* hist = p.hist + meta.histOff;
    const bool isZc = es.kind == KIND_RLHUFF && td.which == 1;

    // 1. largest present symbol
    if (es.kind == KIND_RLHUFF)
        for (u32 s = es.groupFirst + threadIdx.x; s < es.groupFirst + es.groupSize; s += kThreads)
            if (p.counts[s]) atomicAnd(&sAllEmpty, 0u);
    u32 localMax = 0;
    bool any = false;
    for (u32 b = threadIdx.x; b < meta.histSize; b += kThreads)
        if (hist[b]) { localMax = b; any = true; }
    if (any) atomicMax(&sMax, localMax);
    __syncthreads();
    const u32 symbolMax = count ? sMax : 0u;
    // Histogram.cu:117-121: with every stream of the reference call empty the
    // reference builds its tables from stale arena words; for zero-count table
    // i that word is the low half of a device pointer when 2+2i < S (nonzero),
    // else the all-zero run-length scan output.
    const bool quirkLeaf = isZc && sAllEmpty && (2u + 2u * (td.stream - es.groupFirst) < es.groupSize);
    // 2. leaves in symbol order: heap keys go straight to the shared-memory
    //    heap (1-based, see table_build.cuh) when the table fits
    u32* leafSym = p.leafSymWork + meta.leafOff;
    u64* heapG = p.leafWork + meta.leafOff;
    u64* H = reinterpret_cast<u64*>(dyn);                                        // [heapCap + 2]
    u32* parentS = reinterpret_cast<u32*>(dyn + sizeof(u64) * (p.heapCap + 2));  // [2 heapCap]
    u32* orderS = parentS + 2 * p.heapCap;                                       // [heapCap]
    u32 L;
    if (quirkLeaf) {
        L = 1;
        if (L < p.buildLo || L > p.buildHi) return;   // uniform: the other build launch has it
        if (threadIdx.x == 0) {
            leafSym[0] = 0;
            const u64 key = (u64(1) << 32) | 0u;
            if (L <= p.heapCap) H[1] = key; else heapG[0] = key;
        }
    } else if (count == 0) {
        L = 0;
        if (L < p.buildLo || L > p.buildHi) return;
    } else {
        const u32 nb = symbolMax + 1;
        const u32 per = (nb + kThreads - 1) / kThreads;
        const u32 b0 = threadIdx.x * per, b1 = min(nb, b0 + per);
        u32 c = 0;
        for (u32 b = b0; b < b1; ++b) c += hist[b] ? 1u : 0u;
        u32 tot;
        u32 off = blockExclusiveSum<kThreads>(c, sScan, &tot);
        L = tot;
        if (L < p.buildLo || L > p.buildHi) return;
        const bool toSmem = L <= p.heapCap;
        const bool quirk65535 = p.symBytes == 2 && p.bins == 65536u && symbolMax == 65535u;
        for (u32 b = b0; b < b1; ++b) {
            u32 h = hist[b];
            if (h) {
                if (quirk65535 && b == 65535u) h += count & 1u;   // HistogramKernels.cui:165,200 padding word
                leafSym[off] = b;
                const u64 key = (u64(h) << 32) | off;
                if (toSmem) H[off + 1] = key; else heapG[off] = key;
                ++off;
            }
        }
    }
    const bool inSmem = L <= p.heapCap;
    u32* order = inSmem ? orderS : p.orderWork + meta.leafOff;
    if (threadIdx.x == 0) sMaxLen = 0;
    __syncthreads();
    // 3. tree, depths and sort
    if (inSmem) {
        if (L >= 2) tb::blockMakeHeap(H, int(L));
        if (threadIdx.x == 0 && L >= 2) tb::buildTree(H, parentS, int(L));
        __syncthreads();
        const u32 root = L >= 2 ? 2 * L - 2 : 0;
        u32 localMax = 0;
        for (u32 i = threadIdx.x; i < L; i += kThreads) {
            u32 d = 0, node = i;
            while (node != root && d < 32) { node = parentS[node]; ++d; }
            order[i] = (min(d, 31u) << 27) | i;
            localMax = max(localMax, d);
        }
        if (localMax) atomicMax(&sMaxLen, localMax);
        __syncthreads();
        if (sMaxLen <= 31) {
            u16* lList = reinterpret_cast<u16*>(dyn);            // reuses the heap area (5 bytes per key)
            u16* rList = lList + p.heapCap;
            u8* mark = reinterpret_cast<u8*>(rList + p.heapCap);
            tb::blockIntrosort<kThreads>(order, int(L), lList, rList, mark, sSegA, sSegB, sSegCount);
        }
    } else if (threadIdx.x == 0) {
        // tables larger than the shared-memory builder: sequential, global memory
        u32* parent = p.parentWork + 2 * meta.leafOff;
        u32 maxLen = 0;
        hb::buildTree(heapG, parent, int(L));
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
        sMaxLen = maxLen;
    }
    if (threadIdx.x == 0)
        for (int l = 0; l < 32; ++l) lenCount[l] = 0;
    __syncthreads();
    const u32 maxLen = sMaxLen;
    if (maxLen > 31) {
        if (threadIdx.x == 0) atomicOr(p.errors, DEV_ERR_CODEWORD_TOO_LONG);
        return;
    }
    // 4. canonical codes (HuffmanTable.cu:551-593)
    for (u32 k = threadIdx.x; k < L; k += kThreads) {
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
    uint2* enc = p.enc + meta.histOff;
    for (u32 k = threadIdx.x; k < L; k += kThreads) {
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
    u32* hdr = p.headers + meta.hdrOff;
    const u32 hdrWords = u32(ceilDiv(headerBits, 32));
    for (u32 w = threadIdx.x; w < hdrWords; w += kThreads) hdr[w] = 0;
    __syncthreads();
    if (threadIdx.x == 0) {
        u32 pos = 0;
        putBits(hdr, pos, maxLen, 5); pos += 5;
        for (u32 l = 0; l < maxLen; ++l) { putBits(hdr, pos, lenCount[l], p.log2Max); pos += p.log2Max; }
        putBits(hdr, pos, L, p.log2Max); pos += p.log2Max;
        putBits(hdr, pos, symbolBits, longSym ? 5 : 4);
    }
    for (u32 k = threadIdx.x; k < L; k += kThreads)
        putBits(hdr, fixedBits + k * symbolBits, leafSym[order[k] & hb::kLeafMask], symbolBits);
    if (threadIdx.x == 0) {
        meta.symbolMax = symbolMax;
        meta.leaves = L;
        meta.maxLen = maxLen;
        meta.headerBits = headerBits;
        meta.codeBits = 0;
        p.meta[t] = meta;
    }
}

// One table per CTA (kBuildEach), or the CTAs walk the list of one tier.
template <u32 kThreads, int kSegs>
__global__ void __launch_bounds__(kThreads) k_tableBuild(EncParams p) {
    if (p.buildTier == kBuildEach) {
        buildTable<kThreads, kSegs>(p, blockIdx.x);
        return;
    }
    const u32 n = u32(p.totals[4 + p.buildTier]);
    const u32* list = p.tierTables + u64(p.buildTier) * p.T;
    for (u32 i = blockIdx.x; i < n; i += gridDim.x) {
        buildTable<kThreads, kSegs>(p, list[i]);
        __syncthreads();   // the next table reuses the shared memory
    }
}

// Dynamic shared memory that leaves no room on an SM for another table-build
// CTA or most other kernels' CTAs: the device's per-block opt-in limit minus
// the kernel's static shared memory.
static size_t tableBuildSoloSmem(int device) {
    static size_t cached[64] = {};
    if (device < 0 || device >= 64) return 0;
    if (!cached[device]) {
        int optin = 0;
        cudaFuncAttributes fa{};
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
        cudaFuncGetAttributes(&fa, reinterpret_cast<const void*>(k_tableBuild<kBuildThreads, tb::kMaxSegs>));
        cached[device] = optin > int(fa.sharedSizeBytes) ? size_t(optin) - fa.sharedSizeBytes : 0;
    }
    return cached[device];
}

// ---------------------------------------------------------------------------
// Huffman encode (Huffman.cu:73-187): per coding block bit totals, per table
// scan to block offsets, then packing.  One warp per coding block.
// ---------------------------------------------------------------------------
constexpr u32 kPackWarps = 8;

// A lane's 32 symbols of a run, packed as they lie in memory (two 16-bit
// symbols or one 32-bit symbol per word): one 16-byte vector per 8 or 4
// symbols when the run lies inside the stream and is aligned, else element
// loads.  Positions at or past count read 0.
template <class Sym>
struct LaneRun {
    static constexpr u32 kWords = 32 * sizeof(Sym) / 4;
    u32 w[kWords];
    __device__ __forceinline__ u32 at(u32 k) const {   // k a compile-time constant after unrolling
        return sizeof(Sym) == 2 ? (w[k >> 1] >> (16 * (k & 1))) & 0xFFFFu : w[k];
    }
    __device__ __forceinline__ void load(const Sym* in, u32 j0, u32 count) {
        const Sym* q = in + j0;
        if (j0 + 32u <= count && (reinterpret_cast<uintptr_t>(q) & 15u) == 0) {
#pragma unroll
            for (u32 c = 0; c < kWords / 4; ++c) {
                const uint4 v = reinterpret_cast<const uint4*>(q)[c];
                w[4 * c] = v.x; w[4 * c + 1] = v.y; w[4 * c + 2] = v.z; w[4 * c + 3] = v.w;
            }
            return;
        }
#pragma unroll
        for (u32 c = 0; c < kWords; ++c) {
            if (sizeof(Sym) == 2) {
                const u32 lo = j0 + 2 * c < count ? u32(q[2 * c]) : 0u;
                const u32 hi = j0 + 2 * c + 1 < count ? u32(q[2 * c + 1]) : 0u;
                w[c] = lo | (hi << 16);
            } else {
                w[c] = j0 + c < count ? u32(q[c]) : 0u;
            }
        }
    }
};

// Bits of every coding block in use.  Warps walk the call's run list
// (k_usedBlocks): a run is kRunSymbols consecutive symbols of one table, 32
// per lane, so cb / 32 lanes share a coding block; each lane sums the code
// lengths of its symbols and the block's lanes add theirs.
template <class Sym>
__global__ void __launch_bounds__(kPackWarps * 32) k_blockBits(EncParams p) {
    const u32 lane = threadIdx.x & 31;
    if (warpFailed(p)) return;
    const u32 runs = u32(p.totals[3]);
    const u32 lpb = p.cb / 32u, bpr = kRunSymbols / p.cb;
    const u32 stride = gridDim.x * kPackWarps;
    for (u32 r = blockIdx.x * kPackWarps + (threadIdx.x >> 5); r < runs; r += stride) {
        const u32 t = p.runTable[r];
        const TableMeta& m = p.meta[t];
        const EncTableDev td = p.tables[t];
        const u32 rb = r - m.runOff;
        u32 count;
        const Sym* in = tableInput<Sym>(p, td, count);
        const uint2* enc = p.enc + m.histOff;
        const u32 hs = m.histSize;
        const u32 j0 = rb * kRunSymbols + lane * 32u;
        LaneRun<Sym> sv;
        sv.load(in, j0, count);
        u32 bits = 0;
#pragma unroll
        for (u32 k = 0; k < 32; ++k)
            if (j0 + k < count) bits += enc[min(sv.at(k), hs - 1u)].y;
        for (u32 o = 1; o < lpb; o <<= 1) bits += __shfl_xor_sync(0xffffffffu, bits, o);
        const u32 b = rb * bpr + lane / lpb;
        if (lane % lpb == 0 && b < m.blocks) p.blockBits[td.blockOff + b] = bits;
    }
}

// Exclusive scan of each table's block bits: a warp per table, each lane
// summing eight consecutive blocks per step (256 blocks per step).
__global__ void __launch_bounds__(kScanWarps * 32) k_blockScan(EncParams p) {
    if (warpFailed(p)) return;
    const u32 t = blockIdx.x * kScanWarps + (threadIdx.x >> 5);
    if (t >= p.T) return;
    const u32 blocks = p.meta[t].blocks;
    const u32 off = p.tables[t].blockOff;
    const u32 total = warpExclusiveScan8(p.blockBits + off, p.blockOff + off, blocks, 0u);
    if ((threadIdx.x & 31u) == 0) p.meta[t].codeBits = total;
}

// Segment layout per stream (a thread per stream), then the exclusive scan
// of the segments' words over the streams (k_layout, k_layoutCarry).
__global__ void __launch_bounds__(256) k_layoutSegments(EncParams p) {
    if (*reinterpret_cast<volatile const u32*>(p.errors)) return;   // no barriers in this kernel
    const u32 s = blockIdx.x * 256u + threadIdx.x;
    if (s >= p.S) return;
    SegmentLayout L{};
    const EncStreamDev sd = p.streams[s];
    const u32 offW = u32(ceilDiv(ceilDiv(p.counts[s], p.cb), 2));
    const TableMeta ms = p.meta[sd.tableFirst];
    u32 words;
    if (sd.kind == KIND_RLHUFF) {
        const TableMeta mz = p.meta[sd.tableFirst + 1];
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
        const u32 r = sd.startBit;
        L.hdrWord[0] = 0;
        L.cwWord[0] = u32(ceilDiv(r + ms.headerBits, 32)) + 1;
        L.offWord[0] = L.cwWord[0] + u32(ceilDiv(ms.codeBits, 32));
        words = L.offWord[0] + offW;
        L.startBit = r;
    }
    L.words = words;
    L.bitLength = words * 32u;
    p.layout[s] = L;
}

// CTA b scans the segment words of streams 1024 b .. 1024 b + 1023; with more
// than one chunk its sum goes to planPart and k_layoutCarry adds the chunks
// before each one (the histogram plan's sums are consumed by then).
__global__ void __launch_bounds__(1024) k_layout(EncParams p) {
    __shared__ u32 scratch[40];
    if (blockFailed(p)) return;
    const u32 s = blockIdx.x * 1024u + threadIdx.x;
    const u32 words = s < p.S ? p.layout[s].words : 0u;
    u32 tot;   // a chunk's words fit 32 bits; the offsets over chunks are 64-bit
    const u32 ex = blockExclusiveSum<1024>(words, scratch, &tot);
    if (s < p.S) p.layout[s].startWord = ex;
    if (threadIdx.x == 0) {
        if (gridDim.x == 1) {
            p.totals[0] = tot;
            if (tot > p.outWordsMax) atomicOr(p.errors, DEV_ERR_OUTPUT_CAPACITY);
        } else {
            p.planPart[blockIdx.x] = tot;
        }
    }
}

// Chunk b = blockIdx.x + 1 of a layout of more than one chunk: the words of
// chunks 0 .. b-1 added to its streams' start words; the last chunk's CTA
// forms the call's total and checks the output capacity.
__global__ void __launch_bounds__(1024) k_layoutCarry(EncParams p) {
    __shared__ unsigned long long sC;
    if (blockFailed(p)) return;
    const u32 b = blockIdx.x + 1;
    if (threadIdx.x < 32) {
        unsigned long long c = 0;
        for (u32 i = threadIdx.x; i < b; i += 32) c += p.planPart[i];
#pragma unroll
        for (u32 o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
        if (threadIdx.x == 0) sC = c;
    }
    __syncthreads();
    const unsigned long long c = sC;
    const u32 s = b * 1024u + threadIdx.x;
    if (s < p.S) p.layout[s].startWord += c;
    if (b == gridDim.x && threadIdx.x == 0) {
        const unsigned long long total = c + p.planPart[b];
        p.totals[0] = total;
        if (total > p.outWordsMax) atomicOr(p.errors, DEV_ERR_OUTPUT_CAPACITY);
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

// Packing, by runs of coding blocks (as k_blockBits): the run's codewords
// are contiguous in the table's bit stream from its first block's offset, so
// a lane's start bit is that offset plus the code lengths of the lanes
// before it.  Each warp writes the output words whose first bit lies in its
// run (gather ownership: no atomics on global memory, no pre-zeroing),
// assembling them in a shared-memory window; the bits of the last owned word
// that belong to the next run are recomputed from that run's first symbols.
// A lane looks each code up once and keeps code and length packed in a
// register until its bit offset is known.
constexpr u32 kPackWindowWords = kRunSymbols * 31u / 32u + 2u;

template <class Sym>
__global__ void __launch_bounds__(kPackWarps * 32, 3) k_pack(EncParams p) {
    __shared__ u32 winAll[kPackWarps * kPackWindowWords];
    const u32 warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warpFailed(p)) return;
    u32* win = winAll + warp * kPackWindowWords;
    const u32 runs = u32(p.totals[3]);
    const u32 bpr = kRunSymbols / p.cb;
    const u32 stride = gridDim.x * kPackWarps;
    for (u32 r = blockIdx.x * kPackWarps + warp; r < runs; r += stride) {
        const u32 t = p.runTable[r];
        const TableMeta m = p.meta[t];
        const EncTableDev td = p.tables[t];
        const u32 rb = r - m.runOff;
        const u32 bFirst = rb * bpr, bEnd = min(bFirst + bpr, m.blocks);
        u32 count;
        const Sym* in = tableInput<Sym>(p, td, count);
        const u32* bo = p.blockOff + td.blockOff;
        const u32 off0 = bo[bFirst];
        const u32 off1 = bEnd < m.blocks ? bo[bEnd] : m.codeBits;
        const u32 wLo = (off0 + 31) >> 5, wHi = (off1 + 31) >> 5;
        if (wLo >= wHi) continue;
        for (u32 w = lane; w < wHi - wLo; w += 32) win[w] = 0;
        const uint2* enc = p.enc + m.histOff;
        const u32 hs = m.histSize;
        const u32 j0 = rb * kRunSymbols + lane * 32u;
        // one lookup per symbol: code and length kept packed (code << 5 |
        // length) while the lane's bit offset is scanned; a warp meeting a
        // code longer than 27 bits looks its codes up again instead
        u32 pk[32];
        u32 lsum = 0;
        bool longCode = false;
        {
            LaneRun<Sym> sv;
            sv.load(in, j0, count);
#pragma unroll
            for (u32 k = 0; k < 32; ++k) {
                const uint2 c = j0 + k < count ? enc[min(sv.at(k), hs - 1u)] : make_uint2(0u, 0u);
                lsum += c.y;
                longCode |= c.y > 27u;
                pk[k] = (c.x << 5) | c.y;
            }
        }
        const bool reload = __any_sync(0xffffffffu, longCode);
        __syncwarp();
        // the lane's codewords are consecutive: concatenate them in a 64-bit
        // accumulator (bits left-aligned from the lane's start bit in its
        // first word) and OR whole words into the window - one shared atomic
        // per word touched
        const u32 pos = off0 + warpInclusiveSum(lsum) - lsum;
        {
            u32 w = pos >> 5;
            u32 n = pos & 31u;
            unsigned long long acc = 0;
            auto put = [&](u32 code, u32 len) {
                if (len) {
                    acc |= (unsigned long long)code << (64u - n - len);
                    n += len;
                }
                if (n >= 32u) {
                    if (w >= wLo && w < wHi) atomicOr(win + (w - wLo), u32(acc >> 32));
                    acc <<= 32;
                    n -= 32u;
                    ++w;
                }
            };
            if (!reload) {
#pragma unroll
                for (u32 k = 0; k < 32; ++k) put(pk[k] >> 5, pk[k] & 31u);
            } else {
                LaneRun<Sym> sv;
                sv.load(in, j0, count);
#pragma unroll
                for (u32 k = 0; k < 32; ++k) {
                    const uint2 c = j0 + k < count ? enc[min(sv.at(k), hs - 1u)] : make_uint2(0u, 0u);
                    put(c.x, c.y);
                }
            }
            if (n && w >= wLo && w < wHi) atomicOr(win + (w - wLo), u32(acc >> 32));
        }
        // bits of the next run inside the last owned word
        if (bEnd < m.blocks && (wHi << 5) > off1) {
            const u32 j = bEnd * p.cb + lane;
            const uint2 c = j < count ? enc[min(u32(in[j]), hs - 1u)] : make_uint2(0, 0);
            const u32 q = off1 + warpInclusiveSum(c.y) - c.y;
            if (q < (wHi << 5)) orCodeword(win, wLo, wHi, q, c.x, c.y);
        }
        __syncwarp();
        const u32 which = (p.streams[td.stream].kind == KIND_RLHUFF && td.which) ? 1u : 0u;
        const SegmentLayout& L = p.layout[td.stream];
        u32* dst = p.out + L.startWord + L.cwWord[which];
        for (u32 w = lane; w < wHi - wLo; w += 32) dst[wLo + w] = win[w];
        __syncwarp();   // the window is cleared for the next run only after these reads
    }
}

// Count words, table headers, codeword bit counts and offset increments.  A
// group of g threads (a power of two, 32 .. 512) writes one stream: a call of
// many streams packs 512 / g of them into a CTA instead of one (as many as
// still leave four CTAs per SM).
__global__ void __launch_bounds__(512) k_headers(EncParams p, u32 g) {
    if (blockFailed(p)) return;
    const u32 s = blockIdx.x * (blockDim.x / g) + threadIdx.x / g, gt = threadIdx.x & (g - 1u);
    if (s >= p.S) return;   // no barriers below
    const EncStreamDev sd = p.streams[s];
    const SegmentLayout L = p.layout[s];
    u32* seg = p.out + L.startWord;
    const bool rl = sd.kind == KIND_RLHUFF;
    const u32 parts = rl ? 2u : 1u;
    if (rl && gt == 0) seg[L.countWord] = p.counts[s];
    for (u32 part = 0; part < parts; ++part) {
        const u32 t = sd.tableFirst + part;
        const TableMeta m = p.meta[t];
        const u32* hdr = p.headers + m.hdrOff;
        const u32 r = part == 0 ? L.startBit : 0u;
        const u32 hw = u32(ceilDiv(r + m.headerBits, 32));
        u32* dst = seg + L.hdrWord[part];
        const u32 srcWords = u32(ceilDiv(m.headerBits, 32));
        for (u32 w = gt; w < hw; w += g) {
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
        if (gt == 0) seg[L.cwWord[part] - 1] = m.codeBits;
        // offsets: u16 increments, two per word, first in the low half (LE memcpy)
        const u32 nOff = m.blocks;
        const u32* bo = p.blockOff + p.tables[t].blockOff;
        u32* od = seg + L.offWord[part];
        for (u32 w = gt; w < (nOff + 1) / 2; w += g) {
            const u32 k0 = 2 * w, k1 = 2 * w + 1;
            const u32 a = k0 == 0 ? bo[0] : bo[k0] - bo[k0 - 1];
            const u32 b = k1 < nOff ? bo[k1] - bo[k1 - 1] : 0u;
            od[w] = (a & 0xFFFFu) | ((b & 0xFFFFu) << 16);
        }
    }
}

// Word offset and bit size of each volume's stream in a batched encode's
// output: volume v owns streams first[v] .. first[v+1]-1, written back to back.
__global__ void k_volumeExtents(const SegmentLayout* layout, const u32* first, u32 count, u64* wordOff,
                                u64* bitSize, const u32* errors) {
    const u32 v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= count) return;
    if (*errors) { wordOff[v] = 0; bitSize[v] = 0; return; }
    const u32 a = first[v], b = first[v + 1];
    const u64 off = layout[a].startWord;
    const u64 end = layout[b - 1].startWord + layout[b - 1].words;
    wordOff[v] = off;
    bitSize[v] = (end - off) * 32ull;
}

// ---------------------------------------------------------------------------
// Host orchestration.
// ---------------------------------------------------------------------------
// Writes the stream and table descriptors of a call into `slot` (host) and
// returns its summary; slotBytes bounds the descriptors.
int encodePrepare(cc_instance* I, const EncStream* streams, u32 S, char* slot, size_t slotBytes, EncPlan& hp) {
    hp = EncPlan{};
    hp.S = S;
    for (u32 s = 0; s < S; ++s) {
        const EncStream& e = streams[s];
        const u64 nb = ceilDiv(e.n, I->codingBlockSize);
        hp.T += e.kind == KIND_RLHUFF ? 2u : 1u;
        hp.tiles += u32(ceilDiv(e.n, kRleTile));
        hp.blocks += u32(e.kind == KIND_RLHUFF ? 2 * nb : nb);
        hp.maxCount = std::max(hp.maxCount, e.n);
        if (e.kind == KIND_RLHUFF) hp.compact += e.n;
    }
    if (S > I->capStreams || hp.T > I->capTables || hp.tiles > I->capTiles || hp.blocks > I->capBlocks ||
        hp.compact > I->capCompact) {
        setError("encode: call exceeds the instance capacity (%u streams, %llu run-length symbols)", S,
                 (unsigned long long)hp.compact);
        return CC_ERR_CAPACITY;
    }
    hp.offTables = alignUp(sizeof(EncStreamDev) * S, 64);
    hp.bytes = hp.offTables + sizeof(EncTableDev) * hp.T;
    if (hp.bytes > slotBytes) { setError("encode: descriptors exceed the staging slot"); return CC_ERR_CAPACITY; }
    EncStreamDev* sd = reinterpret_cast<EncStreamDev*>(slot);
    EncTableDev* td = reinterpret_cast<EncTableDev*>(slot + hp.offTables);
    u32 tile = 0, table = 0, block = 0;
    u64 compact = 0;
    for (u32 s = 0; s < S; ++s) {
        const EncStream& e = streams[s];
        EncStreamDev d{};
        d.in = e.in;
        d.n = e.n;
        d.kind = e.kind;
        d.startBit = e.kind == KIND_HUFF ? (e.startBit & 31u) : 0u;
        d.groupFirst = e.groupFirst;
        d.groupSize = e.groupSize;
        d.tileOff = tile;
        d.tableFirst = table;
        d.compactOff = compact;
        sd[s] = d;
        tile += u32(ceilDiv(e.n, kRleTile));
        if (e.kind == KIND_RLHUFF) compact += e.n;
        const u32 parts = e.kind == KIND_RLHUFF ? 2u : 1u;
        const u32 nb = u32(ceilDiv(e.n, I->codingBlockSize));
        for (u32 w = 0; w < parts; ++w) {
            td[table++] = EncTableDev{s, w, block, nb};
            block += nb;
        }
    }
    return CC_OK;
}

template <class Sym>
static int launchEncode(cc_instance* I, const EncParams& p) {
    cudaStream_t st = I->stream;
    CC_TRY_CUDA(cudaMemsetAsync(I->errors, 0, 4 * sizeof(u32), st), "memset errors");
    CC_TRY_CUDA(cudaMemsetAsync(I->streamMax, 0, sizeof(u32) * p.S, st), "memset stream max");
    if (p.S) { k_lookupMaps<<<p.S, 256, 0, st>>>(p); countLaunch(); }
    if (p.totalTiles) { SectionTimer t(I, "enc.summary", st); k_summary<Sym><<<p.totalTiles, kRleThreads, 0, st>>>(p); countLaunch(); }
    {
        SectionTimer t(I, "enc.rle_scan", st);
        k_scan<<<u32(ceilDiv(p.S, kScanWarps)), kScanWarps * 32, 0, st>>>(p);
        countLaunch();
    }
    {
        SectionTimer t(I, "enc.hist_plan", st);
        const u32 chunks = std::max<u32>(1, u32(ceilDiv(p.T, kPlanChunk)));
        k_histPlan<<<chunks, 1024, 0, st>>>(p);
        countLaunch();
        if (chunks > 1) { k_histPlanCarry<<<chunks - 1, 1024, 0, st>>>(p); countLaunch(); }
    }
    { SectionTimer t(I, "enc.hist_zero", st); k_zeroHist<<<2 * 148, 256, 0, st>>>(p); countLaunch(); }
    if (p.totalTiles) {
        CC_TRY_CUDA(ensureSmemAttribute(reinterpret_cast<const void*>(k_write<Sym>),
                                        sizeof(Sym) == 2 ? kAttrWrite16 : kAttrWrite32, I->device, writeSmem<Sym>()),
                    "write smem");
        SectionTimer t(I, "enc.rle_write_hist", st);
        k_write<Sym><<<p.totalTiles, kRleThreads, writeSmem<Sym>(), st>>>(p);
        countLaunch();
    }
    size_t buildSmem = sizeof(u64) * (p.heapCap + 2) + 3 * sizeof(u32) * size_t(p.heapCap);
    // an instance whose tables run beside other kernels (the batched codec's
    // lowpass encode) may ask for an SM of its own per table: the sequential
    // heap merge is latency-bound and loses issue slots to co-resident CTAs
    if (I->tableBuildSoloSM && p.T <= u32(std::max(1, I->smCount > 0 ? I->smCount : 148)))
        buildSmem = std::max(buildSmem, tableBuildSoloSmem(I->device));
    CC_TRY_CUDA(ensureSmemAttribute(reinterpret_cast<const void*>(k_tableBuild<kBuildThreads, tb::kMaxSegs>),
                                    kAttrTableBuild, I->device, buildSmem),
                "tableBuild smem");
    {
        SectionTimer t(I, "enc.table_build", st);
        EncParams q = p;
        q.buildLo = 0;
        q.buildHi = ~0u;
        q.buildTier = kBuildEach;
        const u32 sms = u32(std::max(1, I->smCount > 0 ? I->smCount : 148));
        const bool solo = I->tableBuildSoloSM && p.T <= sms;
        auto heapBytes = [](u32 cap) { return sizeof(u64) * (cap + 2) + 3 * sizeof(u32) * size_t(cap); };
        // a call of few tables builds them in one launch, a CTA each (the
        // tiers' pre-pass, launches and stream forks would cost it more than
        // they save)
        if (!solo && p.T > kTierMinTables) {
            // tables sorted by leaf count, each tier's list walked by its own
            // builder, at the same time: tier 0 on the instance stream, tier 1
            // on the second side stream, tiers 3 and 2 on the first
            k_leafTiers<<<u32(ceilDiv(p.T, 8)), 256, 0, st>>>(q);
            countLaunch();
            const bool side = p.heapCap > kSmallLeaves, side2 = p.heapCap > kTinyLeaves;
            if (side2) {
                CC_TRY_CUDA(cudaEventRecord(I->buildFork, st), "table build fork");
                CC_TRY_CUDA(cudaStreamWaitEvent(I->buildSide2, I->buildFork, 0), "table build fork");
                EncParams small = q;
                small.buildTier = 1;
                small.buildLo = kTinyLeaves + 1;
                small.buildHi = kSmallLeaves;
                small.heapCap = std::min(p.heapCap, kSmallLeaves);
                k_tableBuild<64u, kSmallSegs>
                    <<<std::min(p.T, 10u * sms), 64, heapBytes(small.heapCap), I->buildSide2>>>(small);
                countLaunch();
                CC_TRY_CUDA(cudaEventRecord(I->buildJoin2, I->buildSide2), "table build join");
            }
            if (side) {
                CC_TRY_CUDA(cudaStreamWaitEvent(I->buildSide, I->buildFork, 0), "table build fork");
                if (p.heapCap > kBuildSplitLeaves) {
                    EncParams big = q;
                    big.buildTier = 3;
                    big.buildLo = kBuildSplitLeaves + 1;
                    k_tableBuild<kBuildThreads, tb::kMaxSegs>
                        <<<std::min(p.T, sms), kBuildThreads, buildSmem, I->buildSide>>>(big);
                    countLaunch();
                }
                EncParams mid = q;
                mid.buildTier = 2;
                mid.buildLo = kSmallLeaves + 1;
                mid.buildHi = kBuildSplitLeaves;
                mid.heapCap = std::min(p.heapCap, kBuildSplitLeaves);
                k_tableBuild<kBuildThreads, tb::kMaxSegs>
                    <<<std::min(p.T, 5u * sms), kBuildThreads, heapBytes(mid.heapCap), I->buildSide>>>(mid);
                countLaunch();
                CC_TRY_CUDA(cudaEventRecord(I->buildJoin, I->buildSide), "table build join");
            }
            EncParams tiny = q;
            tiny.buildTier = 0;
            tiny.buildHi = kTinyLeaves;
            tiny.heapCap = std::min(p.heapCap, kTinyLeaves);
            k_tableBuild<32u, kTinySegs><<<std::min(p.T, 32u * sms), 32, heapBytes(tiny.heapCap), st>>>(tiny);
            countLaunch();
            if (side2) CC_TRY_CUDA(cudaStreamWaitEvent(st, I->buildJoin2, 0), "table build join");
            if (side) CC_TRY_CUDA(cudaStreamWaitEvent(st, I->buildJoin, 0), "table build join");
        } else {
            k_tableBuild<kBuildThreads, tb::kMaxSegs><<<p.T, kBuildThreads, buildSmem, st>>>(q);
            countLaunch();
        }
    }
    // used-block list (after the plan, k_histPlan); the block kernels walk it
    // with a grid of a few CTAs per SM
    if (p.totalBlocks && p.T) { k_usedBlocks<<<u32(ceilDiv(p.T, 8)), 256, 0, st>>>(p); countLaunch(); }
    const u32 blockGrid = u32(std::max(1, I->smCount > 0 ? I->smCount : 148)) * 8u;
    // runs of the call: at most the used blocks / blocks per run, plus one per table
    const u32 runBound = u32(ceilDiv(p.totalBlocks, kRunSymbols / p.cb)) + p.T;
    if (p.totalBlocks) {
        const u32 g = std::min<u32>(blockGrid, u32(ceilDiv(runBound, kPackWarps)));
        { SectionTimer t(I, "enc.block_bits", st); k_blockBits<Sym><<<g, kPackWarps * 32, 0, st>>>(p); countLaunch(); }
        {
            SectionTimer t(I, "enc.block_scan", st);
            k_blockScan<<<u32(ceilDiv(p.T, kScanWarps)), kScanWarps * 32, 0, st>>>(p);
            countLaunch();
        }
    }
    {
        SectionTimer t(I, "enc.layout", st);
        k_layoutSegments<<<u32(ceilDiv(p.S, 256)), 256, 0, st>>>(p);
        countLaunch();
        const u32 chunks = std::max<u32>(1, u32(ceilDiv(p.S, 1024)));
        k_layout<<<chunks, 1024, 0, st>>>(p);
        countLaunch();
        if (chunks > 1) { k_layoutCarry<<<chunks - 1, 1024, 0, st>>>(p); countLaunch(); }
    }
    if (p.totalBlocks) {
        const u32 g = std::min<u32>(blockGrid, u32(ceilDiv(runBound, kPackWarps)));
        SectionTimer t(I, "enc.pack", st);
        k_pack<Sym><<<g, kPackWarps * 32, 0, st>>>(p);
        countLaunch();
    }
    {
        SectionTimer t(I, "enc.headers", st);
        // streams per CTA: as few as keep four CTAs per SM busy
        const u32 sms = u32(std::max(1, I->smCount > 0 ? I->smCount : 148));
        u32 per = 1;
        while (per < 16 && u64(2 * per) * 4 * sms <= p.S) per <<= 1;
        const u32 g = 512 / per;
        k_headers<<<u32(ceilDiv(p.S, per)), 512, 0, st>>>(p, g);
        countLaunch();
    }
    CC_TRY_CUDA(cudaGetLastError(), "encode launch");
    return CC_OK;
}

int prepareDecodeAttributes(cc_instance* I);

int prepareKernelAttributes(cc_instance* I) {
    const u32 heapCap = std::min<u32>(I->leavesMax, kBuildSmemLeaves);
    size_t buildSmem = sizeof(u64) * (heapCap + 2) + 3 * sizeof(u32) * size_t(heapCap);
    if (I->tableBuildSoloSM) buildSmem = std::max(buildSmem, tableBuildSoloSmem(I->device));
    CC_TRY_CUDA(ensureSmemAttribute(reinterpret_cast<const void*>(k_tableBuild<kBuildThreads, tb::kMaxSegs>),
                                    kAttrTableBuild, I->device, buildSmem),
                "tableBuild smem");
    if (I->symBytes == 2)
        CC_TRY_CUDA(ensureSmemAttribute(reinterpret_cast<const void*>(k_write<u16>), kAttrWrite16, I->device,
                                        writeSmem<u16>()), "write smem");
    else
        CC_TRY_CUDA(ensureSmemAttribute(reinterpret_cast<const void*>(k_write<u32>), kAttrWrite32, I->device,
                                        writeSmem<u32>()), "write smem");
    return prepareDecodeAttributes(I);
}

void volumeExtents(cc_instance* I, const u32* first, u32 count, u64* wordOff, u64* bitSize, cudaStream_t st) {
    k_volumeExtents<<<u32(ceilDiv(count, 256)), 256, 0, st>>>(I->layout, first, count, wordOff, bitSize, I->errors);
    countLaunch();
}

// Launches the encode of a prepared call whose descriptors are at
// plan.dev (device); writes the segments to out (at most outCap words).
// Only kernel launches and device-side memsets.
int encodeLaunch(cc_instance* I, const EncPlan& hp, u32* out, u64 outCap) {
    const char* dPlan = static_cast<const char*>(hp.dev);
    EncParams p{};
    p.S = hp.S;
    p.T = hp.T;
    p.totalTiles = hp.tiles;
    p.totalBlocks = hp.blocks;
    p.cb = I->codingBlockSize;
    p.log2Max = I->log2Max;
    p.bins = I->bins;
    p.symBytes = I->symBytes;
    p.streams = reinterpret_cast<const EncStreamDev*>(dPlan);
    p.tables = reinterpret_cast<const EncTableDev*>(dPlan + hp.offTables);
    p.compact = static_cast<char*>(I->compact);
    p.zc = static_cast<char*>(I->zc);
    p.tiles = I->tiles;
    p.tileStart = I->tileStart;
    p.streamMax = I->streamMax;
    p.counts = I->counts;
    p.hist = I->hist;
    p.enc = I->enc;
    p.meta = I->meta;
    p.headers = I->headers;
    p.blockBits = I->blockBits;
    p.blockOff = I->blockOff;
    p.blockTable = I->blockTable;
    p.runTable = I->runTable;
    p.tileStream = I->tileStream;
    p.layout = I->layout;
    p.out = out;
    p.outWordsMax = outCap;
    p.capHist = I->capHist;
    p.capLeaves = I->capLeaves;
    p.capHdr = I->capHdr;
    p.errors = I->errors;
    p.totals = I->totals;
    p.leafWork = I->leafWork;
    p.parentWork = I->parentWork;
    p.orderWork = I->orderWork;
    p.leafSymWork = I->leafSymWork;
    p.tierTables = I->tierTables;
    p.planPart = I->planPart;
    p.heapCap = std::min<u32>(std::min<u32>(I->leavesMax, kBuildSmemLeaves), hp.maxCount + 1u);
    return I->symBytes == 2 ? launchEncode<u16>(I, p) : launchEncode<u32>(I, p);
}

int encodeDevice(cc_instance* I, const EncStream* streams, u32 S, const EncOutput& outSpec, bool download,
                 u64* totalWords) {
    if (totalWords) *totalWords = 0;
    if (S == 0) { I->lastLayout.clear(); return CC_OK; }
    cudaStream_t st = I->stream;
    char* slot = I->takeRingSlot();
    EncPlan hp;
    int rc = encodePrepare(I, streams, S, slot, I->hostRingBytes, hp);
    if (rc) return rc;
    hp.dev = I->dPlan;
    CC_TRY_CUDA(cudaMemcpyAsync(I->dPlan, slot, hp.bytes, cudaMemcpyHostToDevice, st), "upload plan");
    cudaEventRecord(I->ringEvent[(I->ringNext + cc_instance::kRing - 1) % cc_instance::kRing], st);
    u32* out = outSpec.words ? outSpec.words : I->out;
    rc = encodeLaunch(I, hp, out, outSpec.words ? outSpec.capacity : I->outWordsMax);
    if (rc) return rc;
    // results: layout, total words, error flags
    char* down = I->hostDown;
    CC_TRY_CUDA(cudaMemcpyAsync(down, I->layout, sizeof(SegmentLayout) * S, cudaMemcpyDeviceToHost, st), "download layout");
    char* tail = down + alignUp(sizeof(SegmentLayout) * S, 64);
    CC_TRY_CUDA(cudaMemcpyAsync(tail, I->totals, sizeof(u64), cudaMemcpyDeviceToHost, st), "download totals");
    CC_TRY_CUDA(cudaMemcpyAsync(tail + 64, I->errors, sizeof(u32), cudaMemcpyDeviceToHost, st), "download errors");
    CC_TRY_CUDA(cudaStreamSynchronize(st), "encode");
    const u32 flags = *reinterpret_cast<u32*>(tail + 64);
    if (flags) return deviceErrorStatus(flags, "encode");
    const u64 total = *reinterpret_cast<u64*>(tail);
    I->lastLayout.assign(reinterpret_cast<SegmentLayout*>(down), reinterpret_cast<SegmentLayout*>(down) + S);
    if (totalWords) *totalWords = total;
    if (download && total) {
        if (total > I->hostWordsMax) { setError("encode: result larger than the host staging"); return CC_ERR_CAPACITY; }
        CC_TRY_CUDA(cudaMemcpyAsync(I->hostWords, out, total * 4, cudaMemcpyDeviceToHost, st), "download words");
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
    if (S > I->streamCountMax) { setError("stream count %u exceeds instance limit %u", S, I->streamCountMax); return CC_ERR_CAPACITY; }
    if (n > I->elemCountPerStreamMax) { setError("symbol count %u exceeds instance limit %u", n, I->elemCountPerStreamMax); return CC_ERR_CAPACITY; }
    DeviceGuard deviceGuard(I->device);
    std::vector<EncStream> st(S);
    for (u32 i = 0; i < S; ++i) {
        st[i].in = dStreams[i];
        st[i].n = n;
        st[i].startBit = (kind == KIND_HUFF && startBits) ? (startBits[i] & 31u) : 0u;
        st[i].groupFirst = 0;
        st[i].groupSize = S;
        st[i].kind = u32(kind);
    }
    return encodeDevice(I, st.data(), S, EncOutput{}, true);
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
