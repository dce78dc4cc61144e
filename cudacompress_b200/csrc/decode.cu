// decode.cu - device entropy decoder: decodeRLHuff / decodeHuff
// (Encode.cpp:473-646, :792-917; Huffman.cu:189-279; HuffmanTable.cu:117-266;
// RunLength.cu:257-328).
//
// One call decodes a batch of streams of any sizes and of both kinds.  Two
// front ends fill the same descriptors:
//  * cc_decode (the reference's decode entry points, caller's host bit
//    streams): the host walks the stream headers - the reference's own
//    decode parses them on the host too and returns before the GPU work is
//    done - and stages the touched words once;
//  * decodePrepare / decodeLaunch (batched volume codec, device-resident bit
//    streams): one thread per bit stream walks its headers on the device, so
//    nothing goes through the host and the launches can be replayed.
// Back end, one launch per stage over the whole batch (coding blocks are
// numbered across the streams of a kind and found back by binary search):
//   symPlan -> tables -> huffman (Huff) | zero counts -> run scan -> symbols
// Every read of the bit stream is bounds-checked, and malformed tables or
// codes raise CC_ERR_CORRUPT_STREAM instead of reading or writing out of
// bounds.
#include <algorithm>
#include <cstring>

#include "capi_internal.cuh"

namespace ccb {

struct DecParams {
    u32 S, T, nSrc, nRl, nH;
    u32 rlBlocks, hBlocks;     // coding blocks (upper bounds) of the RLHuff / Huff streams
    u32 rlMaxN;                // largest output of an RLHuff stream
    u32 cb, log2Max, symBytes, leavesMax;
    u64 capLeaves;
    DecStreamDesc* streams;
    DecTableDesc* tables;
    DecSource* sources;
    const u32* rlList;         // RLHuff stream indices (by blockFirst)
    const u32* hList;          // Huff stream indices (by blockFirst)
    const u32* wordsBase;      // indirect sources (device walk): base + wordOff[k], bitSize[k]
    const u64* wordOff;
    const u64* bitSize;
    DecTable* dec;
    u32* syms;                 // [capLeaves]
    u32* lut;                  // [T][1 << kLutBits]
    u32* blockOff;             // coding-block bit offsets, by table blockOff
    u32* blockSum;             // RLHuff: per zero-count block output lengths
    u64* rlTasks;              // RLHuff decode warp tasks (stream << 32 | first block); count at rlTasks[rlTaskCap]
    u32 rlTaskCap;
    char* zc;                  // decoded zero counts, by stream zcOff
    u64* planPart;             // sums of each chunk of the symbol plan (k_decSymPlan)
    u32* errors;
};

// Bounds-checked view of one bit stream's words.
struct WordSrc {
    const u32* w;
    u64 n;
    __device__ __forceinline__ u32 at(u64 i) const { return i < n ? w[i] : 0u; }
    __device__ __forceinline__ u32 bits(u64 bit, u32 count) const {
        if (count == 0) return 0;
        const u64 wi = bit >> 5;
        const u32 b = u32(bit & 31u);
        const u64 window = (u64(at(wi)) << 32) | at(wi + 1);
        return u32((window << b) >> (64 - count));
    }
};

__device__ __forceinline__ WordSrc srcOf(const DecParams& p, u32 stream) {
    const DecSource& s = p.sources[p.streams[stream].source];
    return WordSrc{s.words, s.wordCount};
}

__device__ __forceinline__ bool capacityFailed(const DecParams& p) {
    return (*reinterpret_cast<volatile const u32*>(p.errors) & DEV_ERR_TABLE_CAPACITY) != 0;
}

// Stream owning flattened block `b` of the RLHuff (or Huff) list.
__device__ __forceinline__ u32 streamOfBlock(const DecParams& p, const u32* list, u32 count, u32 b) {
    u32 lo = 0, hi = count;
    while (hi - lo > 1) {
        const u32 mid = (lo + hi) >> 1;
        if (p.streams[list[mid]].blockFirst <= b) lo = mid; else hi = mid;
    }
    return list[lo];
}

// ---------------------------------------------------------------------------
// Device walk (HuffmanTable.cu:117-151 header fields, Encode.cpp:473-646 /
// 792-917 stream layout, BitStream.h:290-308 alignment).
// ---------------------------------------------------------------------------
struct DevReader {
    const u32* w;
    u64 nWords, size, pos;
    bool ok;
    __device__ u32 read(u32 n) {
        if (n == 0) return 0;
        if (pos + n > size) { ok = false; pos = size; return 0; }
        const u64 wi = pos >> 5;
        const u32 b = u32(pos & 31u);
        const u64 window = (u64(wi < nWords ? w[wi] : 0u) << 32) | (wi + 1 < nWords ? w[wi + 1] : 0u);
        pos += n;
        return u32((window << b) >> (64 - n));
    }
    __device__ void align() {
        const u64 a = (pos + 31) / 32 * 32;
        pos = a < size ? a : size;
    }
    __device__ void skip(u64 n) { pos = pos + n < size ? pos + n : size; }
};

__device__ bool walkTableDev(DevReader& r, u32 log2Max, u32 leavesMax, DecTableDesc& d) {
    d.hdrBit = r.pos;
    d.nLen = r.read(5);
    r.skip(u64(d.nLen) * log2Max);
    d.nSym = r.read(log2Max);
    const bool longSym = log2Max > 16;
    d.symbolBits = r.read(longSym ? 5 : 4);
    if (!longSym && d.symbolBits == 0 && d.nSym > 1) d.symbolBits = 16;   // HuffmanTable.cu:138-139
    r.skip(u64(d.nSym) * d.symbolBits);
    return r.ok && d.nSym <= leavesMax && d.nLen <= 31;
}

__device__ bool walkPayloadDev(DevReader& r, u32 count, u32 cb, DecTableDesc& d) {
    r.align();
    d.cwBits = r.read(32);
    d.cwWord = r.pos / 32;
    r.skip(ceilDiv(d.cwBits, 32) * 32);
    r.align();
    d.offWord = r.pos / 32;
    r.skip(ceilDiv(count, cb) * 16);
    r.align();
    d.count = count;
    return r.ok;
}

__global__ void __launch_bounds__(64) k_decWalk(DecParams p) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.nSrc) return;
    DecSource& src = p.sources[i];
    if (p.wordOff) {
        const u64 bits = p.bitSize[i];
        src.words = p.wordsBase + p.wordOff[i];
        src.bitSize = bits;
        src.wordCount = ceilDiv(bits, 32);
    }
    const u64 wordBits = src.wordCount * 32ull;
    DevReader r{src.words, src.wordCount, src.bitSize < wordBits ? src.bitSize : wordBits, src.startBit, true};
    bool ok = true;
    for (u32 k = 0; k < src.streamCount && ok; ++k) {
        const u32 s = src.firstStream + k;
        DecStreamDesc& sd = p.streams[s];
        DecTableDesc& t0 = p.tables[sd.tableFirst];
        if (sd.kind == KIND_RLHUFF) {
            r.align();
            const u32 m = r.read(32);
            ok = r.ok && m <= sd.n;
            sd.m = ok ? m : 0u;
            DecTableDesc& t1 = p.tables[sd.tableFirst + 1];
            ok = ok && walkTableDev(r, p.log2Max, p.leavesMax, t0) && walkPayloadDev(r, m, p.cb, t0);
            ok = ok && walkTableDev(r, p.log2Max, p.leavesMax, t1) && walkPayloadDev(r, m, p.cb, t1);
        } else {
            sd.m = sd.n;
            ok = walkTableDev(r, p.log2Max, p.leavesMax, t0) && walkPayloadDev(r, sd.n, p.cb, t0);
        }
    }
    if (!ok) {
        atomicOr(p.errors, DEV_ERR_CORRUPT);
        // nothing of this source is decoded
        for (u32 k = 0; k < src.streamCount; ++k) {
            DecStreamDesc& sd = p.streams[src.firstStream + k];
            sd.m = 0;
            const u32 parts = sd.kind == KIND_RLHUFF ? 2u : 1u;
            for (u32 w = 0; w < parts; ++w) {
                DecTableDesc& t = p.tables[sd.tableFirst + w];
                t.count = 0;
                t.nSym = 0;
                t.nLen = 0;
                t.hdrBit = t.cwWord = t.offWord = 0;
                t.cwBits = 0;
                t.symbolBits = 0;
            }
        }
    }
    src.endBit = r.pos;
}

// Symbol array offsets of the tables (prefix of nSym) and capacity check.
// CTA b takes the kPlanChunk tables of chunk b (four consecutive per thread):
// offsets within the chunk and the chunk's sum (planPart); with more than one
// chunk, k_decSymPlanCarry adds the chunks before each one.
__global__ void __launch_bounds__(1024) k_decSymPlan(DecParams p) {
    constexpr u32 kPer = kPlanChunk / 1024;
    __shared__ u32 scratch[40];
    const u32 t0 = blockIdx.x * kPlanChunk + threadIdx.x * kPer;
    u32 v[kPer], sum = 0;
#pragma unroll
    for (u32 j = 0; j < kPer; ++j) {
        v[j] = t0 + j < p.T ? min(p.tables[t0 + j].nSym, p.leavesMax) : 0u;
        sum += v[j];
    }
    u32 tot;
    u32 at = blockExclusiveSum<1024>(sum, scratch, &tot);
#pragma unroll
    for (u32 j = 0; j < kPer; ++j) {
        if (t0 + j < p.T) p.tables[t0 + j].symOff = at;
        at += v[j];
    }
    if (threadIdx.x == 0) {
        if (gridDim.x == 1) {
            if (tot > p.capLeaves) atomicOr(p.errors, DEV_ERR_TABLE_CAPACITY);
        } else {
            p.planPart[blockIdx.x] = tot;
        }
    }
}

// Chunk b = blockIdx.x + 1 of a symbol plan of more than one chunk: the sum
// of chunks 0 .. b-1 added to its tables' offsets; the last chunk's CTA
// checks the capacity.
__global__ void __launch_bounds__(1024) k_decSymPlanCarry(DecParams p) {
    constexpr u32 kPer = kPlanChunk / 1024;
    __shared__ unsigned long long sC;
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
    const u32 t0 = b * kPlanChunk + threadIdx.x * kPer;
#pragma unroll
    for (u32 j = 0; j < kPer; ++j)
        if (t0 + j < p.T) p.tables[t0 + j].symOff += u32(c);
    if (b == gridDim.x && threadIdx.x == 0 && c + p.planPart[b] > p.capLeaves)
        atomicOr(p.errors, DEV_ERR_TABLE_CAPACITY);
}

// ---------------------------------------------------------------------------
// Table parse and decode structures (HuffmanTable.cu:117-151, :205-266).
// ---------------------------------------------------------------------------
// One 64-thread CTA per table (up to 32 tables per SM: the work per table is
// a short chain of dependent steps).
constexpr u32 kDecThreads = 64;

__global__ void __launch_bounds__(kDecThreads) k_decTables(DecParams p) {
    __shared__ u32 cpl[32];
    __shared__ int sFirst[32], sMin[32], sMax[32];
    __shared__ u32 sLim[kLutBits + 1];
    __shared__ u32 sScan[40];
    __shared__ u32 sCarry, sFail;
    const u32 t = blockIdx.x;
    if (threadIdx.x == 0) sFail = capacityFailed(p) ? 1u : 0u;
    __syncthreads();
    if (sFail) return;
    const DecTableDesc d = p.tables[t];
    const WordSrc ws = srcOf(p, d.stream);
    DecTable* D = p.dec + t;
    u32* syms = p.syms + d.symOff;
    u32* lut = p.lut + (u64(t) << kLutBits);
    const u64 cntBit = d.hdrBit + 5;
    if (threadIdx.x < 32) cpl[threadIdx.x] = threadIdx.x < d.nLen ? ws.bits(cntBit + u64(threadIdx.x) * p.log2Max, p.log2Max) : 0u;
    __syncthreads();
    if (threadIdx.x == 0) {
        // canonical codes: codeword[i] = (codeword[i-1]+1) << (len_i - len_{i-1})
        u32 total = 0;
        bool ok = d.nLen <= 31 && d.nSym <= p.leavesMax;
        int code = 0, idx = 0;
        bool first = true;
        int prevLen = 0;
        for (u32 l = 1; l <= 31; ++l) {
            u32 c = cpl[l - 1];
            total += c;
            if (c) {
                if (first) { code = 0; first = false; }
                else code = (code + 1) << (int(l) - prevLen);
                sFirst[l - 1] = idx;
                sMin[l - 1] = code;
                code += int(c) - 1;
                sMax[l - 1] = code;
                idx += int(c);
                prevLen = int(l);
            } else {
                sFirst[l - 1] = sMin[l - 1] = sMax[l - 1] = -1;
            }
        }
        sFirst[31] = sMin[31] = sMax[31] = -1;
        // left-justified kLutBits-bit limits: a prefix e holds a code of
        // length l <= kLutBits iff sLim[l-1] <= e < sLim[l] (the canonical
        // codes of one length are consecutive, each length starting where
        // the previous one ends)
        sLim[0] = 0;
        for (u32 l = 1; l <= kLutBits; ++l)
            sLim[l] = sMax[l - 1] >= 0 ? u32(sMax[l - 1] + 1) << (kLutBits - l) : sLim[l - 1];
        if (d.nLen == 0) ok = ok && d.nSym <= 1;
        else ok = ok && total == d.nSym;
        if (!ok) atomicOr(p.errors, DEV_ERR_CORRUPT);
        sCarry = ok ? 1u : 0u;
    }
    __syncthreads();
    if (!sCarry) {
        if (threadIdx.x == 0) D->nSym = 0xFFFFFFFFu;   // marks the table unusable
        return;
    }
    const u64 symBit = cntBit + u64(d.nLen) * p.log2Max + p.log2Max + (p.log2Max > 16 ? 5u : 4u);
    for (u32 i = threadIdx.x; i < d.nSym; i += kDecThreads) {
        u32 v = ws.bits(symBit + u64(i) * d.symbolBits, d.symbolBits);
        syms[i] = p.symBytes == 2 ? (v & 0xFFFFu) : v;
    }
    // lookup table: first length l <= kLutBits whose prefix fits the canonical
    // range; the entry holds (l << 24) | the symbol's value for 16-bit
    // symbols, | its index otherwise
    const bool valueLut = p.symBytes == 2;
    if (valueLut) __syncthreads();   // syms[] of this table written above
    for (u32 e = threadIdx.x; e < (1u << kLutBits); e += kDecThreads) {
        u32 below = 0;   // lengths whose codes all lie below e
#pragma unroll
        for (u32 l = 1; l <= kLutBits; ++l) below += e >= sLim[l] ? 1u : 0u;
        const u32 l = below + 1;
        u32 entry = 0;
        if (l <= kLutBits) {
            const u32 idx = u32(sFirst[l - 1] + int(e >> (kLutBits - l)) - sMin[l - 1]);
            entry = (l << 24) | (valueLut ? syms[idx] : idx);
        }
        lut[e] = entry;
    }
    if (threadIdx.x < 32) {
        D->firstIndex[threadIdx.x] = sFirst[threadIdx.x];
        D->minCode[threadIdx.x] = sMin[threadIdx.x];
        D->maxCode[threadIdx.x] = sMax[threadIdx.x];
    }
    if (threadIdx.x == 0) {
        D->nSym = d.nSym;
        const u32 v0 = d.nSym >= 1 ? ws.bits(symBit, d.symbolBits) : 0u;
        D->single = p.symBytes == 2 ? (v0 & 0xFFFFu) : v0;
        sCarry = 0;
    }
    // absolute block offsets: inclusive prefix of the u16 increments
    // (PackInc.cu:220-229), eight blocks (four words) per thread per step
    const u32 blocks = u32(ceilDiv(d.count, p.cb));
    u32* bo = p.blockOff + d.blockOff;
    __syncthreads();
    for (u32 base = 0; base < blocks; base += 8 * kDecThreads) {
        const u32 k0 = base + 8 * threadIdx.x;
        u32 inc[8], sum = 0;
#pragma unroll
        for (u32 j = 0; j < 4; ++j) {
            const u32 w = k0 + 2 * j < blocks ? ws.at(d.offWord + k0 / 2 + j) : 0u;
            inc[2 * j] = k0 + 2 * j < blocks ? (w & 0xFFFFu) : 0u;
            inc[2 * j + 1] = k0 + 2 * j + 1 < blocks ? (w >> 16) : 0u;
            sum += inc[2 * j] + inc[2 * j + 1];
        }
        u32 tot;
        const u32 ex = blockExclusiveSum<kDecThreads>(sum, sScan, &tot);
        u32 off = sCarry + ex;
#pragma unroll
        for (u32 j = 0; j < 8; ++j) {
            off += inc[j];
            if (k0 + j < blocks) {
                bo[k0 + j] = off;
                if (off > d.cwBits) atomicOr(p.errors, DEV_ERR_CORRUPT);
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) sCarry += tot;
        __syncthreads();
    }
}

// Decodes up to `cnt` symbols of one coding block starting at absolute bit
// `bit`, calling emit(i, symbol).  kValueLut: lookup entries hold symbol
// values (16-bit symbols), else symbol indices.  The 64-bit window is two
// words, read with a funnel shift.
template <bool kValueLut, class Src, class Emit>
__device__ __forceinline__ void decodeBlock(const Src& ws, const DecTable& D, const u32* syms, const u32* lut,
                                            u64 bit, u32 cnt, bool& corrupt, Emit emit) {
    const u32 nSym = D.nSym;
    if (nSym == 0xFFFFFFFFu) { corrupt = true; return; }
    if (nSym <= 1) {
        const u32 single = D.single;
        for (u32 i = 0; i < cnt; ++i) emit(i, single);
        return;
    }
    u64 w = bit >> 5;
    u32 bpos = u32(bit & 31u);
    u32 hi = ws.at(w), lo = ws.at(w + 1);
    w += 2;
    for (u32 i = 0; i < cnt; ++i) {
        const u32 v = __funnelshift_l(lo, hi, bpos);
        const u32 e = lut[v >> (32 - kLutBits)];
        u32 len, val;
        if (e) {
            len = e >> 24;
            val = e & 0xFFFFFFu;
            if (!kValueLut) {
                if (val >= nSym) { corrupt = true; return; }
                val = syms[val];
            }
        } else {
            len = kLutBits + 1;
            while (len <= 31 && int(v >> (32 - len)) > D.maxCode[len - 1]) ++len;
            if (len > 31) { corrupt = true; return; }
            const u32 idx = u32(D.firstIndex[len - 1] + int(v >> (32 - len)) - D.minCode[len - 1]);
            if (idx >= nSym) { corrupt = true; return; }
            val = syms[idx];
        }
        emit(i, val);
        bpos += len;
        if (bpos >= 32) {
            hi = lo;
            lo = ws.at(w);
            ++w;
            bpos -= 32;
        }
    }
}

// One table's decode data in shared memory: the lookup table, and for codes
// longer than it the left-justified limits - lim[l] = (maxCode[l] + 1) <<
// (32 - l), carried over lengths without codes, so a 32-bit window v holds a
// code longer than l iff v >= lim[l] (the canonical codes of one length are
// consecutive and each length starts where the shorter ones end, so lim never
// decreases) - and the first index / first code of each length.
struct CanonSmem {
    u32 lut[1u << kLutBits];
    unsigned long long lim[36];   // lengths 1..31; 32..35 above every window
    int first[32], minc[32];
};

// Stages table t into cs (all 32 lanes of the calling warp).
__device__ __forceinline__ void stageCanon(CanonSmem& cs, const DecParams& p, u32 t) {
    const u32 lane = threadIdx.x & 31u;
    const u32* g = p.lut + (u64(t) << kLutBits);
    for (u32 e = lane; e < (1u << kLutBits); e += 32) cs.lut[e] = g[e];
    const DecTable& D = p.dec[t];
    const int mc = D.maxCode[lane];
    const u32 l = lane + 1;
    unsigned long long lim = l <= 31 && mc >= 0 ? (unsigned long long)(u32(mc) + 1u) << (32 - l) : 0ull;
#pragma unroll
    for (u32 d = 1; d < 32; d <<= 1) {
        const unsigned long long o = __shfl_up_sync(0xffffffffu, lim, d);
        if (lane >= d) lim = o > lim ? o : lim;   // running maximum
    }
    cs.lim[l] = l <= 31 ? lim : ~0ull;
    if (lane < 4) cs.lim[32 + lane] = ~0ull;
    if (lane == 0) cs.lim[0] = 0;
    cs.first[lane] = D.firstIndex[lane];
    cs.minc[lane] = D.minCode[lane];
    __syncwarp();
}

// decodeBlock with the table in shared memory: the length of a code longer
// than the lookup table is found four lengths per step.
template <bool kValueLut, class Emit>
__device__ __forceinline__ void decodeBlockStaged(const WordSrc& ws, const DecTable& D, const CanonSmem& cs,
                                                  const u32* syms, u64 bit, u32 cnt, bool& corrupt, Emit emit) {
    const u32 nSym = D.nSym;
    if (nSym == 0xFFFFFFFFu) { corrupt = true; return; }
    if (nSym <= 1) {
        const u32 single = D.single;
        for (u32 i = 0; i < cnt; ++i) emit(i, single);
        return;
    }
    u64 w = bit >> 5;
    u32 bpos = u32(bit & 31u);
    u32 hi = ws.at(w), lo = ws.at(w + 1);
    w += 2;
    for (u32 i = 0; i < cnt; ++i) {
        const u32 v = __funnelshift_l(lo, hi, bpos);
        const u32 e = cs.lut[v >> (32 - kLutBits)];
        u32 len, val;
        if (e) {
            len = e >> 24;
            val = e & 0xFFFFFFu;
            if (!kValueLut) {
                if (val >= nSym) { corrupt = true; return; }
                val = syms[val];
            }
        } else {
            const unsigned long long vv = v;
            len = kLutBits + 1;
            for (;;) {
                const u32 c = (vv >= cs.lim[len] ? 1u : 0u) + (vv >= cs.lim[len + 1] ? 1u : 0u) +
                              (vv >= cs.lim[len + 2] ? 1u : 0u) + (vv >= cs.lim[len + 3] ? 1u : 0u);
                len += c;
                if (c < 4 || len > 31) break;
            }
            if (len > 31) { corrupt = true; return; }
            const u32 idx = u32(cs.first[len - 1] + int(v >> (32 - len)) - cs.minc[len - 1]);
            if (idx >= nSym) { corrupt = true; return; }
            val = syms[idx];
        }
        emit(i, val);
        bpos += len;
        if (bpos >= 32) {
            hi = lo;
            lo = ws.at(w);
            ++w;
            bpos -= 32;
        }
    }
}

// decodeHuff: one thread per coding block; when a warp's 32 blocks belong to
// one stream its table is staged in shared memory and its output staged
// there too and written coalesced.
template <class Sym>
__global__ void __launch_bounds__(32) k_decHuff(DecParams p) {
    extern __shared__ __align__(16) unsigned char stage[];
    __shared__ CanonSmem cs;
    if (__any_sync(0xffffffffu, capacityFailed(p))) return;
    const u32 lane = threadIdx.x;
    const u32 b0 = blockIdx.x * 32;
    const u32 gb = b0 + lane;
    const bool valid = gb < p.hBlocks;
    const u32 s = streamOfBlock(p, p.hList, p.nH, valid ? gb : p.hBlocks - 1);
    const u32 s0 = __shfl_sync(0xffffffffu, s, 0);
    const bool uniform = __all_sync(0xffffffffu, !valid || s == s0);
    const DecStreamDesc sd = p.streams[s];
    const u32 b = gb - sd.blockFirst;
    const u32 blocks = u32(ceilDiv(sd.n, p.cb));
    const u32 rowPitch = p.cb + (sizeof(Sym) == 2 ? 2 : 1);
    Sym* rows = reinterpret_cast<Sym*>(stage);
    Sym* out = reinterpret_cast<Sym*>(sd.out);
    bool corrupt = false;
    const bool mine = valid && b < blocks;
    const u32 i0 = b * p.cb;
    if (uniform) stageCanon(cs, p, p.streams[s0].tableFirst);   // the warp's one table
    if (mine) {
        const u32 t = sd.tableFirst;
        const DecTableDesc& td = p.tables[t];
        const WordSrc ws = srcOf(p, s);
        const u32 cnt = min(p.cb, sd.n - i0);
        const u64 bit = td.cwWord * 32ull + p.blockOff[td.blockOff + b];
        if (uniform)
            decodeBlockStaged<sizeof(Sym) == 2>(ws, p.dec[t], cs, p.syms + td.symOff, bit, cnt, corrupt,
                        [&](u32 i, u32 v) { rows[lane * rowPitch + i] = Sym(v); });
        else
            decodeBlock<sizeof(Sym) == 2>(ws, p.dec[t], p.syms + td.symOff, p.lut + (u64(t) << kLutBits), bit, cnt, corrupt,
                        [&](u32 i, u32 v) { out[i0 + i] = Sym(v); });
    }
    if (corrupt) atomicOr(p.errors, DEV_ERR_CORRUPT);
    if (!uniform) return;
    __syncwarp();
    // every lane's sd is the stream of block b0 here
    const u32 bFirst = b0 - sd.blockFirst;
    if (bFirst >= blocks) return;
    const u32 nb = min(32u, blocks - bFirst);
    const u64 base = u64(bFirst) * p.cb;
    const u64 lim = u64(sd.n) - base;
    const u64 total = u64(nb) * p.cb < lim ? u64(nb) * p.cb : lim;
    for (u64 k = lane; k < total; k += 32) out[base + k] = rows[(k / p.cb) * rowPitch + (k % p.cb)];
}

// Coding blocks of RLHuff stream s that a decode covers: its run-length
// symbol count in blocks, within the blocks planned for its length.
__device__ __forceinline__ u32 rlBlocksOf(const DecParams& p, const DecStreamDesc& sd) {
    return u32(min(ceilDiv(u64(sd.m), p.cb), ceilDiv(u64(sd.n), p.cb)));
}

// Warp tasks of the run-length decode, once the headers are walked: every
// RLHuff stream's coding blocks in groups of 32, so that a warp's blocks
// belong to one stream and warps without blocks are not started.  CTA b
// takes the 1024 streams of chunk b; with more than one chunk,
// k_decRlTaskCounts first writes each chunk's task count (planPart) and CTA b
// starts its tasks after the counts of the chunks before it.
__device__ __forceinline__ u32 rlTaskWarps(const DecParams& p, u32 k, u32& s) {
    s = 0;
    if (k >= p.nRl) return 0;
    s = p.rlList[k];
    return u32(ceilDiv(rlBlocksOf(p, p.streams[s]), 32));
}

__global__ void __launch_bounds__(1024) k_decRlTaskCounts(DecParams p) {
    __shared__ u32 scratch[40];
    u32 s, tot;
    const u32 warps = rlTaskWarps(p, blockIdx.x * 1024 + threadIdx.x, s);
    blockExclusiveSum<1024>(warps, scratch, &tot);
    if (threadIdx.x == 0) p.planPart[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(1024) k_decRlTasks(DecParams p) {
    __shared__ u32 scratch[40];
    __shared__ u32 sOff[1024], sStr[1024];   // the chunk's streams: first task, stream index
    __shared__ u32 sCarry;
    const u32 b = blockIdx.x;
    if (threadIdx.x < 32) {
        // tasks of the chunks before this one
        u32 c = 0;
        for (u32 i = threadIdx.x; i < b; i += 32) c += u32(p.planPart[i]);
        c = __reduce_add_sync(0xffffffffu, c);
        if (threadIdx.x == 0) sCarry = c;
    }
    const u32 base = b * 1024;
    u32 s, tot;
    const u32 warps = rlTaskWarps(p, base + threadIdx.x, s);
    const u32 ex = blockExclusiveSum<1024>(warps, scratch, &tot);   // synchronizes (sCarry visible)
    sOff[threadIdx.x] = ex;
    sStr[threadIdx.x] = s;
    __syncthreads();
    const u32 carry = sCarry;
    // the chunk's tasks over all threads: task i belongs to the last stream
    // whose first task is <= i (streams without tasks share their offset
    // with the next one, so that is never one of them)
    const int n = int(min(1024u, p.nRl - base));
    for (u32 i = threadIdx.x; i < tot; i += 1024) {
        int lo = 0, hi = n - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (sOff[mid] <= i) lo = mid;
            else hi = mid - 1;
        }
        const u32 at = carry + i;
        if (at < p.rlTaskCap) p.rlTasks[at] = (u64(sStr[lo]) << 32) | (32u * (i - sOff[lo]));
    }
    if (b + 1 == gridDim.x && threadIdx.x == 0)
        reinterpret_cast<u32*>(p.rlTasks + p.rlTaskCap)[0] = min(carry + tot, p.rlTaskCap);
}

// The RLHuff streams' outputs, zeroed before the symbol pass writes the
// nonzero symbols (so callers need not zero them): CTA (k, c) zeroes chunk c
// of kZeroChunk symbols of RLHuff stream k, 16-byte stores.
constexpr u32 kZeroChunk = 16384;

template <class Sym>
__global__ void __launch_bounds__(256) k_decZero(DecParams p) {
    const DecStreamDesc& sd = p.streams[p.rlList[blockIdx.x]];
    const u64 lo = u64(blockIdx.y) * kZeroChunk;
    if (lo >= sd.n) return;
    const u64 hi = min(u64(sd.n), lo + kZeroChunk);
    Sym* o = reinterpret_cast<Sym*>(sd.out);
    constexpr u64 kPer = 16 / sizeof(Sym);
    const u64 mis = (reinterpret_cast<uintptr_t>(o + lo) & 15u) / sizeof(Sym);
    const u64 head = min(hi - lo, mis ? kPer - mis : 0);
    if (threadIdx.x < head) o[lo + threadIdx.x] = Sym(0);
    const u64 a = lo + head;
    const u64 nv = (hi - a) / kPer;
    uint4* v = reinterpret_cast<uint4*>(o + a);
    for (u64 k = threadIdx.x; k < nv; k += 256) v[k] = make_uint4(0u, 0u, 0u, 0u);
    for (u64 k = a + nv * kPer + threadIdx.x; k < hi; k += 256) o[k] = Sym(0);
}

// decodeRLHuff (RunLengthKernels.cui:56-66 for the scatter): one lane per
// coding block, 32 consecutive blocks of one stream per warp (k_decRlTasks).
// Each lane decodes its block in rounds of kRlRound symbols into its row of
// the warp's shared rows, its bit reader staying in registers between
// rounds; after a round the warp moves the rows out block by block, lane k
// taking the block's element k of the round.  Zero counts (kSymbols false)
// are stored and their (zc + 1) summed per block.  Symbols are scattered to
// out[block start + sum of (zc + 1) before the element + zc]: the round's
// zero counts of the warp's blocks are staged with coalesced loads and a
// warp scan gives the positions.  Lanes read their code words through L1;
// the CTA stages the lookup table of its first warp's stream in shared
// memory (a warp decoding another stream reads its table from global
// memory).  About 13 KB of shared memory per CTA of four warps.
constexpr u32 kRlRound = 32;

struct BitReader {
    u64 w;      // next word
    u32 bpos;   // bit position in hi
    u32 hi, lo;
};

// Decodes cnt symbols from r, calling emit(i, symbol) (decodeBlock's steps).
template <bool kValueLut, class Lut, class Emit>
__device__ __forceinline__ void decodeRun(const WordSrc& ws, const DecTable& D, u32 nSym, const u32* syms,
                                          const Lut& lut, BitReader& r, u32 cnt, bool& corrupt, Emit emit) {
    for (u32 i = 0; i < cnt; ++i) {
        const u32 v = __funnelshift_l(r.lo, r.hi, r.bpos);
        const u32 e = lut(v >> (32 - kLutBits));
        u32 len, val;
        if (e) {
            len = e >> 24;
            val = e & 0xFFFFFFu;
            if (!kValueLut) {
                if (val >= nSym) { corrupt = true; return; }
                val = syms[val];
            }
        } else {
            len = kLutBits + 1;
            while (len <= 31 && int(v >> (32 - len)) > D.maxCode[len - 1]) ++len;
            if (len > 31) { corrupt = true; return; }
            const u32 idx = u32(D.firstIndex[len - 1] + int(v >> (32 - len)) - D.minCode[len - 1]);
            if (idx >= nSym) { corrupt = true; return; }
            val = syms[idx];
        }
        emit(i, val);
        r.bpos += len;
        if (r.bpos >= 32) {
            r.hi = r.lo;
            r.lo = ws.at(r.w);
            ++r.w;
            r.bpos -= 32;
        }
    }
}

template <class Sym, bool kSymbols>
__global__ void __launch_bounds__(128) k_decRl(DecParams p) {
    constexpr u32 kPitch = kRlRound + (sizeof(Sym) == 2 ? 2 : 1);
    __shared__ Sym sRows[4][32 * kPitch];
    __shared__ Sym sZc[kSymbols ? 4 : 1][32 * kRlRound];
    __shared__ u32 sLut[1u << kLutBits];
    __shared__ u32 sLutTable, sFail;
    const u32 lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const u32 wt = blockIdx.x * 4u + warp;
    const bool hasTask = wt < reinterpret_cast<const u32*>(p.rlTasks + p.rlTaskCap)[0];
    u32 s = 0, bFirst = 0, t = 0;
    if (hasTask) {
        const u64 task = p.rlTasks[wt];
        s = u32(task >> 32);
        bFirst = u32(task);
        t = p.streams[s].tableFirst + (kSymbols ? 0u : 1u);
    }
    if (threadIdx.x == 0) {
        sFail = capacityFailed(p) ? 1u : 0u;
        sLutTable = hasTask ? t : 0xFFFFFFFFu;
    }
    __syncthreads();
    if (sFail) return;   // CTA-uniform
    const u32 lutT = sLutTable;
    if (lutT != 0xFFFFFFFFu) {
        const u32* g = p.lut + (u64(lutT) << kLutBits);
        for (u32 e = threadIdx.x; e < (1u << kLutBits); e += 128) sLut[e] = g[e];
    }
    __syncthreads();
    if (!hasTask) return;
    const DecStreamDesc sd = p.streams[s];
    const u32 b = bFirst + lane;
    const u32 blocks = rlBlocksOf(p, sd);
    const bool mine = b < blocks;
    const u32 nMine = __popc(__ballot_sync(0xffffffffu, mine));   // lanes 0 .. nMine-1
    if (nMine == 0) return;
    const DecTableDesc& td = p.tables[t];
    const WordSrc ws = srcOf(p, s);
    const u32* symv = p.syms + td.symOff;
    const u32* lutG = p.lut + (u64(t) << kLutBits);
    const bool lutShared = t == lutT;   // warp-uniform
    const DecTable& D = p.dec[t];
    const u32 nSym = D.nSym;
    const bool single = nSym <= 1;
    const u32 singleVal = D.single;
    bool corrupt = nSym == 0xFFFFFFFFu;
    const u32 cnt = mine ? min(p.cb, sd.m - b * p.cb) : 0u;
    BitReader rd{0ull, 0u, 0u, 0u};
    if (mine && !corrupt && !single) {
        const u64 bit = td.cwWord * 32ull + p.blockOff[td.blockOff + b];
        rd.w = bit >> 5;
        rd.bpos = u32(bit & 31u);
        rd.hi = ws.at(rd.w);
        rd.lo = ws.at(rd.w + 1);
        rd.w += 2;
    }
    u32 sum = 0;   // zero counts: the block's sum of (zc + 1)
    // symbols: the block's next output position (its start from the zero-count scan)
    u32 pos = 0;
    if (kSymbols && mine) pos = p.blockSum[p.tables[t + 1].blockOff + b];
    Sym* rows = sRows[warp];
    const u32 cnt0 = __shfl_sync(0xffffffffu, cnt, 0);   // the first block is the longest
    for (u32 r0 = 0; r0 < cnt0; r0 += kRlRound) {
        const u32 n = cnt > r0 ? min(kRlRound, cnt - r0) : 0u;
        if (!corrupt) {
            auto emit = [&](u32 i, u32 v) {
                rows[lane * kPitch + i] = Sym(v);
                if (!kSymbols) sum += v + 1u;
            };
            if (single) {
                for (u32 i = 0; i < n; ++i) emit(i, singleVal);
            } else if (lutShared) {
                decodeRun<sizeof(Sym) == 2>(ws, D, nSym, symv, [&](u32 k) { return sLut[k]; }, rd, n, corrupt, emit);
            } else {
                decodeRun<sizeof(Sym) == 2>(ws, D, nSym, symv, [&](u32 k) { return lutG[k]; }, rd, n, corrupt, emit);
            }
        }
        __syncwarp();
        const u32 k = r0 + lane;   // the element of every block this lane moves
        if (!kSymbols) {
            Sym* zc = reinterpret_cast<Sym*>(p.zc) + sd.zcOff;
            for (u32 j = 0; j < nMine; ++j) {
                const u32 c = min(p.cb, sd.m - (bFirst + j) * p.cb);
                if (k < c) zc[u64(bFirst + j) * p.cb + k] = rows[j * kPitch + lane];
            }
        } else {
            Sym* zs = sZc[warp];
            const Sym* zcG = reinterpret_cast<const Sym*>(p.zc) + sd.zcOff;
            for (u32 j = 0; j < nMine; ++j) {
                const u32 c = min(p.cb, sd.m - (bFirst + j) * p.cb);
                zs[j * kRlRound + lane] = k < c ? zcG[u64(bFirst + j) * p.cb + k] : Sym(0);
            }
            __syncwarp();
            Sym* out = reinterpret_cast<Sym*>(sd.out);
            for (u32 j = 0; j < nMine; ++j) {
                const u32 c = min(p.cb, sd.m - (bFirst + j) * p.cb);
                const bool act = k < c;
                const u32 z = act ? u32(zs[j * kRlRound + lane]) : 0u;
                const u32 v = act ? z + 1u : 0u;
                u32 incl = v;
#pragma unroll
                for (int d = 1; d < 32; d <<= 1) {
                    const u32 y = __shfl_up_sync(0xffffffffu, incl, d);
                    if (int(lane) >= d) incl += y;
                }
                const u32 at = __shfl_sync(0xffffffffu, pos, j) + incl - v + z;
                if (act) {
                    if (at < sd.n) out[at] = rows[j * kPitch + lane];
                    else corrupt = true;
                }
                const u32 tot = __shfl_sync(0xffffffffu, incl, 31);
                if (lane == j) pos += tot;
            }
        }
        __syncwarp();
    }
    if (!kSymbols && mine) p.blockSum[td.blockOff + b] = sum;
    if (corrupt) atomicOr(p.errors, DEV_ERR_CORRUPT);
}

// Exclusive scan of the per-block output lengths: a warp per RLHuff stream.
__global__ void __launch_bounds__(256) k_decScan(DecParams p) {
    const u32 k = blockIdx.x * 8u + (threadIdx.x >> 5);
    if (k >= p.nRl) return;
    const DecStreamDesc sd = p.streams[p.rlList[k]];
    const u32 blocks = u32(ceilDiv(sd.m, p.cb));
    u32* bs = p.blockSum + p.tables[sd.tableFirst + 1].blockOff;
    const u32 total = warpExclusiveScan8(bs, bs, blocks, 0u);
    // the last symbol's position must be < n: total length <= n
    if ((threadIdx.x & 31u) == 0 && total > sd.n) atomicOr(p.errors, DEV_ERR_CORRUPT);
}

// ---------------------------------------------------------------------------
// Host side.
// ---------------------------------------------------------------------------
struct HostReader {
    const u32* w;
    u32 size;
    u64 pos;
    bool ok = true;
    u32 readBits(u32 n) {
        if (n == 0) return 0;
        if (pos + n > size) { ok = false; pos = size; return 0; }
        u32 v = 0;
        for (u32 k = 0; k < n;) {
            u32 bp = u32(pos & 31u);
            u32 cur = std::min(n - k, 32 - bp);
            u32 bits = (w[pos >> 5] >> (32 - bp - cur)) & (cur == 32 ? 0xffffffffu : ((1u << cur) - 1u));
            v = cur == 32 ? bits : ((v << cur) | bits);
            pos += cur;
            k += cur;
        }
        return v;
    }
    void align() {  // BitStream.h:290-308 (stops at the end)
        u64 a = ceilDiv(pos, 32) * 32;
        pos = std::min<u64>(a, size);
    }
    void skip(u64 n) { pos = std::min<u64>(pos + n, size); }
};

// Parses one table header (HuffmanTable.cu:117-151) into d (bit positions in
// the caller's stream) and returns false on a malformed header.
static bool walkTable(HostReader& r, u32 log2Max, u32 leavesMax, DecTableDesc& d) {
    d.hdrBit = r.pos;
    d.nLen = r.readBits(5);
    r.skip(u64(d.nLen) * log2Max);
    d.nSym = r.readBits(log2Max);
    const bool longSym = log2Max > 16;
    d.symbolBits = r.readBits(longSym ? 5 : 4);
    if (!longSym && d.symbolBits == 0 && d.nSym > 1) d.symbolBits = 16;   // HuffmanTable.cu:138-139
    r.skip(u64(d.nSym) * d.symbolBits);
    return r.ok && d.nSym <= leavesMax;
}

static bool walkPayload(HostReader& r, u32 count, u32 cb, DecTableDesc& d) {
    r.align();
    d.cwBits = r.readBits(32);
    d.cwWord = r.pos / 32;
    r.skip(ceilDiv(d.cwBits, 32) * 32);
    r.align();
    d.offWord = r.pos / 32;
    r.skip(ceilDiv(count, cb) * 16);
    r.align();
    d.count = count;
    return r.ok;
}

// Descriptor layout of one call in a host buffer and in device memory.
struct DecLayout {
    size_t offStreams = 0, offTables, offSources, offRl, offH, bytes;
    DecLayout(u32 S, u32 T, u32 B) {
        offTables = alignUp(sizeof(DecStreamDesc) * S, 64);
        offSources = alignUp(offTables + sizeof(DecTableDesc) * T, 64);
        offRl = alignUp(offSources + sizeof(DecSource) * B, 64);
        offH = alignUp(offRl + sizeof(u32) * S, 64);
        bytes = offH + sizeof(u32) * S;
    }
};

// Fills the stream/table skeleton (kinds, sizes, table and block offsets)
// and the RLHuff / Huff lists of a call.
static int planDecode(cc_instance* I, const u32* kinds, const u32* ns, void* const* outs, const u32* sourceOf, u32 S,
                      u32 B, char* slot, size_t slotBytes, DecPlan& dc) {
    dc = DecPlan{};
    u32 T = 0;
    for (u32 s = 0; s < S; ++s) T += kinds[s] == KIND_RLHUFF ? 2u : 1u;
    const DecLayout L(S, T, B);
    if (S > I->capStreams || T > I->capTables || L.bytes > slotBytes) {
        setError("decode: call exceeds the instance capacity (%u streams)", S);
        return CC_ERR_CAPACITY;
    }
    DecStreamDesc* sd = reinterpret_cast<DecStreamDesc*>(slot + L.offStreams);
    DecTableDesc* td = reinterpret_cast<DecTableDesc*>(slot + L.offTables);
    u32* rl = reinterpret_cast<u32*>(slot + L.offRl);
    u32* hl = reinterpret_cast<u32*>(slot + L.offH);
    u32 t = 0;
    u64 blocks = 0, zc = 0, rlBlocks = 0, hBlocks = 0;
    for (u32 s = 0; s < S; ++s) {
        const u32 nb = u32(ceilDiv(ns[s], I->codingBlockSize));
        DecStreamDesc d{};
        d.out = outs[s];
        d.n = ns[s];
        d.m = ns[s];
        d.kind = kinds[s];
        d.tableFirst = t;
        d.source = sourceOf[s];
        const u32 parts = d.kind == KIND_RLHUFF ? 2u : 1u;
        for (u32 w = 0; w < parts; ++w) {
            DecTableDesc tt{};
            tt.stream = s;
            tt.blockOff = u32(blocks);
            blocks += nb;
            td[t++] = tt;
        }
        if (d.kind == KIND_RLHUFF) {
            d.zcOff = zc;
            zc = alignUp(zc + ns[s], 8);   // 16-byte aligned zero counts of every stream
            d.blockFirst = u32(rlBlocks);
            rlBlocks += nb;
            rl[dc.nRl++] = s;
            dc.rlMaxN = std::max<u32>(dc.rlMaxN, ns[s]);
        } else {
            d.blockFirst = u32(hBlocks);
            hBlocks += nb;
            hl[dc.nH++] = s;
        }
        sd[s] = d;
    }
    if (blocks > I->capBlocks || zc > I->capCompact + 8ull * I->capStreams) {
        setError("decode: call exceeds the instance capacity (%llu coding blocks, %llu run-length symbols)",
                 (unsigned long long)blocks, (unsigned long long)zc);
        return CC_ERR_CAPACITY;
    }
    dc.S = S;
    dc.T = T;
    dc.B = B;
    dc.rlBlocks = u32(rlBlocks);
    dc.hBlocks = u32(hBlocks);
    dc.bytes = L.bytes;
    dc.offStreams = L.offStreams;
    dc.offTables = L.offTables;
    dc.offSources = L.offSources;
    dc.offRl = L.offRl;
    dc.offH = L.offH;
    return CC_OK;
}

template <class Sym>
static int launchDecodeBackEnd(cc_instance* I, const DecParams& p) {
    cudaStream_t st = I->stream;
    {
        SectionTimer t(I, "dec.sym_plan", st);
        const u32 chunks = std::max<u32>(1, u32(ceilDiv(p.T, kPlanChunk)));
        k_decSymPlan<<<chunks, 1024, 0, st>>>(p);
        countLaunch();
        if (chunks > 1) { k_decSymPlanCarry<<<chunks - 1, 1024, 0, st>>>(p); countLaunch(); }
    }
    { SectionTimer t(I, "dec.tables", st); k_decTables<<<p.T, kDecThreads, 0, st>>>(p); countLaunch(); }
    // the Huff streams decode on a side stream beside the RLHuff chain (they
    // share only the read-only tables and the error flags), joined below
    const bool fork = p.hBlocks && p.rlBlocks;
    cudaStream_t hs = fork ? I->buildSide2 : st;
    if (fork) {
        CC_TRY_CUDA(cudaEventRecord(I->decFork, st), "decode fork");
        CC_TRY_CUDA(cudaStreamWaitEvent(hs, I->decFork, 0), "decode fork");
    }
    if (p.hBlocks) {
        const size_t smem = size_t(32) * (p.cb + 2) * sizeof(Sym);
        CC_TRY_CUDA(ensureSmemAttribute(reinterpret_cast<const void*>(k_decHuff<Sym>),
                                        sizeof(Sym) == 2 ? kAttrDecHuff16 : kAttrDecHuff32, I->device, smem),
                    "decHuff smem");
        SectionTimer t(I, "dec.huffman", hs);
        k_decHuff<Sym><<<u32(ceilDiv(p.hBlocks, 32)), 32, smem, hs>>>(p);
        countLaunch();
    }
    if (fork) CC_TRY_CUDA(cudaEventRecord(I->decJoin, hs), "decode join");
    if (p.rlBlocks) {
        const u32 g = u32(ceilDiv(u64(p.rlBlocks) / 32 + p.nRl, 4));   // warp tasks <= rlBlocks / 32 + nRl
        {
            SectionTimer t(I, "dec.rl_tasks", st);
            const u32 chunks = std::max<u32>(1, u32(ceilDiv(p.nRl, 1024)));
            if (chunks > 1) { k_decRlTaskCounts<<<chunks, 1024, 0, st>>>(p); countLaunch(); }
            k_decRlTasks<<<chunks, 1024, 0, st>>>(p);
            countLaunch();
        }
        {
            SectionTimer t(I, "dec.zero_fill", st);
            k_decZero<Sym><<<dim3(p.nRl, u32(ceilDiv(p.rlMaxN, kZeroChunk))), 256, 0, st>>>(p);
            countLaunch();
        }
        { SectionTimer t(I, "dec.zero_counts", st); k_decRl<Sym, false><<<g, 128, 0, st>>>(p); countLaunch(); }
        { SectionTimer t(I, "dec.run_scan", st); k_decScan<<<u32(ceilDiv(p.nRl, 8)), 256, 0, st>>>(p); countLaunch(); }
        { SectionTimer t(I, "dec.symbols_scatter", st); k_decRl<Sym, true><<<g, 128, 0, st>>>(p); countLaunch(); }
    }
    if (fork) CC_TRY_CUDA(cudaStreamWaitEvent(st, I->decJoin, 0), "decode join");
    CC_TRY_CUDA(cudaGetLastError(), "decode launch");
    return CC_OK;
}

int prepareDecodeAttributes(cc_instance* I) {
    const size_t smem = size_t(32) * (I->codingBlockSize + 2) * I->symBytes;
    const int dev = I->device;
    if (I->symBytes == 2) {
        CC_TRY_CUDA(ensureSmemAttribute(reinterpret_cast<const void*>(k_decHuff<u16>), kAttrDecHuff16, dev, smem), "decHuff smem");
    } else {
        CC_TRY_CUDA(ensureSmemAttribute(reinterpret_cast<const void*>(k_decHuff<u32>), kAttrDecHuff32, dev, smem), "decHuff smem");
    }
    return CC_OK;
}

static DecParams makeDecParams(cc_instance* I, const DecPlan& dc) {
    char* d = static_cast<char*>(dc.dev);
    DecParams p{};
    p.S = dc.S;
    p.T = dc.T;
    p.nSrc = dc.B;
    p.nRl = dc.nRl;
    p.nH = dc.nH;
    p.rlBlocks = dc.rlBlocks;
    p.rlMaxN = dc.rlMaxN;
    p.hBlocks = dc.hBlocks;
    p.cb = I->codingBlockSize;
    p.log2Max = I->log2Max;
    p.symBytes = I->symBytes;
    p.leavesMax = I->leavesMax;
    p.capLeaves = I->capLeaves;
    p.streams = reinterpret_cast<DecStreamDesc*>(d + dc.offStreams);
    p.tables = reinterpret_cast<DecTableDesc*>(d + dc.offTables);
    p.sources = reinterpret_cast<DecSource*>(d + dc.offSources);
    p.rlList = reinterpret_cast<const u32*>(d + dc.offRl);
    p.hList = reinterpret_cast<const u32*>(d + dc.offH);
    p.wordsBase = dc.wordsBase;
    p.wordOff = dc.wordOff;
    p.bitSize = dc.bitSize;
    p.dec = I->decTables;
    p.syms = I->decSyms;
    p.lut = I->decLut;
    p.blockOff = I->blockOff;
    p.blockSum = I->blockSum;
    p.rlTasks = I->decRlTasks;
    p.rlTaskCap = u32(u64(I->capBlocks) / 32 + I->capStreams);
    p.zc = static_cast<char*>(I->zc);
    p.planPart = I->planPart + planPartWords(I->capTables);
    p.errors = I->errors + 4;
    return p;
}

// Host-walk front end (cc_decode): the reference's decode entry points.
int decodeDevice(cc_instance* I, int kind, const u32* const* words, const u32* bitSizes, u32* bitPos, u32 bsCount,
                 const u32* bsIndex, void* const* outs, u32 S, u32 n) {
    if (S == 0) return CC_OK;
    if (S > I->streamCountMax) { setError("stream count %u exceeds instance limit %u", S, I->streamCountMax); return CC_ERR_CAPACITY; }
    if (n > I->elemCountPerStreamMax) { setError("symbol count %u exceeds instance limit %u", n, I->elemCountPerStreamMax); return CC_ERR_CAPACITY; }
    std::vector<u32> kinds(S, u32(kind)), ns(S, n), srcOf(S);
    for (u32 s = 0; s < S; ++s) {
        srcOf[s] = bsIndex ? bsIndex[s] : 0u;
        if (srcOf[s] >= bsCount) { setError("decode: bit stream index out of range"); return CC_ERR_INVALID_ARGUMENT; }
    }
    char* slot = I->takeRingSlot();
    DecPlan dc;
    int rc = planDecode(I, kinds.data(), ns.data(), outs, srcOf.data(), S, bsCount, slot, I->hostRingBytes, dc);
    if (rc) return rc;
    const DecLayout L(dc.S, dc.T, dc.B);
    DecStreamDesc* sd = reinterpret_cast<DecStreamDesc*>(slot + L.offStreams);
    DecTableDesc* td = reinterpret_cast<DecTableDesc*>(slot + L.offTables);
    DecSource* src = reinterpret_cast<DecSource*>(slot + L.offSources);
    // walk the headers
    std::vector<u64> lo(bsCount, ~0ull), hi(bsCount, 0);
    std::vector<HostReader> rd(bsCount);
    for (u32 k = 0; k < bsCount; ++k) rd[k] = HostReader{words[k], bitSizes[k], bitPos[k]};
    for (u32 s = 0; s < S; ++s) {
        const u32 k = srcOf[s];
        HostReader& r = rd[k];
        u64 start = r.pos;
        bool ok = true;
        u32 m = n;
        DecTableDesc& t0 = td[sd[s].tableFirst];
        if (kind == KIND_RLHUFF) {
            r.align();
            start = r.pos;
            m = r.readBits(32);
            ok = r.ok && m <= n;
            DecTableDesc& t1 = td[sd[s].tableFirst + 1];
            ok = ok && walkTable(r, I->log2Max, I->leavesMax, t0) && walkPayload(r, m, I->codingBlockSize, t0);
            ok = ok && walkTable(r, I->log2Max, I->leavesMax, t1) && walkPayload(r, m, I->codingBlockSize, t1);
        } else {
            ok = walkTable(r, I->log2Max, I->leavesMax, t0) && walkPayload(r, n, I->codingBlockSize, t0);
        }
        if (!ok) { setError("decode: corrupt or truncated bit stream (stream %u)", s); return CC_ERR_CORRUPT_STREAM; }
        lo[k] = std::min<u64>(lo[k], start / 32);
        hi[k] = std::max<u64>(hi[k], ceilDiv(r.pos, 32));
        sd[s].m = m;
    }
    // stage the touched words of every bit stream and rebase the positions
    std::vector<u64> base(bsCount, 0);
    u64 total = 0;
    for (u32 k = 0; k < bsCount; ++k) {
        if (hi[k] <= lo[k]) continue;
        base[k] = total;
        total += hi[k] - lo[k] + 2;
    }
    if (total > I->stagedWordsMax) { setError("decode: bit stream larger than the instance staging (%llu words)", (unsigned long long)total); return CC_ERR_CAPACITY; }
    cudaStream_t st = I->stream;
    for (u32 k = 0; k < bsCount; ++k) {
        const u64 span = hi[k] > lo[k] ? hi[k] - lo[k] + 2 : 0;
        src[k] = DecSource{I->stagedWords + base[k], span, span * 32, 0, 0, 0, 0};
        if (hi[k] <= lo[k]) continue;
        const u64 nw = std::min<u64>(hi[k], ceilDiv(bitSizes[k], 32)) - lo[k];
        CC_TRY_CUDA(cudaMemcpyAsync(I->stagedWords + base[k], words[k] + lo[k], nw * 4, cudaMemcpyHostToDevice, st), "stage bit stream");
        CC_TRY_CUDA(cudaMemsetAsync(I->stagedWords + base[k] + nw, 0, (span - nw) * 4, st), "pad staging");
    }
    for (u32 t = 0; t < dc.T; ++t) {
        const u32 k = srcOf[td[t].stream];
        td[t].hdrBit -= lo[k] * 32;
        td[t].cwWord -= lo[k];
        td[t].offWord -= lo[k];
    }
    dc.dev = I->dPlan;
    CC_TRY_CUDA(cudaMemcpyAsync(I->dPlan, slot, L.bytes, cudaMemcpyHostToDevice, st), "upload decode plan");
    cudaEventRecord(I->ringEvent[(I->ringNext + cc_instance::kRing - 1) % cc_instance::kRing], st);
    CC_TRY_CUDA(cudaMemsetAsync(I->errors + 4, 0, sizeof(u32), st), "memset errors");
    const DecParams p = makeDecParams(I, dc);
    rc = I->symBytes == 2 ? launchDecodeBackEnd<u16>(I, p) : launchDecodeBackEnd<u32>(I, p);
    if (rc) return rc;
    for (u32 k = 0; k < bsCount; ++k) bitPos[k] = u32(rd[k].pos);
    return CC_OK;
}

// Device-walk front end, step 1: descriptors into `slot`.
int decodePrepare(cc_instance* I, const DecStreamSpec* streams, u32 S, const DecSourceSpec* sources, u32 B,
                  char* slot, size_t slotBytes, DecPlan& dc) {
    std::vector<u32> kinds(S), ns(S), srcOf(S);
    std::vector<void*> outs(S);
    for (u32 s = 0; s < S; ++s) {
        kinds[s] = streams[s].kind;
        ns[s] = streams[s].n;
        outs[s] = streams[s].out;
        srcOf[s] = streams[s].source;
        if (srcOf[s] >= B) { setError("decode: source index out of range"); return CC_ERR_INVALID_ARGUMENT; }
        if (s > 0 && srcOf[s] < srcOf[s - 1]) { setError("decode: streams must be grouped by source"); return CC_ERR_INVALID_ARGUMENT; }
    }
    int rc = planDecode(I, kinds.data(), ns.data(), outs.data(), srcOf.data(), S, B, slot, slotBytes, dc);
    if (rc) return rc;
    const DecLayout L(dc.S, dc.T, dc.B);
    DecSource* src = reinterpret_cast<DecSource*>(slot + L.offSources);
    for (u32 k = 0; k < B; ++k)
        src[k] = DecSource{sources[k].words, ceilDiv(sources[k].bitSize, 32), sources[k].bitSize, sources[k].startBit, 0, 0, 0};
    for (u32 s = 0; s < S; ++s) {
        DecSource& d = src[srcOf[s]];
        if (d.streamCount == 0) d.firstStream = s;
        ++d.streamCount;
    }
    return CC_OK;
}

// Device-walk front end, step 2: the launches (descriptors at dc.dev).
int decodeLaunch(cc_instance* I, const DecPlan& dc) {
    if (dc.S == 0) return CC_OK;
    cudaStream_t st = I->stream;
    CC_TRY_CUDA(cudaMemsetAsync(I->errors + 4, 0, sizeof(u32), st), "memset errors");
    const DecParams p = makeDecParams(I, dc);
    { SectionTimer t(I, "dec.walk", st); k_decWalk<<<u32(ceilDiv(dc.B, 64)), 64, 0, st>>>(p); countLaunch(); }
    return I->symBytes == 2 ? launchDecodeBackEnd<u16>(I, p) : launchDecodeBackEnd<u32>(I, p);
}

}  // namespace ccb

using namespace ccb;

extern "C" {

int cc_decode(cc_instance* I, int kind, int symbolBytes, const uint32_t* const* words, const uint32_t* bitSizes,
              uint32_t* bitPositions, uint32_t bsCount, const uint32_t* bsIndex, void* const* dOut, uint32_t S,
              uint32_t n) {
    if (!I || (S && (!words || !bitSizes || !bitPositions || !dOut || bsCount == 0))) {
        setError("cc_decode: null argument");
        return CC_ERR_INVALID_ARGUMENT;
    }
    if (kind != KIND_RLHUFF && kind != KIND_HUFF) { setError("cc_decode: bad kind %d", kind); return CC_ERR_INVALID_ARGUMENT; }
    if (u32(symbolBytes) != I->symBytes) {
        setError("cc_decode: %d-byte symbols need an instance with log2HuffmanDistinctSymbolCountMax %s 16",
                 symbolBytes, symbolBytes == 2 ? "<=" : ">");
        return CC_ERR_INVALID_ARGUMENT;
    }
    DeviceGuard deviceGuard(I->device);
    return decodeDevice(I, kind, words, bitSizes, bitPositions, bsCount, bsIndex, dOut, S, n);
}

// Reads the device error flags of the last decode (synchronizes the stream).
int cc_decode_status(cc_instance* I) {
    if (!I) return CC_ERR_INVALID_ARGUMENT;
    u32 flags = 0;
    CC_TRY_CUDA(cudaMemcpyAsync(&flags, I->errors + 4, sizeof(u32), cudaMemcpyDeviceToHost, I->stream), "decode status");
    CC_TRY_CUDA(cudaStreamSynchronize(I->stream), "decode status");
    return deviceErrorStatus(flags, "decode");
}

}  // extern "C"
