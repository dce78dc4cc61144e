// decode.cu - device entropy decoder: decodeRLHuff / decodeHuff
// (Encode.cpp:473-646, :792-917; Huffman.cu:189-279; HuffmanTable.cu:117-266;
// RunLength.cu:257-328).
//
// The host only walks the stream headers to find where each table, codeword
// block and offset block lies (O(table size field count) per table); all
// table parsing, offset prefix sums, Huffman decoding and zero-run expansion
// run on the device.  Every read of the staged words is bounds-checked, and
// malformed tables or codes raise CC_ERR_CORRUPT_STREAM instead of reading or
// writing out of bounds.
#include <cstring>

#include "capi_internal.cuh"

namespace ccb {

struct DecParams {
    int kind;
    u32 S;
    u32 cb;
    u32 log2Max;
    u32 symBytes;
    u32 leavesMax;
    u32 blocksMax;
    u64 nStride;
    const u32* words;        // staged bit-stream words
    u64 wordCount;
    const DecTableDesc* tables;
    const DecStreamDesc* streams;
    DecTable* dec;
    u32* syms;               // [T][leavesMax]
    u32* lut;                // [T][1 << kLutBits]
    u32* blockOff;           // [T][blocksMax]  absolute bit offsets
    u32* blockSum;           // [S][blocksMax]
    char* zc;                // decoded zero counts [S][nStride]
    u32* errors;
};

__device__ __forceinline__ u32 wordAt(const DecParams& p, u64 w) { return w < p.wordCount ? p.words[w] : 0u; }

__device__ __forceinline__ u32 readBitsAt(const DecParams& p, u64 bit, u32 count) {
    if (count == 0) return 0;
    const u64 w = bit >> 5;
    const u32 b = u32(bit & 31u);
    const u64 window = (u64(wordAt(p, w)) << 32) | wordAt(p, w + 1);
    return u32((window << b) >> (64 - count));
}

// Table parse and decode structures (HuffmanTable.cu:117-151, :205-266).
constexpr u32 kDecThreads = 256;

__global__ void __launch_bounds__(kDecThreads) k_decTables(DecParams p) {
    __shared__ u32 cpl[32];
    __shared__ int sFirst[32], sMin[32], sMax[32];
    __shared__ u32 sScan[40];
    __shared__ u32 sCarry;
    const u32 t = blockIdx.x;
    const DecTableDesc d = p.tables[t];
    DecTable* D = p.dec + t;
    u32* syms = p.syms + u64(t) * p.leavesMax;
    u32* lut = p.lut + (u64(t) << kLutBits);
    const u64 cntBit = d.hdrBit + 5;
    if (threadIdx.x < 32) cpl[threadIdx.x] = threadIdx.x < d.nLen ? readBitsAt(p, cntBit + u64(threadIdx.x) * p.log2Max, p.log2Max) : 0u;
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
        if (d.nLen == 0) ok = ok && d.nSym <= 1;
        else ok = ok && total == d.nSym;
        if (!ok) atomicOr(p.errors, DEV_ERR_CORRUPT);
        sCarry = ok ? 1u : 0u;
    }
    __syncthreads();
    if (!sCarry) return;
    const u64 symBit = cntBit + u64(d.nLen) * p.log2Max + p.log2Max + (p.log2Max > 16 ? 5u : 4u);
    for (u32 i = threadIdx.x; i < d.nSym; i += kDecThreads) {
        u32 v = readBitsAt(p, symBit + u64(i) * d.symbolBits, d.symbolBits);
        syms[i] = p.symBytes == 2 ? (v & 0xFFFFu) : v;
    }
    // lookup table: first length l <= kLutBits whose prefix fits the canonical range
    for (u32 e = threadIdx.x; e < (1u << kLutBits); e += kDecThreads) {
        u32 entry = 0;
        for (u32 l = 1; l <= kLutBits; ++l) {
            int pref = int(e >> (kLutBits - l));
            if (sMax[l - 1] >= 0 && pref <= sMax[l - 1]) {
                entry = (l << 24) | u32(sFirst[l - 1] + pref - sMin[l - 1]);
                break;
            }
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
        D->single = d.nSym >= 1 ? (p.symBytes == 2 ? readBitsAt(p, symBit, d.symbolBits) & 0xFFFFu : readBitsAt(p, symBit, d.symbolBits)) : 0u;
        sCarry = 0;
    }
    // absolute block offsets: inclusive prefix of the u16 increments (PackInc.cu:220-229)
    const u32 blocks = u32(ceilDiv(d.count, p.cb));
    u32* bo = p.blockOff + u64(t) * p.blocksMax;
    __syncthreads();
    for (u32 base = 0; base < blocks; base += kDecThreads) {
        const u32 k = base + threadIdx.x;
        u32 inc = 0;
        if (k < blocks) {
            const u32 w = wordAt(p, d.offWord + k / 2);
            inc = (k & 1) ? (w >> 16) : (w & 0xFFFFu);
        }
        u32 tot;
        u32 ex = blockExclusiveSum<kDecThreads>(inc, sScan, &tot);
        const u32 off = sCarry + ex + inc;
        if (k < blocks) {
            bo[k] = off;
            if (off > d.cwBits) atomicOr(p.errors, DEV_ERR_CORRUPT);
        }
        __syncthreads();
        if (threadIdx.x == 0) sCarry += tot;
        __syncthreads();
    }
}

// Decodes up to `cnt` symbols of one coding block starting at absolute bit
// `bit`, calling emit(i, symbol).
template <class Emit>
__device__ __forceinline__ void decodeBlock(const DecParams& p, const DecTable& D, const u32* syms, const u32* lut,
                                            u64 bit, u32 cnt, bool& corrupt, Emit emit) {
    if (D.nSym <= 1) {
        for (u32 i = 0; i < cnt; ++i) emit(i, D.single);
        return;
    }
    u64 w = bit >> 5;
    u32 bpos = u32(bit & 31u);
    u64 cache = (u64(wordAt(p, w)) << 32) | wordAt(p, w + 1);
    w += 2;
    for (u32 i = 0; i < cnt; ++i) {
        const u32 v = u32((cache << bpos) >> 32);
        const u32 e = lut[v >> (32 - kLutBits)];
        u32 len, idx;
        if (e) {
            len = e >> 24;
            idx = e & 0xFFFFFFu;
        } else {
            len = kLutBits + 1;
            while (len <= 31 && int(v >> (32 - len)) > D.maxCode[len - 1]) ++len;
            if (len > 31) { corrupt = true; return; }
            idx = u32(D.firstIndex[len - 1] + int(v >> (32 - len)) - D.minCode[len - 1]);
        }
        if (idx >= D.nSym) { corrupt = true; return; }
        emit(i, syms[idx]);
        bpos += len;
        if (bpos >= 32) {
            cache = (cache << 32) | wordAt(p, w);
            ++w;
            bpos -= 32;
        }
    }
}

// decodeHuff: one thread per coding block, output staged through shared
// memory so each warp writes its 32 blocks coalesced.
template <class Sym>
__global__ void __launch_bounds__(32) k_decHuff(DecParams p) {
    extern __shared__ __align__(16) unsigned char stage[];
    const u32 s = blockIdx.y;
    const u32 lane = threadIdx.x;
    const DecStreamDesc sd = p.streams[s];
    const u32 blocks = u32(ceilDiv(sd.n, p.cb));
    const u32 b0 = blockIdx.x * 32;
    if (b0 >= blocks) return;
    const u32 b = b0 + lane;
    const u32 rowPitch = p.cb + (sizeof(Sym) == 2 ? 2 : 1);
    Sym* rows = reinterpret_cast<Sym*>(stage);
    bool corrupt = false;
    __shared__ DecTable D;
    if (lane == 0) D = p.dec[s];
    __syncwarp();
    const u32* syms = p.syms + u64(s) * p.leavesMax;
    const u32* lut = p.lut + (u64(s) << kLutBits);
    if (b < blocks) {
        const u32 i0 = b * p.cb;
        const u32 cnt = min(p.cb, sd.n - i0);
        const u64 bit = p.tables[s].cwWord * 32ull + p.blockOff[u64(s) * p.blocksMax + b];
        decodeBlock(p, D, syms, lut, bit, cnt, corrupt, [&](u32 i, u32 v) { rows[lane * rowPitch + i] = Sym(v); });
    }
    if (corrupt) atomicOr(p.errors, DEV_ERR_CORRUPT);
    __syncwarp();
    Sym* out = reinterpret_cast<Sym*>(sd.out);
    const u32 nb = min(32u, blocks - b0);
    const u64 base = u64(b0) * p.cb;
    const u64 lim = u64(sd.n) - base;
    const u64 total = u64(nb) * p.cb < lim ? u64(nb) * p.cb : lim;
    for (u64 k = lane; k < total; k += 32) out[base + k] = rows[(k / p.cb) * rowPitch + (k % p.cb)];
}

// decodeRLHuff, zero counts: decode and store them, and sum (zc + 1) per block.
template <class Sym>
__global__ void __launch_bounds__(128) k_decZc(DecParams p) {
    const u32 s = blockIdx.y;
    const u32 b = blockIdx.x * blockDim.x + threadIdx.x;
    const DecStreamDesc sd = p.streams[s];
    const u32 blocks = u32(ceilDiv(sd.m, p.cb));
    if (b >= blocks) return;
    const u32 t = p.S + s;
    const DecTable& D = p.dec[t];
    const u32 i0 = b * p.cb;
    const u32 cnt = min(p.cb, sd.m - i0);
    const u64 bit = p.tables[t].cwWord * 32ull + p.blockOff[u64(t) * p.blocksMax + b];
    Sym* zc = reinterpret_cast<Sym*>(p.zc) + u64(s) * p.nStride + i0;
    u32 sum = 0;
    bool corrupt = false;
    decodeBlock(p, D, p.syms + u64(t) * p.leavesMax, p.lut + (u64(t) << kLutBits), bit, cnt, corrupt,
                [&](u32 i, u32 v) { zc[i] = Sym(v); sum += v + 1; });
    if (corrupt) atomicOr(p.errors, DEV_ERR_CORRUPT);
    p.blockSum[u64(s) * p.blocksMax + b] = sum;
}

// Exclusive scan of the per-block output lengths (one block per stream).
__global__ void __launch_bounds__(1024) k_decScan(DecParams p) {
    __shared__ u32 scratch[40];
    __shared__ u32 carry;
    const u32 s = blockIdx.x;
    const DecStreamDesc sd = p.streams[s];
    const u32 blocks = u32(ceilDiv(sd.m, p.cb));
    u32* bs = p.blockSum + u64(s) * p.blocksMax;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (u32 base = 0; base < blocks; base += 1024) {
        const u32 i = base + threadIdx.x;
        const u32 v = i < blocks ? bs[i] : 0u;
        u32 tot;
        const u32 ex = blockExclusiveSum<1024>(v, scratch, &tot);
        if (i < blocks) bs[i] = carry + ex;
        __syncthreads();
        if (threadIdx.x == 0) carry += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0 && carry > sd.n + (sd.m ? 0u : 0u)) {
        // the last symbol's position must be < n: total length <= n
        if (carry > sd.n) atomicOr(p.errors, DEV_ERR_CORRUPT);
    }
}

// decodeRLHuff, symbols: decode and scatter out[scan(zc)+i] = symbol
// (RunLengthKernels.cui:56-66).
template <class Sym>
__global__ void __launch_bounds__(128) k_decSymScatter(DecParams p) {
    const u32 s = blockIdx.y;
    const u32 b = blockIdx.x * blockDim.x + threadIdx.x;
    const DecStreamDesc sd = p.streams[s];
    const u32 blocks = u32(ceilDiv(sd.m, p.cb));
    if (b >= blocks) return;
    const u32 t = s;
    const DecTable& D = p.dec[t];
    const u32 i0 = b * p.cb;
    const u32 cnt = min(p.cb, sd.m - i0);
    const u64 bit = p.tables[t].cwWord * 32ull + p.blockOff[u64(t) * p.blocksMax + b];
    const Sym* zc = reinterpret_cast<const Sym*>(p.zc) + u64(s) * p.nStride + i0;
    Sym* out = reinterpret_cast<Sym*>(sd.out);
    u32 pos = p.blockSum[u64(s) * p.blocksMax + b];
    bool corrupt = false;
    decodeBlock(p, D, p.syms + u64(t) * p.leavesMax, p.lut + (u64(t) << kLutBits), bit, cnt, corrupt,
                [&](u32 i, u32 v) {
                    pos += u32(zc[i]);
                    if (pos < sd.n) out[pos] = Sym(v);
                    else corrupt = true;
                    ++pos;
                });
    if (corrupt) atomicOr(p.errors, DEV_ERR_CORRUPT);
}

// ---------------------------------------------------------------------------
// Host side: header walk over the caller's bit streams.
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

template <class Sym>
static int launchDecode(cc_instance* I, const DecParams& p, u32 nMax, u32 mMax) {
    cudaStream_t st = I->stream;
    const u32 T = p.kind == KIND_RLHUFF ? 2 * p.S : p.S;
    { SectionTimer t(I, "dec.tables", st); k_decTables<<<T, kDecThreads, 0, st>>>(p); countLaunch(); }
    if (p.kind == KIND_HUFF) {
        const u32 blocks = std::max<u32>(1u, u32(ceilDiv(nMax, p.cb)));
        const size_t smem = size_t(32) * (p.cb + 2) * sizeof(Sym);
        CC_TRY_CUDA(cudaFuncSetAttribute(k_decHuff<Sym>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)), "decHuff smem");
        { SectionTimer t(I, "dec.huffman", st); k_decHuff<Sym><<<dim3(u32(ceilDiv(blocks, 32)), p.S), 32, smem, st>>>(p); countLaunch(); }
    } else {
        const u32 blocks = std::max<u32>(1u, u32(ceilDiv(mMax, p.cb)));
        dim3 g(u32(ceilDiv(blocks, 128)), p.S);
        { SectionTimer t(I, "dec.zero_counts", st); k_decZc<Sym><<<g, 128, 0, st>>>(p); countLaunch(); }
        { SectionTimer t(I, "dec.run_scan", st); k_decScan<<<p.S, 1024, 0, st>>>(p); countLaunch(); }
        { SectionTimer t(I, "dec.symbols_scatter", st); k_decSymScatter<Sym><<<g, 128, 0, st>>>(p); countLaunch(); }
    }
    CC_TRY_CUDA(cudaGetLastError(), "decode launch");
    return CC_OK;
}

int decodeDevice(cc_instance* I, int kind, const u32* const* words, const u32* bitSizes, u32* bitPos, u32 bsCount,
                 const u32* bsIndex, void* const* outs, u32 S, u32 n) {
    if (S == 0) return CC_OK;
    if (S > I->streamCountMax) { setError("stream count %u exceeds instance limit %u", S, I->streamCountMax); return CC_ERR_CAPACITY; }
    if (n > I->elemCountPerStreamMax) { setError("symbol count %u exceeds instance limit %u", n, I->elemCountPerStreamMax); return CC_ERR_CAPACITY; }
    const u32 T = kind == KIND_RLHUFF ? 2 * S : S;
    char* slot = I->takeRingSlot();
    DecTableDesc* td = reinterpret_cast<DecTableDesc*>(slot);
    DecStreamDesc* sd = reinterpret_cast<DecStreamDesc*>(slot + alignUp(sizeof(DecTableDesc) * T, 64));
    // walk the headers
    std::vector<u64> lo(bsCount, ~0ull), hi(bsCount, 0);
    std::vector<HostReader> rd(bsCount);
    for (u32 k = 0; k < bsCount; ++k) rd[k] = HostReader{words[k], bitSizes[k], bitPos[k]};
    u32 mMax = 0;
    for (u32 s = 0; s < S; ++s) {
        const u32 k = bsIndex ? bsIndex[s] : 0u;
        if (k >= bsCount) { setError("decode: bit stream index out of range"); return CC_ERR_INVALID_ARGUMENT; }
        HostReader& r = rd[k];
        u64 start = r.pos;
        bool ok = true;
        u32 m = n;
        if (kind == KIND_RLHUFF) {
            r.align();
            start = r.pos;
            m = r.readBits(32);
            ok = r.ok && m <= n;
            ok = ok && walkTable(r, I->log2Max, I->leavesMax, td[s]) && walkPayload(r, m, I->codingBlockSize, td[s]);
            ok = ok && walkTable(r, I->log2Max, I->leavesMax, td[S + s]) && walkPayload(r, m, I->codingBlockSize, td[S + s]);
        } else {
            ok = walkTable(r, I->log2Max, I->leavesMax, td[s]) && walkPayload(r, n, I->codingBlockSize, td[s]);
        }
        if (!ok) { setError("decode: corrupt or truncated bit stream (stream %u)", s); return CC_ERR_CORRUPT_STREAM; }
        lo[k] = std::min<u64>(lo[k], start / 32);
        hi[k] = std::max<u64>(hi[k], ceilDiv(r.pos, 32));
        sd[s].out = outs[s];
        sd[s].n = n;
        sd[s].m = m;
        mMax = std::max(mMax, m);
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
        if (hi[k] <= lo[k]) continue;
        const u64 nw = std::min<u64>(hi[k], ceilDiv(bitSizes[k], 32)) - lo[k];
        CC_TRY_CUDA(cudaMemcpyAsync(I->stagedWords + base[k], words[k] + lo[k], nw * 4, cudaMemcpyHostToDevice, st), "stage bit stream");
        CC_TRY_CUDA(cudaMemsetAsync(I->stagedWords + base[k] + nw, 0, (hi[k] - lo[k] + 2 - nw) * 4, st), "pad staging");
    }
    for (u32 t = 0; t < T; ++t) {
        const u32 s = t < S ? t : t - S;
        const u32 k = bsIndex ? bsIndex[s] : 0u;
        const u64 shiftBits = (lo[k] - base[k]) * 32;
        td[t].hdrBit -= shiftBits;
        td[t].cwWord -= lo[k] - base[k];
        td[t].offWord -= lo[k] - base[k];
    }
    CC_TRY_CUDA(cudaMemcpyAsync(I->dDecTables, td, sizeof(DecTableDesc) * T, cudaMemcpyHostToDevice, st), "upload tables");
    CC_TRY_CUDA(cudaMemcpyAsync(I->dDecStreams, sd, sizeof(DecStreamDesc) * S, cudaMemcpyHostToDevice, st), "upload streams");
    cudaEventRecord(I->ringEvent[(I->ringNext + cc_instance::kRing - 1) % cc_instance::kRing], st);
    CC_TRY_CUDA(cudaMemsetAsync(I->errors + 4, 0, sizeof(u32), st), "memset errors");
    DecParams p{};
    p.kind = kind;
    p.S = S;
    p.cb = I->codingBlockSize;
    p.log2Max = I->log2Max;
    p.symBytes = I->symBytes;
    p.leavesMax = I->leavesMax;
    p.blocksMax = I->blocksMax;
    p.nStride = I->elemCountPerStreamMax;
    p.words = I->stagedWords;
    p.wordCount = total;
    p.tables = I->dDecTables;
    p.streams = I->dDecStreams;
    p.dec = I->decTables;
    p.syms = I->decSyms;
    p.lut = I->decLut;
    p.blockOff = I->blockOff;
    p.blockSum = I->blockSum;
    p.zc = static_cast<char*>(I->zc);
    p.errors = I->errors + 4;
    int rc = I->symBytes == 2 ? launchDecode<u16>(I, p, n, mMax) : launchDecode<u32>(I, p, n, mMax);
    if (rc) return rc;
    for (u32 k = 0; k < bsCount; ++k) bitPos[k] = u32(rd[k].pos);
    return CC_OK;
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
    cudaSetDevice(I->device);
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
