// oracle.cpp - CPU restatement of cudaCompress's compress/decompress hot path.
//
// TEST INFRASTRUCTURE ONLY.  This is the checker for the CUDA product library
// (cudacompress_b200).  Only tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline / reference arm may load it; the product library never links it.
//
// Every function restates the reference algorithm it cites (paths relative to
// the cudaCompress project root).  Where the reference's observable output is
// decided by the C++ standard library (Huffman tree tie-breaks and the order of
// equal-length symbols), this file uses the same std:: containers and
// algorithms with the same comparators, so that a build with the same
// libstdc++ reproduces the reference byte for byte.
//
// Build: oracle/Makefile -> oracle/liboracle.so (g++ -O2 -ffp-contract=off).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <queue>
#include <vector>

#include <omp.h>

typedef uint32_t u32;
typedef uint16_t u16;
typedef int16_t i16;
typedef uint8_t u8;

namespace orc {

// ---------------------------------------------------------------------------
// Bit stream (include/cudaCompress/BitStream.h:14-494).
// Bits are MSB-first inside little-endian u32 words; *Aligned writes align to
// 4 bytes before and after and memcpy raw bytes (BitStream.h:420-455).
// ---------------------------------------------------------------------------
struct BitStream {
    std::vector<u32> buf;
    u32 bitSize = 0;
    u32 pos = 0;

    void resizeWords(u32 words) { buf.resize(words, 0u); }

    // BitStream.h:377-418
    void writeBits(u32 data, u32 count) {
        u32 newSize = pos + count;
        if (newSize > bitSize) {
            bitSize = newSize;
            u32 w = (bitSize + 31) / 32;
            if (w > buf.size()) resizeWords(w);
        }
        while (count > 0) {
            u32 bitPos = pos % 32;
            u32 cur = std::min(count, 32 - bitPos);
            u32 mask = cur == 32 ? ~0u : ((1u << cur) - 1u);
            u32 value = (data >> (count - cur)) & mask;
            u32 shift = 32 - cur - bitPos;
            u32& word = buf[pos / 32];
            word = (word & ~(mask << shift)) | (value << shift);
            pos += cur;
            count -= cur;
        }
    }
    // BitStream.h:463-480
    void writeAlign(u32 bytes) {
        u32 bits = bytes * 8;
        u32 off = pos % bits;
        if (off) pos += bits - off;
        if (pos > bitSize) {
            bitSize = pos;
            resizeWords((bitSize + 31) / 32);
        }
    }
    // BitStream.h:420-455
    void writeAligned(const void* src, u32 elemSize, u32 count) {
        writeAlign(4);
        writeAlign(elemSize);
        if (count == 0) return;
        u32 start = pos;
        pos += count * elemSize * 8;
        if (pos > bitSize) {
            bitSize = pos;
            resizeWords((bitSize + 31) / 32);
        }
        std::memcpy(reinterpret_cast<uint8_t*>(buf.data()) + start / 8, src, size_t(count) * elemSize);
        writeAlign(4);
    }
};

struct BitReader {
    const u32* buf;
    u32 bitSize;
    u32 pos;
    // BitStream.h:169-200
    u32 readBits(u32 count) {
        u32 avail = bitSize - pos;
        if (count > avail) count = avail;
        u32 data = 0;
        while (count > 0) {
            u32 bitPos = pos % 32;
            u32 cur = std::min(count, 32 - bitPos);
            u32 mask = cur == 32 ? ~0u : ((1u << cur) - 1u);
            u32 v = (buf[pos / 32] >> (32 - cur - bitPos)) & mask;
            data |= v << (count - cur);
            pos += cur;
            count -= cur;
        }
        return data;
    }
    // BitStream.h:290-308
    bool align(u32 bytes) {
        u32 bits = bytes * 8;
        u32 off = pos % bits;
        u32 offMax = bitSize - pos;
        bool ok = true;
        if (off > offMax) { off = offMax; ok = false; }
        if (off) pos += bits - off;
        return ok;
    }
    // BitStream.h:213-241
    u32 readAligned(void* dst, u32 elemSize, u32 count) {
        align(4);
        align(elemSize);
        u32 bytesAvail = (bitSize - pos) / 8;
        u32 n = std::min(bytesAvail / elemSize, count);
        std::memcpy(dst, reinterpret_cast<const uint8_t*>(buf) + pos / 8, size_t(n) * elemSize);
        pos += n * elemSize * 8;
        align(4);
        return n;
    }
    const u32* alignedPtr() { align(4); return buf + pos / 32; }
    // BitStream.h:243-262 (skipAligned)
    void skipAligned(u32 elemSize, u32 count) {
        align(4);
        align(elemSize);
        u32 bytesAvail = (bitSize - pos) / 8;
        u32 n = std::min(bytesAvail / elemSize, count);
        pos += n * elemSize * 8;
        align(4);
    }
    void skipBits(u32 count) { pos += std::min(count, bitSize - pos); }
};

// util.h:23-32
static u32 requiredBits(u32 v) {
    u32 b = 0;
    while (v > 0) { ++b; v >>= 1; }
    return b;
}

// ---------------------------------------------------------------------------
// Huffman table design (HuffmanTable.cu:487-596, HuffmanDesign.h:13-63).
// ---------------------------------------------------------------------------
struct Node {
    u32 symbol;
    u32 prob;
    int len;
    Node* left;
    Node* right;
    void init(u32 s, u32 p) { symbol = s; prob = p; len = -1; left = right = nullptr; }
    // HuffmanDesign.h:27-39 (recursive depth assignment, same visiting order)
    int assign(int l) {
        len = l;
        int r = l;
        if (left) r = std::max(r, left->assign(l + 1));
        if (right) r = std::max(r, right->assign(l + 1));
        return r;
    }
};
// HuffmanDesign.h:42-51
struct ProbInvLess {
    bool operator()(const Node* a, const Node* b) const { return b->prob < a->prob; }
};
// HuffmanDesign.h:53-60
struct LenLess {
    bool operator()(const Node* a, const Node* b) const { return a->len < b->len; }
};

struct EncodeTable {
    u32 symbolMax = 0;
    std::vector<u32> symbols;            // by codeword index (length order)
    std::vector<u32> countPerLength;     // index = length-1
    std::vector<u32> codewords;          // by symbol, size symbolMax+1
    std::vector<u32> lengths;            // by symbol (0xFFFFFFFF = unused)
};

// HuffmanTable.cu:487-596
static void buildTable(EncodeTable& t, const u32* prob, u32 distinct) {
    t.symbols.clear();
    t.countPerLength.clear();
    std::vector<Node> nodes(distinct ? 2 * distinct - 1 : 1);
    u32 next = 0;
    std::vector<Node*> leaves;
    for (u32 s = 0; s < distinct; ++s) {
        if (prob[s] > 0) {
            nodes[next].init(s, prob[s]);
            leaves.push_back(&nodes[next]);
            ++next;
        }
    }
    t.codewords.assign(distinct, 0u);
    t.lengths.assign(distinct, 0xFFFFFFFFu);
    if (leaves.empty()) return;
    // range construction: heap built by make_heap over the leaves (HuffmanTable.cu:507)
    std::priority_queue<Node*, std::vector<Node*>, ProbInvLess> todo(leaves.begin(), leaves.end());
    while (todo.size() > 1) {
        Node& nn = nodes[next++];
        nn.init(0xFFFFFFFFu, 0);
        Node* l = todo.top(); todo.pop();
        Node* r = todo.top(); todo.pop();
        nn.left = l;
        nn.right = r;
        nn.prob = l->prob + r->prob;
        todo.push(&nn);
    }
    Node& root = *todo.top();
    u32 maxLen = u32(root.assign(0));
    std::sort(leaves.begin(), leaves.end(), LenLess());   // HuffmanTable.cu:538
    t.countPerLength.assign(maxLen, 0u);
    t.symbols.resize(leaves.size());
    for (size_t i = 0; i < leaves.size(); ++i) {
        if (leaves[i]->len > 0) t.countPerLength[leaves[i]->len - 1]++;
        t.symbols[i] = leaves[i]->symbol;
    }
    u32 count = 0;
    for (u32 c : t.countPerLength) count += c;
    if (t.countPerLength.empty()) count = 1;
    std::vector<u32> lenByIndex(count), cwByIndex(count);
    if (!t.countPerLength.empty()) {
        u32 idx = 0;
        for (u32 l = 1; l <= maxLen; ++l)
            for (u32 i = 0; i < t.countPerLength[l - 1]; ++i) lenByIndex[idx++] = l;
    } else {
        lenByIndex[0] = 0;
    }
    cwByIndex[0] = 0;
    for (u32 i = 1; i < count; ++i) {
        cwByIndex[i] = cwByIndex[i - 1] + 1;
        cwByIndex[i] <<= (lenByIndex[i] - lenByIndex[i - 1]);
    }
    for (u32 i = 0; i < count; ++i) {
        t.codewords[t.symbols[i]] = cwByIndex[i];
        t.lengths[t.symbols[i]] = lenByIndex[i];
    }
}

// HuffmanTable.cu:470-485
static void writeTable(const EncodeTable& t, BitStream& bs, u32 log2Max) {
    bool longSym = log2Max > 16;
    bs.writeBits(u32(t.countPerLength.size()), 5);
    for (u32 c : t.countPerLength) bs.writeBits(c, log2Max);
    bs.writeBits(u32(t.symbols.size()), log2Max);
    u32 symbolBits = requiredBits(t.symbolMax);
    bs.writeBits(symbolBits, longSym ? 5 : 4);
    for (u32 s : t.symbols) bs.writeBits(s, symbolBits);
}

struct DecodeTable {
    std::vector<u32> symbols;
    int firstIndex[32], minCode[32], maxCode[32];
};

// HuffmanTable.cu:117-151 and :205-266
static void readTable(DecodeTable& d, BitReader& br, u32 log2Max) {
    for (int i = 0; i < 32; ++i) d.firstIndex[i] = d.minCode[i] = d.maxCode[i] = -1;
    bool longSym = log2Max > 16;
    u32 nLen = br.readBits(5);
    std::vector<u32> cpl(nLen);
    for (u32 i = 0; i < nLen; ++i) cpl[i] = br.readBits(log2Max);
    u32 nSym = br.readBits(log2Max);
    u32 symbolBits = br.readBits(longSym ? 5 : 4);
    if (!longSym && symbolBits == 0 && nSym > 1) symbolBits = 16;   // HuffmanTable.cu:138-139
    d.symbols.resize(nSym);
    for (u32 i = 0; i < nSym; ++i) {
        u32 s = br.readBits(symbolBits);
        d.symbols[i] = longSym ? s : (s & 0xFFFFu);
    }
    if (nSym == 0) return;
    u32 count = 0;
    for (u32 c : cpl) count += c;
    if (cpl.empty()) count = 1;
    std::vector<u32> lens;
    for (u32 i = 0; i < nLen; ++i) lens.insert(lens.end(), cpl[i], i + 1);
    std::vector<int> cw(1, 0);
    for (u32 i = 1; i < count && i < lens.size(); ++i) {
        int c = cw[i - 1] + 1;
        c <<= (lens[i] - lens[i - 1]);
        cw.push_back(c);
    }
    for (u32 l = 0, e = 0; l < nLen; ++l) {
        if (cpl[l] > 0) {
            d.firstIndex[l] = int(e);
            d.minCode[l] = cw[e];
            e += cpl[l] - 1;
            d.maxCode[l] = cw[e];
            ++e;
        }
    }
}

// ---------------------------------------------------------------------------
// Histogram (Histogram.cu:90-289, HistogramKernels.cui:38-250).
// Counts values in [0, bins).  Input is padded with all-ones up to a multiple
// of 8 elements (Histogram.cu:90-106); the 16-bit large-bin kernels read whole
// u32 words, so when bins == 65536 the one padding 0xFFFF inside the last word
// of an odd-length stream is counted (HistogramKernels.cui:165,200).
// ---------------------------------------------------------------------------
template <typename S>
static void histogram(const S* data, u32 count, u32 bins, u32* hist) {
    std::fill(hist, hist + bins, 0u);
    for (u32 i = 0; i < count; ++i)
        if (u32(data[i]) < bins) hist[data[i]]++;
    if (sizeof(S) == 2 && bins == 65536 && (count & 1)) hist[65535]++;
}

// HuffmanTable.cu:385-447 (design over several streams at once)
template <typename S>
static bool designTables(std::vector<EncodeTable>& tables, const std::vector<const S*>& streams,
                         const std::vector<u32>& counts, u32 log2Max, bool allEmptyZeroCountQuirk,
                         u32 quirkStreamCount) {
    u32 n = u32(streams.size());
    tables.assign(n, EncodeTable());
    u32 globalMax = 0;
    u32 countMax = 0;
    for (u32 i = 0; i < n; ++i) {
        u32 m = 0;
        for (u32 k = 0; k < counts[i]; ++k) m = std::max<u32>(m, streams[i][k]);
        tables[i].symbolMax = m;
        globalMax = std::max(globalMax, m);
        countMax = std::max(countMax, counts[i]);
    }
    u32 distinct = globalMax + 1;
    if (distinct > (1u << log2Max)) return false;   // HuffmanTable.cu:411-419
    std::vector<u32> hist(distinct);
    for (u32 i = 0; i < n; ++i) {
        u32 d = tables[i].symbolMax + 1;
        if (countMax == 0) {
            // Histogram.cu:117-121 returns before touching the histogram
            // buffers when every stream is empty; the table is then built from
            // whatever the arena holds there.  For the zero-count tables of an
            // encodeRLHuff call that is the low word of the symbol-stream
            // pointer of the HuffmanGPUStreamInfo array left there by the
            // preceding huffmanEncode (64-byte records, 128-byte histogram
            // slots: table i reads record 2+2i); elsewhere it is the all-zero
            // run-length scan output.
            hist[0] = (allEmptyZeroCountQuirk && 2 + 2 * i < quirkStreamCount) ? 1u : 0u;
        } else {
            histogram(streams[i], counts[i], d, hist.data());
        }
        buildTable(tables[i], hist.data(), d);
    }
    return true;
}

// ---------------------------------------------------------------------------
// Huffman encode/decode of one stream (HuffmanKernels.cui:35-190 semantics,
// Huffman.cu:73-187): MSB-first packing, coding-block bit offsets.
// ---------------------------------------------------------------------------
template <typename S>
static void huffEncode(const EncodeTable& t, const S* sym, u32 count, u32 cb,
                       std::vector<u32>& words, u32& bits, std::vector<u32>& offsets) {
    BitStream bs;
    offsets.clear();
    for (u32 i = 0; i < count; ++i) {
        if (i % cb == 0) offsets.push_back(bs.pos);
        u32 s = sym[i];
        if (t.lengths[s]) bs.writeBits(t.codewords[s], t.lengths[s]);
    }
    bits = bs.pos;
    words = bs.buf;
    words.resize((bits + 31) / 32);
}

template <typename S>
static void huffDecode(const DecodeTable& d, const u32* words, u32 bitSize, u32 count, S* out) {
    if (d.symbols.size() <= 1) {
        S v = d.symbols.empty() ? S(0) : S(d.symbols[0]);
        for (u32 i = 0; i < count; ++i) out[i] = v;
        return;
    }
    BitReader br{words, bitSize, 0};
    for (u32 i = 0; i < count; ++i) {
        int len = 0, code = 0;
        do {
            code = (code << 1) | int(br.readBits(1));
            ++len;
        } while (len < 32 && code > d.maxCode[len - 1]);
        out[i] = S(d.symbols[d.firstIndex[len - 1] + code - d.minCode[len - 1]]);
    }
}

// PackInc.cu:210-229
static void packInc16(const std::vector<u32>& off, std::vector<u16>& inc) {
    inc.resize(off.size());
    u32 prev = off.empty() ? 0 : off[0];
    if (!off.empty()) inc[0] = u16(prev);
    for (size_t i = 1; i < off.size(); ++i) { inc[i] = u16(off[i] - prev); prev = off[i]; }
}

// ---------------------------------------------------------------------------
// Zero-run RLE (RunLength.cu:82-188, RunLengthKernels.cui:5-45).
// ---------------------------------------------------------------------------
template <typename S>
static void rleEncode(const S* sym, u32 n, std::vector<S>& compact, std::vector<S>& zc) {
    compact.clear();
    zc.clear();
    u32 run = 0;
    for (u32 i = 0; i < n; ++i) {
        if (sym[i] == 0) { ++run; continue; }
        for (u32 k = 0; k < run / 256; ++k) { compact.push_back(0); zc.push_back(S(255)); }
        compact.push_back(sym[i]);
        zc.push_back(S(run % 256));
        run = 0;
    }
}

// RunLengthKernels.cui:56-77 (inclusive scan of zero counts, scatter)
template <typename S>
static void rleDecode(const S* compact, const S* zc, u32 m, S* out, u32 n) {
    std::fill(out, out + n, S(0));
    uint64_t idx = 0;
    for (u32 i = 0; i < m; ++i) {
        idx += zc[i];
        if (idx < n) out[idx] = compact[i];
        ++idx;
    }
}

static u32 numOffsets(u32 count, u32 cb) { return (count + cb - 1) / cb; }

// ---------------------------------------------------------------------------
// encodeRLHuff / encodeHuff / decodeRLHuff / decodeHuff (Encode.cpp:207-917).
// ---------------------------------------------------------------------------
template <typename S>
static int encodeRLHuff(BitStream& bs, const std::vector<const S*>& streams, u32 n, u32 cb, u32 log2Max) {
    u32 S_ = u32(streams.size());
    std::vector<std::vector<S>> comp(S_), zcs(S_);
    std::vector<u32> counts(S_);
    std::vector<const S*> pc(S_), pz(S_);
    for (u32 i = 0; i < S_; ++i) {
        rleEncode(streams[i], n, comp[i], zcs[i]);
        counts[i] = u32(comp[i].size());
        pc[i] = comp[i].data();
        pz[i] = zcs[i].data();
    }
    std::vector<EncodeTable> tSym, tZc;
    if (!designTables(tSym, pc, counts, log2Max, false, S_)) return -1;
    if (!designTables(tZc, pz, counts, log2Max, true, S_)) return -1;
    for (u32 i = 0; i < S_; ++i) {
        if (tSym[i].countPerLength.size() > 31 || tZc[i].countPerLength.size() > 31) return -3;
    }
    for (u32 i = 0; i < S_; ++i) {
        std::vector<u32> words, off;
        std::vector<u16> inc;
        u32 bits;
        bs.writeAligned(&counts[i], 4, 1);
        writeTable(tSym[i], bs, log2Max);
        huffEncode(tSym[i], pc[i], counts[i], cb, words, bits, off);
        bs.writeAligned(&bits, 4, 1);
        bs.writeAligned(words.data(), 4, u32(words.size()));
        packInc16(off, inc);
        bs.writeAligned(inc.data(), 2, u32(inc.size()));
        writeTable(tZc[i], bs, log2Max);
        huffEncode(tZc[i], pz[i], counts[i], cb, words, bits, off);
        bs.writeAligned(&bits, 4, 1);
        bs.writeAligned(words.data(), 4, u32(words.size()));
        packInc16(off, inc);
        bs.writeAligned(inc.data(), 2, u32(inc.size()));
    }
    return 0;
}

template <typename S>
static int encodeHuff(BitStream& bs, const std::vector<const S*>& streams, u32 n, u32 cb, u32 log2Max) {
    u32 S_ = u32(streams.size());
    std::vector<u32> counts(S_, n);
    std::vector<EncodeTable> t;
    if (!designTables(t, streams, counts, log2Max, false, S_)) return -1;
    for (u32 i = 0; i < S_; ++i)
        if (t[i].countPerLength.size() > 31) return -3;
    for (u32 i = 0; i < S_; ++i) {
        std::vector<u32> words, off;
        std::vector<u16> inc;
        u32 bits;
        writeTable(t[i], bs, log2Max);
        huffEncode(t[i], streams[i], n, cb, words, bits, off);
        bs.writeAligned(&bits, 4, 1);
        bs.writeAligned(words.data(), 4, u32(words.size()));
        packInc16(off, inc);
        bs.writeAligned(inc.data(), 2, u32(inc.size()));
    }
    return 0;
}

template <typename S>
static void decodeStreamPayload(BitReader& br, u32 log2Max, u32 count, u32 cb, S* out) {
    DecodeTable d;
    readTable(d, br, log2Max);
    u32 bits = 0;
    br.readAligned(&bits, 4, 1);
    const u32* cw = br.buf + br.pos / 32;
    u32 words = (bits + 31) / 32;
    br.skipBits(words * 32);
    br.align(4);
    br.skipAligned(2, numOffsets(count, cb));
    huffDecode(d, cw, bits, count, out);
}

template <typename S>
static void decodeRLHuff(BitReader& br, std::vector<S*> outs, u32 n, u32 cb, u32 log2Max) {
    for (S* out : outs) {
        u32 m = 0;
        br.readAligned(&m, 4, 1);
        std::vector<S> comp(m), zc(m);
        decodeStreamPayload(br, log2Max, m, cb, comp.data());
        decodeStreamPayload(br, log2Max, m, cb, zc.data());
        rleDecode(comp.data(), zc.data(), m, out, n);
    }
}

template <typename S>
static void decodeHuff(BitReader& br, std::vector<S*> outs, u32 n, u32 cb, u32 log2Max) {
    for (S* out : outs) decodeStreamPayload(br, log2Max, n, cb, out);
}

// ---------------------------------------------------------------------------
// Float DWT (util/DWTFloatKernels.cui, util/DWTFloatFilters.cuh:42-49,
// util/DWTCommon.cuh:54-55).  Every axis pass is a 9-tap FIR with
// whole-sample symmetric extension; output tap set chosen by the parity of the
// output position; fp32 FMA chain sum = fma(c[i], v[i], sum), i = 0..8, from
// 0.0f (DWTFloatKernels.cui:68-79).  Forward writes even->[0,N/2), odd->[N/2,N);
// inverse reads the halves as the interleaved signal.
// ---------------------------------------------------------------------------
static const float kFwd[2][9] = {
    {0.0267488f, -0.0168641f, -0.0782233f, 0.2668641f, 0.6029490f, 0.2668641f, -0.0782233f, -0.0168641f, 0.0267488f},
    {0.0f, 0.0456359f, -0.0287718f, -0.2956359f, 0.5575435f, -0.2956359f, -0.0287718f, 0.0456359f, 0.0f}};
static const float kInv[2][9] = {
    {0.0f, 0.0337282f, -0.0575435f, -0.5337281f, 1.1150871f, -0.5337281f, -0.0575435f, 0.0337282f, 0.0f},
    {0.0534975f, -0.0912718f, -0.1564465f, 0.5912718f, 1.2058980f, 0.5912718f, -0.1564465f, -0.0912718f, 0.0534975f}};

static inline long mirror(long i, long n) {
    if (i < 0) i = -i;
    if (i > n - 1) i = 2 * (n - 1) - i;
    return i;
}

// One axis pass over a dense array with extent (nx, ny, nz); axis 0/1/2.
template <typename T>
static void firAxis(const T* src, T* dst, long nx, long ny, long nz, int axis, bool inverse) {
    long n = axis == 0 ? nx : axis == 1 ? ny : nz;
    long stride = axis == 0 ? 1 : axis == 1 ? nx : nx * ny;
    long h = n / 2;
    long lines = nx * ny * nz / n;
#pragma omp parallel
    {
    std::vector<T> line(n), outl(n);
#pragma omp for schedule(static)
    for (long li = 0; li < lines; ++li) {
        long base;
        if (axis == 0) base = li * nx;
        else if (axis == 1) base = (li / nx) * nx * ny + (li % nx);
        else base = li;
        // gather the signal in the filtering domain
        for (long k = 0; k < n; ++k) {
            if (!inverse) line[k] = src[base + k * stride];
            else line[k] = src[base + ((k & 1) ? (h + k / 2) : (k / 2)) * stride];
        }
        for (long x = 0; x < n; ++x) {
            const float* c = inverse ? kInv[x & 1] : kFwd[x & 1];
            T sum = T(0);
            for (int i = 0; i < 9; ++i) {
                T v = line[mirror(x + i - 4, n)];
                if (sizeof(T) == 4) sum = T(std::fmaf(c[i], float(v), float(sum)));
                else sum = std::fma(double(c[i]), double(v), double(sum));
            }
            outl[x] = sum;
        }
        for (long x = 0; x < n; ++x) {
            long o = inverse ? x : ((x & 1) ? (h + x / 2) : (x / 2));
            dst[base + o * stride] = outl[x];
        }
    }
    }
}

// DWTFloat.cu:84-202 (X, Y, Z) and :204-323 (Z, Y, X)
template <typename T>
static void dwtFloat(const T* src, T* dst, long nx, long ny, long nz, bool inverse) {
    std::vector<T> a(src, src + nx * ny * nz), b(a.size());
    int axes[3] = {0, 1, 2};
    int nAxes = nz > 1 ? 3 : 2;
    if (inverse) { if (nAxes == 3) { axes[0] = 2; axes[1] = 1; axes[2] = 0; } else { axes[0] = 1; axes[1] = 0; } }
    for (int k = 0; k < nAxes; ++k) {
        firAxis(a.data(), b.data(), nx, ny, nz, axes[k], inverse);
        std::swap(a, b);
    }
    std::copy(a.begin(), a.end(), dst);
}

// ---------------------------------------------------------------------------
// Integer CDF 5/3 lifting (util/DWTIntKernels.cui:14-101 forward,
// :596-686 inverse; rounding util/DWTCommon.cuh:133-142).  All arithmetic
// narrows to short exactly where the reference does.
// ---------------------------------------------------------------------------
static inline i16 div2(i16 v) { v = i16(v + ((v >= 0) ? 1 : -1)); return i16(v / 2); }
static inline i16 div4(i16 v) { v = i16(v + ((v >= 0) ? 2 : -2)); return i16(v / 4); }

// DWTInt.cu:111-135 with DWTIntKernels.cui:104-200 (and the inverse,
// DWTInt.cu:271-310, DWTIntKernels.cui:596-780): the X pass lifts whole
// 256-sample blocks, then the remainder in 32-sample blocks of which the
// kernel's predict/update loops cover only whole pairs (blockCount/2).  With
// an odd count of remainder blocks the last one is not lifted: its samples
// are only split into the L and H halves.  Y and Z passes lift every sample.
static long xLiftEnd(long n) {
    long done = n / 256 * 256, rest = n - done, blocks = (rest + 31) / 32;
    return std::min(n, done + 64 * (blocks / 2));
}

static void liftAxis(const i16* src, i16* dst, long nx, long ny, long nz, int axis, bool inverse) {
    long n = axis == 0 ? nx : axis == 1 ? ny : nz;
    const long end = axis == 0 ? xLiftEnd(n) : n;   // samples at or beyond `end` stay unlifted
    long stride = axis == 0 ? 1 : axis == 1 ? nx : nx * ny;
    long h = n / 2;
    long lines = nx * ny * nz / n;
#pragma omp parallel
    {
    std::vector<i16> s(n + 2);
#pragma omp for schedule(static)
    for (long li = 0; li < lines; ++li) {
        long base;
        if (axis == 0) base = li * nx;
        else if (axis == 1) base = (li / nx) * nx * ny + (li % nx);
        else base = li;
        if (!inverse) {
            for (long k = 0; k < n; ++k) s[k] = src[base + k * stride];
            for (long k = 1; k < end; k += 2) {
                i16 r = (k + 1 < n) ? s[k + 1] : s[n - 2];
                s[k] = i16(s[k] - div2(i16(s[k - 1] + r)));
            }
            for (long k = 0; k < end; k += 2) {
                i16 l = (k > 0) ? s[k - 1] : s[1];
                s[k] = i16(s[k] + div4(i16(l + s[k + 1])));
            }
            for (long k = 0; k < n; ++k) dst[base + ((k & 1) ? (h + k / 2) : (k / 2)) * stride] = s[k];
        } else {
            for (long k = 0; k < n; ++k) s[k] = src[base + ((k & 1) ? (h + k / 2) : (k / 2)) * stride];
            for (long k = 0; k < end; k += 2) {
                i16 l = (k > 0) ? s[k - 1] : s[1];
                s[k] = i16(s[k] - div4(i16(l + s[k + 1])));
            }
            for (long k = 1; k < end; k += 2) {
                i16 r = (k + 1 < n) ? s[k + 1] : s[n - 2];
                s[k] = i16(s[k] + div2(i16(s[k - 1] + r)));
            }
            for (long k = 0; k < n; ++k) dst[base + k * stride] = s[k];
        }
    }
    }
}

// DWTInt.cu:79-187 (X, Y[, Z]) and :189-317 ([Z,] Y, X)
static void dwtInt(const i16* src, i16* dst, long nx, long ny, long nz, bool inverse) {
    std::vector<i16> a(src, src + nx * ny * nz), b(a.size());
    int axes[3] = {0, 1, 2};
    int nAxes = nz > 1 ? 3 : 2;
    if (inverse) { if (nAxes == 3) { axes[0] = 2; axes[1] = 1; axes[2] = 0; } else { axes[0] = 1; axes[1] = 0; } }
    for (int k = 0; k < nAxes; ++k) {
        liftAxis(a.data(), b.data(), nx, ny, nz, axes[k], inverse);
        std::swap(a, b);
    }
    std::copy(a.begin(), a.end(), dst);
}

// ---------------------------------------------------------------------------
// Quantization (util/Quantize.cuh:55-147, util/Quantize.cu:78-100).
// ---------------------------------------------------------------------------
// Quantize.cuh:26-35,55-59: 2|v| + getNegativeSign(v), where getNegativeSign is
// -1 for negative values: v >= 0 -> 2v (even), v < 0 -> 2|v|-1 (odd).
static inline u32 symbolize(int v) { return 2u * u32(std::abs(v)) - (v < 0 ? 1u : 0u); }
static inline int unsymbolize(u32 s) { int neg = int(s % 2); return (1 - 2 * neg) * int((s + u32(neg)) / 2); }
static inline int quantDeadzone(float v, float inv) { return int(v * inv); }                  // Quantize.cuh:75-82
static inline float unquantDeadzone(int q, float step) {                                     // Quantize.cuh:104-110
    float sg = q > 0 ? 1.0f : (q < 0 ? -1.0f : 0.0f);
    return (float(q) + sg * 0.5f) * step;
}

// Extract band (bx,by,bz) of a level volume in [L|H] layout as symbols.
template <typename S>
static void quantizeBand(const float* lvl, long n0, long n1, long n2, int bx, int by, int bz, float step, S* out) {
    float inv = 1.0f / step;   // Quantize.cu:90 (host reciprocal)
    long hx = n0 / 2, hy = n1 / 2, hz = n2 > 1 ? n2 / 2 : 1;
    for (long z = 0; z < hz; ++z)
        for (long y = 0; y < hy; ++y)
            for (long x = 0; x < hx; ++x) {
                float v = lvl[(z + bz * hz) * n0 * n1 + (y + by * hy) * n0 + (x + bx * hx)];
                out[(z * hy + y) * hx + x] = S(symbolize(quantDeadzone(v, inv)));
            }
}
template <typename S>
static void unquantizeBand(float* lvl, long n0, long n1, long n2, int bx, int by, int bz, float step, const S* in) {
    long hx = n0 / 2, hy = n1 / 2, hz = n2 > 1 ? n2 / 2 : 1;
    for (long z = 0; z < hz; ++z)
        for (long y = 0; y < hy; ++y)
            for (long x = 0; x < hx; ++x)
                lvl[(z + bz * hz) * n0 * n1 + (y + by * hy) * n0 + (x + bx * hx)] =
                    unquantDeadzone(unsymbolize(in[(z * hy + y) * hx + x]), step);
}

}  // namespace orc

using namespace orc;

// ===========================================================================
// C ABI for the Python test harness.
// ===========================================================================
extern "C" {

// 1-level DWTs on dense arrays in the reference's [L|H]-per-axis layout.
void orc_dwt_float_fwd(const float* src, float* dst, long nx, long ny, long nz) { dwtFloat(src, dst, nx, ny, nz, false); }
void orc_dwt_float_inv(const float* src, float* dst, long nx, long ny, long nz) { dwtFloat(src, dst, nx, ny, nz, true); }
void orc_dwt_double_fwd(const double* src, double* dst, long nx, long ny, long nz) { dwtFloat(src, dst, nx, ny, nz, false); }
void orc_dwt_double_inv(const double* src, double* dst, long nx, long ny, long nz) { dwtFloat(src, dst, nx, ny, nz, true); }
void orc_dwt_int_fwd(const i16* src, i16* dst, long nx, long ny, long nz) { dwtInt(src, dst, nx, ny, nz, false); }
void orc_dwt_int_inv(const i16* src, i16* dst, long nx, long ny, long nz) { dwtInt(src, dst, nx, ny, nz, true); }

// Threads of the OpenMP loops (the CPU baseline's single- and all-core runs).
void orc_set_threads(int n) { omp_set_num_threads(n > 0 ? n : 1); }

// getMaxAbs (util/Quantize.cu:355-361): reduceArray with OperatorMax over
// FunctorAbs (reduce/reduce_app.cui:122-142, tools/Operator.h:31-52,
// tools/Functor.h:25-29), whose identity is -FLT_MAX.
float orc_max_abs(const float* src, long n) {
    float m = -3.40282347e38f;
    for (long i = 0; i < n; ++i) m = std::max(m, std::fabs(src[i]));
    return m;
}

// Quantize.cu:78-100 on a dense (nx,ny,nz) block with the reference's pitches.
void orc_quantize_to_symbols16(u16* out, const float* src, long nx, long ny, long nz, float step, long rowPitch, long slicePitch) {
    float inv = 1.0f / step;
#pragma omp parallel for schedule(static)
    for (long z = 0; z < nz; ++z)
        for (long y = 0; y < ny; ++y)
            for (long x = 0; x < nx; ++x)
                out[(z * ny + y) * nx + x] = u16(symbolize(quantDeadzone(src[z * slicePitch + y * rowPitch + x], inv)));
}
void orc_unquantize_from_symbols16(float* dst, const u16* in, long nx, long ny, long nz, float step, long rowPitch, long slicePitch) {
    for (long z = 0; z < nz; ++z)
        for (long y = 0; y < ny; ++y)
            for (long x = 0; x < nx; ++x)
                dst[z * slicePitch + y * rowPitch + x] = unquantDeadzone(unsymbolize(in[(z * ny + y) * nx + x]), step);
}

// Zero-run RLE of one stream; returns the compact count.
u32 orc_rle_encode16(const u16* sym, u32 n, u16* compact, u16* zc) {
    std::vector<u16> c, z;
    rleEncode(sym, n, c, z);
    std::copy(c.begin(), c.end(), compact);
    std::copy(z.begin(), z.end(), zc);
    return u32(c.size());
}

// Build one table from a histogram; returns code/length by symbol and the
// serialized table (fresh bit stream).  Returns the max codeword length.
int orc_huffman_build(const u32* hist, u32 bins, u32 symbolMax, u32 log2Max, u32* codewords, u32* lengths,
                      u32* tableWords, u32 tableCap, u32* tableBits) {
    EncodeTable t;
    t.symbolMax = symbolMax;
    buildTable(t, hist, bins);
    for (u32 i = 0; i < bins; ++i) { codewords[i] = t.codewords[i]; lengths[i] = t.lengths[i]; }
    BitStream bs;
    writeTable(t, bs, log2Max);
    *tableBits = bs.bitSize;
    if (bs.buf.size() > tableCap) return -2;
    std::copy(bs.buf.begin(), bs.buf.end(), tableWords);
    return int(t.countPerLength.size());
}

// Shared state for the codec entry points: an in/out bit stream.
static int finishBits(const BitStream& bs, u32* words, u32 cap, u32* bitSize, u32* bitPos) {
    if (bs.buf.size() > cap) return -2;
    std::copy(bs.buf.begin(), bs.buf.end(), words);
    *bitSize = bs.bitSize;
    *bitPos = bs.pos;
    return 0;
}

// kind: 0 = encodeRLHuff, 1 = encodeHuff.  symBytes: 2 or 4.  Streams are
// contiguous: stream i at symbols + i*n.  The bit stream starts from
// (words, *bitSize, *bitPos) and is appended to as the reference would.
int orc_encode(int kind, int symBytes, const void* symbols, u32 streamCount, u32 n, u32 cb, u32 log2Max,
               u32* words, u32 cap, u32* bitSize, u32* bitPos) {
    BitStream bs;
    bs.bitSize = *bitSize;
    bs.pos = *bitPos;
    bs.buf.assign(words, words + (bs.bitSize + 31) / 32);
    int r;
    if (symBytes == 2) {
        std::vector<const u16*> s(streamCount);
        for (u32 i = 0; i < streamCount; ++i) s[i] = static_cast<const u16*>(symbols) + size_t(i) * n;
        r = kind == 0 ? encodeRLHuff(bs, s, n, cb, log2Max) : encodeHuff(bs, s, n, cb, log2Max);
    } else {
        std::vector<const u32*> s(streamCount);
        for (u32 i = 0; i < streamCount; ++i) s[i] = static_cast<const u32*>(symbols) + size_t(i) * n;
        r = kind == 0 ? encodeRLHuff(bs, s, n, cb, log2Max) : encodeHuff(bs, s, n, cb, log2Max);
    }
    if (r) return r;
    return finishBits(bs, words, cap, bitSize, bitPos);
}

int orc_decode(int kind, int symBytes, const u32* words, u32 bitSize, u32* bitPos, void* out, u32 streamCount,
               u32 n, u32 cb, u32 log2Max) {
    BitReader br{words, bitSize, *bitPos};
    if (symBytes == 2) {
        std::vector<u16*> o(streamCount);
        for (u32 i = 0; i < streamCount; ++i) o[i] = static_cast<u16*>(out) + size_t(i) * n;
        if (kind == 0) decodeRLHuff(br, o, n, cb, log2Max); else decodeHuff(br, o, n, cb, log2Max);
    } else {
        std::vector<u32*> o(streamCount);
        for (u32 i = 0; i < streamCount; ++i) o[i] = static_cast<u32*>(out) + size_t(i) * n;
        if (kind == 0) decodeRLHuff(br, o, n, cb, log2Max); else decodeHuff(br, o, n, cb, log2Max);
    }
    *bitPos = br.pos;
    return 0;
}

// ---------------------------------------------------------------------------
// Lossy volume codec (examples CompressVolume.cpp:312-409 / :411-516):
// multi-level 3D DWT, deadzone quantization with step q0/2^level (LP uses the
// coarsest step), LP band encodeHuff, then per level coarse->fine the 7 HP
// bands (index x+2y+4z) with encodeRLHuff.  Symbol16 streams.
// ---------------------------------------------------------------------------
int orc_compress_volume_float_ex(const float* vol, long nx, long ny, long nz, int levels, float q0, u32 cb,
                                 u32 log2Max, int rleOnlyLevel0, u32* words, u32 cap, u32* bitSize) {
    std::vector<std::vector<float>> lv(levels);
    std::vector<float> cur(vol, vol + nx * ny * nz);
    long sx = nx, sy = ny, sz = nz;
    for (int l = 0; l < levels; ++l) {
        lv[l].resize(sx * sy * sz);
        dwtFloat(cur.data(), lv[l].data(), sx, sy, sz, false);
        long hx = sx / 2, hy = sy / 2, hz = sz / 2;
        cur.resize(hx * hy * hz);
        for (long z = 0; z < hz; ++z)
            for (long y = 0; y < hy; ++y)
                for (long x = 0; x < hx; ++x) cur[(z * hy + y) * hx + x] = lv[l][(z * sy + y) * sx + x];
        sx = hx; sy = hy; sz = hz;
    }
    BitStream bs;
    float stepLP = q0 / float(1 << (levels - 1));
    {
        std::vector<u16> lp(cur.size());
        orc_quantize_to_symbols16(lp.data(), cur.data(), sx, sy, sz, stepLP, sx, sx * sy);
        std::vector<const u16*> s(1, lp.data());
        int r = encodeHuff(bs, s, u32(lp.size()), cb, log2Max);
        if (r) return r;
    }
    for (int l = levels - 1; l >= 0; --l) {
        long n0 = nx >> l, n1 = ny >> l, n2 = nz >> l;
        float step = q0 / float(1 << l);
        long bandN = (n0 / 2) * (n1 / 2) * (n2 / 2);
        std::vector<u16> bands(7 * bandN);
        std::vector<const u16*> s(7);
        for (int b = 1; b < 8; ++b) {
            quantizeBand(lv[l].data(), n0, n1, n2, b % 2, (b / 2) % 2, b / 4, step, bands.data() + (b - 1) * bandN);
            s[b - 1] = bands.data() + (b - 1) * bandN;
        }
        // CompressVolume.cpp:389-395: with doRLEOnlyOnLvl0 the levels above 0 skip the RLE
        int r = (rleOnlyLevel0 && l > 0) ? encodeHuff(bs, s, u32(bandN), cb, log2Max)
                                         : encodeRLHuff(bs, s, u32(bandN), cb, log2Max);
        if (r) return r;
    }
    u32 pos;
    return finishBits(bs, words, cap, bitSize, &pos);
}

int orc_compress_volume_float(const float* vol, long nx, long ny, long nz, int levels, float q0, u32 cb,
                              u32 log2Max, u32* words, u32 cap, u32* bitSize) {
    return orc_compress_volume_float_ex(vol, nx, ny, nz, levels, q0, cb, log2Max, 0, words, cap, bitSize);
}

int orc_decompress_volume_float_ex(const u32* words, u32 bitSize, float* out, long nx, long ny, long nz, int levels,
                                   float q0, u32 cb, u32 log2Max, int rleOnlyLevel0) {
    BitReader br{words, bitSize, 0};
    long sx = nx >> levels, sy = ny >> levels, sz = nz >> levels;
    std::vector<u16> lp(sx * sy * sz);
    std::vector<u16*> o(1, lp.data());
    decodeHuff(br, o, u32(lp.size()), cb, log2Max);
    std::vector<float> cur(lp.size());
    orc_unquantize_from_symbols16(cur.data(), lp.data(), sx, sy, sz, q0 / float(1 << (levels - 1)), sx, sx * sy);
    for (int l = levels - 1; l >= 0; --l) {
        long n0 = nx >> l, n1 = ny >> l, n2 = nz >> l;
        long bandN = (n0 / 2) * (n1 / 2) * (n2 / 2);
        std::vector<u16> bands(7 * bandN);
        std::vector<u16*> ob(7);
        for (int b = 0; b < 7; ++b) ob[b] = bands.data() + b * bandN;
        if (rleOnlyLevel0 && l > 0) decodeHuff(br, ob, u32(bandN), cb, log2Max);   // CompressVolume.cpp:491-495
        else decodeRLHuff(br, ob, u32(bandN), cb, log2Max);
        float step = q0 / float(1 << l);
        std::vector<float> coef(n0 * n1 * n2);
        for (long z = 0; z < n2 / 2; ++z)
            for (long y = 0; y < n1 / 2; ++y)
                for (long x = 0; x < n0 / 2; ++x)
                    coef[(z * n1 + y) * n0 + x] = cur[(z * (n1 / 2) + y) * (n0 / 2) + x];
        for (int b = 1; b < 8; ++b)
            unquantizeBand(coef.data(), n0, n1, n2, b % 2, (b / 2) % 2, b / 4, step, ob[b - 1]);
        cur.resize(coef.size());
        dwtFloat(coef.data(), cur.data(), n0, n1, n2, true);
    }
    std::copy(cur.begin(), cur.end(), out);
    return 0;
}

int orc_decompress_volume_float(const u32* words, u32 bitSize, float* out, long nx, long ny, long nz, int levels,
                                float q0, u32 cb, u32 log2Max) {
    return orc_decompress_volume_float_ex(words, bitSize, out, nx, ny, nz, levels, q0, cb, log2Max, 0);
}

// ---------------------------------------------------------------------------
// Quantize-first lossy volume codec (examples CompressVolume.cpp:651-757 /
// :759-856): uniform quantization of the whole volume to short
// (Quantize.cuh:86-93, int(v * (1/step) + sign(v) * 0.5), restated with the
// product contracted into one fma), then an integer 5/3 DWT per level on the
// LLL region of the previous level, the final lowpass symbolized and
// encodeHuff'd, and per level coarse -> fine the 7 highpass bands (index
// x+2y+4z) symbolized and encodeRLHuff'd (encodeHuff above level 0 with
// doRLEOnlyOnLvl0).  Decoding inverts the levels coarse -> fine and
// unquantizes q * step (Quantize.cuh:113-119).
// ---------------------------------------------------------------------------
static inline i16 quantUniform(float v, float inv) {
    const float s = v > 0.0f ? 1.0f : (v < 0.0f ? -1.0f : 0.0f);
    return i16(int(std::fmaf(v, inv, s * 0.5f)));
}

int orc_compress_volume_quantfirst(const float* vol, long nx, long ny, long nz, int levels, float step, u32 cb,
                                   u32 log2Max, int rleOnlyLevel0, u32* words, u32 cap, u32* bitSize) {
    const float inv = 1.0f / step;   // Quantize.cu:236: reciprocal on the host
    std::vector<i16> cur(nx * ny * nz);
    for (long i = 0; i < nx * ny * nz; ++i) cur[i] = quantUniform(vol[i], inv);
    std::vector<std::vector<i16>> lv(levels);
    long sx = nx, sy = ny, sz = nz;
    for (int l = 0; l < levels; ++l) {
        lv[l].resize(sx * sy * sz);
        dwtInt(cur.data(), lv[l].data(), sx, sy, sz, false);
        long hx = sx / 2, hy = sy / 2, hz = sz / 2;
        cur.resize(hx * hy * hz);
        for (long z = 0; z < hz; ++z)
            for (long y = 0; y < hy; ++y)
                for (long x = 0; x < hx; ++x) cur[(z * hy + y) * hx + x] = lv[l][(z * sy + y) * sx + x];
        sx = hx; sy = hy; sz = hz;
    }
    BitStream bs;
    {
        std::vector<u16> lp(cur.size());
        for (size_t i = 0; i < cur.size(); ++i) lp[i] = u16(symbolize(cur[i]));
        std::vector<const u16*> s(1, lp.data());
        int r = encodeHuff(bs, s, u32(lp.size()), cb, log2Max);
        if (r) return r;
    }
    for (int l = levels - 1; l >= 0; --l) {
        long n0 = nx >> l, n1 = ny >> l, n2 = nz >> l;
        long hx = n0 / 2, hy = n1 / 2, hz = n2 / 2, bandN = hx * hy * hz;
        std::vector<u16> bands(7 * bandN);
        std::vector<const u16*> s(7);
        for (int b = 1; b < 8; ++b) {
            const long bx = b % 2, by = (b / 2) % 2, bz = b / 4;
            u16* o = bands.data() + (b - 1) * bandN;
            for (long z = 0; z < hz; ++z)
                for (long y = 0; y < hy; ++y)
                    for (long x = 0; x < hx; ++x)
                        o[(z * hy + y) * hx + x] = u16(symbolize(lv[l][((z + bz * hz) * n1 + (y + by * hy)) * n0 + x + bx * hx]));
            s[b - 1] = o;
        }
        int r = (rleOnlyLevel0 && l > 0) ? encodeHuff(bs, s, u32(bandN), cb, log2Max)
                                         : encodeRLHuff(bs, s, u32(bandN), cb, log2Max);
        if (r) return r;
    }
    u32 pos;
    return finishBits(bs, words, cap, bitSize, &pos);
}

int orc_decompress_volume_quantfirst(const u32* words, u32 bitSize, float* out, long nx, long ny, long nz,
                                     int levels, float step, u32 cb, u32 log2Max, int rleOnlyLevel0) {
    BitReader br{words, bitSize, 0};
    long sx = nx >> levels, sy = ny >> levels, sz = nz >> levels;
    std::vector<u16> lp(sx * sy * sz);
    std::vector<u16*> o(1, lp.data());
    decodeHuff(br, o, u32(lp.size()), cb, log2Max);
    std::vector<i16> cur(lp.size());
    for (size_t i = 0; i < lp.size(); ++i) cur[i] = i16(unsymbolize(lp[i]));
    for (int l = levels - 1; l >= 0; --l) {
        long n0 = nx >> l, n1 = ny >> l, n2 = nz >> l;
        long hx = n0 / 2, hy = n1 / 2, hz = n2 / 2, bandN = hx * hy * hz;
        std::vector<u16> bands(7 * bandN);
        std::vector<u16*> ob(7);
        for (int b = 0; b < 7; ++b) ob[b] = bands.data() + b * bandN;
        if (rleOnlyLevel0 && l > 0) decodeHuff(br, ob, u32(bandN), cb, log2Max);
        else decodeRLHuff(br, ob, u32(bandN), cb, log2Max);
        std::vector<i16> coef(n0 * n1 * n2);
        for (long z = 0; z < hz; ++z)
            for (long y = 0; y < hy; ++y)
                for (long x = 0; x < hx; ++x) coef[(z * n1 + y) * n0 + x] = cur[(z * hy + y) * hx + x];
        for (int b = 1; b < 8; ++b) {
            const long bx = b % 2, by = (b / 2) % 2, bz = b / 4;
            for (long z = 0; z < hz; ++z)
                for (long y = 0; y < hy; ++y)
                    for (long x = 0; x < hx; ++x)
                        coef[((z + bz * hz) * n1 + (y + by * hy)) * n0 + x + bx * hx] =
                            i16(unsymbolize(ob[b - 1][(z * hy + y) * hx + x]));
        }
        cur.resize(coef.size());
        dwtInt(coef.data(), cur.data(), n0, n1, n2, true);
    }
    for (long i = 0; i < nx * ny * nz; ++i) out[i] = float(cur[i]) * step;
    return 0;
}

// Multi-level quantized coefficients only (parity of the symbol streams):
// writes the LP symbols then, per level coarse->fine, the 7 HP band streams.
void orc_volume_symbols(const float* vol, long nx, long ny, long nz, int levels, float q0, u16* out) {
    std::vector<float> cur(vol, vol + nx * ny * nz);
    std::vector<std::vector<float>> lv(levels);
    long sx = nx, sy = ny, sz = nz;
    for (int l = 0; l < levels; ++l) {
        lv[l].resize(sx * sy * sz);
        dwtFloat(cur.data(), lv[l].data(), sx, sy, sz, false);
        long hx = sx / 2, hy = sy / 2, hz = sz / 2;
        cur.resize(hx * hy * hz);
        for (long z = 0; z < hz; ++z)
            for (long y = 0; y < hy; ++y)
                for (long x = 0; x < hx; ++x) cur[(z * hy + y) * hx + x] = lv[l][(z * sy + y) * sx + x];
        sx = hx; sy = hy; sz = hz;
    }
    orc_quantize_to_symbols16(out, cur.data(), sx, sy, sz, q0 / float(1 << (levels - 1)), sx, sx * sy);
    out += sx * sy * sz;
    for (int l = levels - 1; l >= 0; --l) {
        long n0 = nx >> l, n1 = ny >> l, n2 = nz >> l;
        long bandN = (n0 / 2) * (n1 / 2) * (n2 / 2);
        for (int b = 1; b < 8; ++b) {
            quantizeBand(lv[l].data(), n0, n1, n2, b % 2, (b / 2) % 2, b / 4, q0 / float(1 << l), out);
            out += bandN;
        }
    }
}

// Inverse of orc_volume_symbols: dequantize LP + bands, inverse DWT per level.
void orc_volume_from_symbols(const u16* syms, float* out, long nx, long ny, long nz, int levels, float q0) {
    long sx = nx >> levels, sy = ny >> levels, sz = nz >> levels;
    std::vector<float> cur(sx * sy * sz);
    orc_unquantize_from_symbols16(cur.data(), syms, sx, sy, sz, q0 / float(1 << (levels - 1)), sx, sx * sy);
    syms += sx * sy * sz;
    for (int l = levels - 1; l >= 0; --l) {
        long n0 = nx >> l, n1 = ny >> l, n2 = nz >> l;
        long bandN = (n0 / 2) * (n1 / 2) * (n2 / 2);
        float step = q0 / float(1 << l);
        std::vector<float> coef(n0 * n1 * n2);
        for (long z = 0; z < n2 / 2; ++z)
            for (long y = 0; y < n1 / 2; ++y)
                for (long x = 0; x < n0 / 2; ++x)
                    coef[(z * n1 + y) * n0 + x] = cur[(z * (n1 / 2) + y) * (n0 / 2) + x];
        for (int b = 1; b < 8; ++b) {
            unquantizeBand(coef.data(), n0, n1, n2, b % 2, (b / 2) % 2, b / 4, step, syms);
            syms += bandN;
        }
        cur.resize(coef.size());
        dwtFloat(coef.data(), cur.data(), n0, n1, n2, true);
    }
    std::copy(cur.begin(), cur.end(), out);
}

// ---------------------------------------------------------------------------
// Lossless 2D heightfield codec (config "2048^2 int16, 4 levels"): per level
// an integer 5/3 2D DWT, 3 HP bands (index x+2y, CompressHeightfield.cpp:
// 116-126) symbolized and encodeRLHuff'd; the final LP symbolized and
// encodeHuff'd; stream order LP, then levels coarse->fine
// (CompressVolume.cpp:234-277).
// ---------------------------------------------------------------------------
int orc_compress_heightfield(const i16* img, long nx, long ny, int levels, u32 cb, u32 log2Max, u32* words,
                             u32 cap, u32* bitSize) {
    std::vector<i16> cur(img, img + nx * ny);
    std::vector<BitStream> lvBits(levels);
    long sx = nx, sy = ny;
    for (int l = 0; l < levels; ++l) {
        std::vector<i16> c(sx * sy);
        dwtInt(cur.data(), c.data(), sx, sy, 1, false);
        long hx = sx / 2, hy = sy / 2;
        std::vector<u16> bands(3 * hx * hy);
        std::vector<const u16*> s(3);
        for (int b = 1; b < 4; ++b) {
            for (long y = 0; y < hy; ++y)
                for (long x = 0; x < hx; ++x)
                    bands[(b - 1) * hx * hy + y * hx + x] = u16(symbolize(c[(y + (b / 2) * hy) * sx + x + (b % 2) * hx]));
            s[b - 1] = bands.data() + (b - 1) * hx * hy;
        }
        int r = encodeRLHuff(lvBits[l], s, u32(hx * hy), cb, log2Max);
        if (r) return r;
        cur.resize(hx * hy);
        for (long y = 0; y < hy; ++y)
            for (long x = 0; x < hx; ++x) cur[y * hx + x] = c[y * sx + x];
        sx = hx; sy = hy;
    }
    BitStream bs;
    std::vector<u16> lp(cur.size());
    for (size_t i = 0; i < cur.size(); ++i) lp[i] = u16(symbolize(cur[i]));
    std::vector<const u16*> s(1, lp.data());
    int r = encodeHuff(bs, s, u32(lp.size()), cb, log2Max);
    if (r) return r;
    for (int l = levels - 1; l >= 0; --l) {
        bs.writeAlign(4);
        u32 start = bs.pos / 32;
        u32 w = u32(lvBits[l].buf.size());
        bs.resizeWords(start + w);
        std::copy(lvBits[l].buf.begin(), lvBits[l].buf.end(), bs.buf.begin() + start);
        bs.pos = bs.bitSize = (start + w) * 32;
    }
    u32 pos;
    return finishBits(bs, words, cap, bitSize, &pos);
}

int orc_decompress_heightfield(const u32* words, u32 bitSize, i16* out, long nx, long ny, int levels, u32 cb,
                               u32 log2Max) {
    BitReader br{words, bitSize, 0};
    long sx = nx >> levels, sy = ny >> levels;
    std::vector<u16> lp(sx * sy);
    std::vector<u16*> o(1, lp.data());
    decodeHuff(br, o, u32(lp.size()), cb, log2Max);
    br.align(4);
    std::vector<i16> cur(lp.size());
    for (size_t i = 0; i < lp.size(); ++i) cur[i] = i16(unsymbolize(lp[i]));
    for (int l = levels - 1; l >= 0; --l) {
        long n0 = nx >> l, n1 = ny >> l;
        long hx = n0 / 2, hy = n1 / 2;
        std::vector<u16> bands(3 * hx * hy);
        std::vector<u16*> ob(3);
        for (int b = 0; b < 3; ++b) ob[b] = bands.data() + b * hx * hy;
        decodeRLHuff(br, ob, u32(hx * hy), cb, log2Max);
        br.align(4);
        std::vector<i16> c(n0 * n1);
        for (long y = 0; y < hy; ++y)
            for (long x = 0; x < hx; ++x) c[y * n0 + x] = cur[y * hx + x];
        for (int b = 1; b < 4; ++b)
            for (long y = 0; y < hy; ++y)
                for (long x = 0; x < hx; ++x)
                    c[(y + (b / 2) * hy) * n0 + x + (b % 2) * hx] = i16(unsymbolize(ob[b - 1][y * hx + x]));
        cur.resize(c.size());
        dwtInt(c.data(), cur.data(), n0, n1, 1, true);
    }
    std::copy(cur.begin(), cur.end(), out);
    return 0;
}

}  // extern "C"

// ===========================================================================
// The 2D image side: byte conversions, lowpass-only transforms, byte-image
// quantizers, YCoCg, least-significant-bit planes, and the one-level image
// and heightfield codecs of the reference's examples.
// ===========================================================================

// DWTCommon.cuh:14-41 and Quantize.cuh:15-23
static inline float byteToFloatO(u8 b) { return float(b) - 128.0f; }
static inline u8 floatToByteO(float v) { return u8(std::min(std::max(v + 128.5f, 0.0f), 255.0f)); }

// Quantize.cuh:75-131 (type 0 deadzone, 1 uniform; the uniform product
// contracted into one fma as the device code is compiled)
static inline int quantO(float v, float inv, int type) {
    if (type == 0) return int(v * inv);
    const float s = v > 0.0f ? 1.0f : (v < 0.0f ? -1.0f : 0.0f);
    return int(std::fmaf(v, inv, s * 0.5f));
}
// the dequantized value before its multiplication by the step
static inline float unquantBaseO(int q, int type) {
    if (type == 0) return float(q) + (q > 0 ? 1.0f : (q < 0 ? -1.0f : 0.0f)) * 0.5f;
    return float(q);
}
static inline float unquantO(int q, float step, int type) { return unquantBaseO(q, type) * step; }
// dequantized value plus a reference (QuantizeKernels.cui:261-262, 279-280):
// the device code contracts the step multiply and the add into one fma
static inline float unquantPlusO(int q, float step, float ref, int type) {
    return std::fmaf(unquantBaseO(q, type), step, ref);
}

// 5/3 lowpass of the even sample c with neighbours a b | d e
// (DWTInt2DLowpassKernels.cui:58-88, rounding DWTCommon.cuh:133-142)
static inline i16 lowpass53O(i16 a, i16 b, i16 c, i16 d, i16 e) {
    const i16 d1 = i16(b - div2(i16(a + c)));
    const i16 d3 = i16(d - div2(i16(c + e)));
    return i16(c + div4(i16(d1 + d3)));
}

// removeLSB / appendLSB of one element (Bits.cu:62-174)
static inline i16 removeLsbO(i16 v, i16 shift, u32* bit) {
    const i16 t = i16(v + shift);
    *bit = u32(t & 1);
    return i16((int(t) + (t < 0 ? -1 : 0)) / 2);
}
static inline i16 appendLsbO(i16 v, u32 bit, i16 shift) {
    const i16 t = i16((int(v) * 2) | int(bit));
    return i16(t + shift);
}

extern "C" {

// dwtFloat{2D,3D}ForwardFromByte (DWTFloat.cu:653-670): src addresses the
// channel, element stride `channels`, rows of nx * channels bytes.
void orc_dwt_float_fwd_from_byte(const u8* src, long channels, float* dst, long nx, long ny, long nz) {
    std::vector<float> f(nx * ny * nz);
    for (long i = 0; i < nx * ny * nz; ++i) f[i] = byteToFloatO(src[i * channels]);
    dwtFloat(f.data(), dst, nx, ny, nz, false);
}

// dwtFloat{2D,3D}InverseToByte (DWTFloat.cu:673-690): dst addresses the channel.
void orc_dwt_float_inv_to_byte(const float* src, u8* dst, long channels, long nx, long ny, long nz) {
    std::vector<float> f(nx * ny * nz);
    dwtFloat(src, f.data(), nx, ny, nz, true);
    for (long i = 0; i < nx * ny * nz; ++i) dst[i * channels] = floatToByteO(f[i]);
}

// dwtFloat{2D,3D}InverseFromSymbolsToByte (DWTFloat.cu:693-712): the dense
// lowpass (nx/2 x ny/2 x nz/2) and 3 or 7 dense u16 bands (index x+2y+4z-1)
// dequantized as Quantize.cuh:104-110, then the inverse into bytes.
void orc_dwt_float_inv_from_symbols_to_byte(const float* lowpass, const u16* const* bands, float step, u8* dst,
                                            long channels, long nx, long ny, long nz) {
    const long hx = nx / 2, hy = ny / 2, hz = nz > 1 ? nz / 2 : 1;
    std::vector<float> coef(nx * ny * nz);
    for (long z = 0; z < hz; ++z)
        for (long y = 0; y < hy; ++y)
            for (long x = 0; x < hx; ++x) coef[(z * ny + y) * nx + x] = lowpass[(z * hy + y) * hx + x];
    const int nb = nz > 1 ? 8 : 4;
    for (int b = 1; b < nb; ++b) unquantizeBand(coef.data(), nx, ny, nz, b % 2, (b / 2) % 2, b / 4, step, bands[b - 1]);
    orc_dwt_float_inv_to_byte(coef.data(), dst, channels, nx, ny, nz);
}

// dwtFloat2DForwardLowpassOnlyFromByte (DWTFloat.cu:17-83, kernels
// DWTFloat2DLowpassKernels.cui): the LL band alone, the even outputs of the
// X pass then of the Y pass - the same numbers as the LL band of the full
// transform, which is how it is restated here.
void orc_dwt_float2d_lowpass_from_byte(const u8* src, long channels, float* dst, long nx, long ny) {
    std::vector<float> full(nx * ny);
    orc_dwt_float_fwd_from_byte(src, channels, full.data(), nx, ny, 1);
    for (long y = 0; y < ny / 2; ++y)
        for (long x = 0; x < nx / 2; ++x) dst[y * (nx / 2) + x] = full[y * nx + x];
}

// dwtIntForwardLowpassOnly (DWTInt.cu:14-77): predict + update per row, then
// per column of the row results, keeping only the even samples.
void orc_dwt_int_lowpass(const i16* src, i16* dst, long nx, long ny) {
    const long hx = nx / 2, hy = ny / 2;
    std::vector<i16> xl(ny * hx);
    for (long y = 0; y < ny; ++y)
        for (long L = 0; L < hx; ++L) {
            const i16* r = src + y * nx;
            xl[y * hx + L] = lowpass53O(r[mirror(2 * L - 2, nx)], r[mirror(2 * L - 1, nx)], r[2 * L],
                                        r[mirror(2 * L + 1, nx)], r[mirror(2 * L + 2, nx)]);
        }
    for (long M = 0; M < hy; ++M)
        for (long x = 0; x < hx; ++x)
            dst[M * hx + x] = lowpass53O(xl[mirror(2 * M - 2, ny) * hx + x], xl[mirror(2 * M - 1, ny) * hx + x],
                                         xl[2 * M * hx + x], xl[mirror(2 * M + 1, ny) * hx + x],
                                         xl[mirror(2 * M + 2, ny) * hx + x]);
}

// floatToByte2D / byteToFloat2D (Quantize.cu:19-43, QuantizeKernels.cui:11-34)
void orc_float_to_byte_2d(u8* out, long channels, long channel, const float* in, long nx, long ny, long rowPitch) {
    for (long y = 0; y < ny; ++y)
        for (long x = 0; x < nx; ++x) out[(y * nx + x) * channels + channel] = floatToByteO(in[y * rowPitch + x]);
}
void orc_byte_to_float_2d(float* out, const u8* in, long channels, long channel, long nx, long ny, long rowPitch) {
    for (long y = 0; y < ny; ++y)
        for (long x = 0; x < nx; ++x) out[y * rowPitch + x] = byteToFloatO(in[(y * nx + x) * channels + channel]);
}

// quantizeDifferenceToSymbols(Roundtrip)2D (Quantize.cu:276-326,
// QuantizeKernels.cui:227-263): symbol of (v - (ref - 128)) as 16 bits; the
// round trip writes back the stored symbol's value plus the reference.
void orc_quantize_difference_2d(u16* sym, float* data, float step, const u8* ref, long channels, long channel, long nx,
                                long ny, long rowPitch, int type, int roundtrip) {
    const float inv = 1.0f / step;
    for (long y = 0; y < ny; ++y)
        for (long x = 0; x < nx; ++x) {
            const float r = byteToFloatO(ref[(y * nx + x) * channels + channel]);
            float& v = data[y * rowPitch + x];
            const u16 q = u16(symbolize(quantO(v - r, inv, type)));
            sym[y * nx + x] = q;
            if (roundtrip) v = unquantPlusO(unsymbolize(q), step, r, type);
        }
}
// unquantizeDifferenceFromSymbols2D (Quantize.cu:328-352, QuantizeKernels.cui:265-281)
void orc_unquantize_difference_2d(float* data, const u16* sym, float step, const u8* ref, long channels, long channel,
                                  long nx, long ny, long rowPitch, int type) {
    for (long y = 0; y < ny; ++y)
        for (long x = 0; x < nx; ++x)
            data[y * rowPitch + x] = unquantPlusO(unsymbolize(sym[y * nx + x]), step,
                                                  byteToFloatO(ref[(y * nx + x) * channels + channel]), type);
}

// convertRGBtoYCoCg / convertYCoCgtoRGB (YCoCg.cu:21-88): integer arithmetic
// with C division; `channels` 3 or 4 (the 4th byte is copied).
void orc_ycocg(u8* dst, const u8* src, long n, int channels, int toYCoCg) {
    for (long i = 0; i < n; ++i) {
        const int a = src[i * channels], b = src[i * channels + 1], c = src[i * channels + 2];
        const int w = channels == 4 ? src[i * channels + 3] : 0;
        int o[3];
        if (toYCoCg) {
            o[0] = (a + b * 2 + c + 2) / 4;
            o[1] = (a - c + 1) / 2 + 127;
            o[2] = (-a + b * 2 - c + 2) / 4 + 127;
        } else {
            o[0] = std::min(std::max(a + b - c, 0), 255);
            o[1] = std::min(std::max(a + c - 127, 0), 255);
            o[2] = std::min(std::max(a - b - c + 254, 0), 255);
        }
        for (int k = 0; k < 3; ++k) dst[i * channels + k] = u8(o[k]);
        if (channels == 4) dst[i * channels + 3] = u8(w);
    }
}

// getLSB / removeLSB / appendLSB (Bits.cu:20-174): mode 0 get, 1 remove
// (bits may be null), 2 append; bit j of word w is element 32 w + j.
void orc_lsb(int mode, i16* data, u32* bits, u32 n, i16 shift) {
    const u32 words = (n + 31) / 32;
    if (mode != 2 && bits) std::fill(bits, bits + words, 0u);
    for (u32 e = 0; e < n; ++e) {
        u32 b = 0;
        if (mode == 0) {
            bits[e / 32] |= u32(data[e] & 1) << (e % 32);
        } else if (mode == 1) {
            data[e] = removeLsbO(data[e], shift, &b);
            if (bits) bits[e / 32] |= b << (e % 32);
        } else {
            data[e] = appendLsbO(data[e], (bits[e / 32] >> (e % 32)) & 1u, shift);
        }
    }
}
// shiftElems (Bits.cu:143-151)
void orc_shift_elems(i16* data, u32 n, i16 shift) {
    for (u32 e = 0; e < n; ++e) data[e] = i16(data[e] + shift);
}

// getLowpassImage (CompressImage.cpp:342-365)
void orc_get_lowpass_image(const u8* image, long nx, long ny, long chTotal, long chProc, u8* out) {
    std::vector<float> ll((nx / 2) * (ny / 2));
    for (long c = 0; c < chProc; ++c) {
        orc_dwt_float2d_lowpass_from_byte(image + c, chTotal, ll.data(), nx, ny);
        orc_float_to_byte_2d(out, chTotal, c, ll.data(), nx / 2, ny / 2, nx / 2);
    }
}

// getLowpassHeightfield (CompressHeightfield.cpp:218-235)
void orc_get_lowpass_heightfield(const i16* image, long nx, long ny, i16* out, i16 shift) {
    orc_dwt_int_lowpass(image, out, nx, ny);
    orc_lsb(1, out, nullptr, u32((nx / 2) * (ny / 2)), shift);
}

// compressImageOneLevel (CompressImage.cpp:71-128): image (interleaved,
// chTotal channels) is overwritten with its reconstruction.
int orc_compress_image_one_level(u8* image, long nx, long ny, long chTotal, long chProc, const u8* lpRef, float step,
                                 u32 cb, u32 log2Max, u32* words, u32 cap, u32* bitSize) {
    const long hx = nx / 2, hy = ny / 2, n = hx * hy;
    std::vector<u16> syms(4 * chProc * n);
    std::vector<float> coef(nx * ny);
    const float inv = 1.0f / step;
    for (long c = 0; c < chProc; ++c) {
        orc_dwt_float_fwd_from_byte(image + c, chTotal, coef.data(), nx, ny, 1);
        orc_quantize_difference_2d(syms.data() + c * n, coef.data(), step, lpRef, chTotal, c, hx, hy, nx, 0, 1);
        for (int b = 1; b < 4; ++b) {
            u16* out = syms.data() + (chProc + 3 * c + b - 1) * n;
            // quantizeToSymbolsRoundtrip (QuantizeKernels.cui:95-113): back from the full quantized value
            for (long y = 0; y < hy; ++y)
                for (long x = 0; x < hx; ++x) {
                    float& v = coef[(y + (b / 2) * hy) * nx + x + (b % 2) * hx];
                    const int q = quantO(v, inv, 0);
                    out[y * hx + x] = u16(symbolize(q));
                    v = unquantO(q, step, 0);
                }
        }
        orc_dwt_float_inv_to_byte(coef.data(), image + c, chTotal, nx, ny, 1);
    }
    std::vector<const u16*> s(4 * chProc);
    for (long k = 0; k < 4 * chProc; ++k) s[k] = syms.data() + k * n;
    BitStream bs;
    int r = encodeRLHuff(bs, s, u32(n), cb, log2Max);
    if (r) return r;
    u32 pos;
    return finishBits(bs, words, cap, bitSize, &pos);
}

// decompressImageOneLevel (CompressImage.cpp:135-186)
int orc_decompress_image_one_level(const u32* words, u32 bitSize, u8* image, long nx, long ny, long chTotal,
                                   long chProc, const u8* lpRef, float step, u32 cb, u32 log2Max) {
    const long hx = nx / 2, hy = ny / 2, n = hx * hy;
    std::vector<u16> syms(4 * chProc * n);
    std::vector<u16*> o(4 * chProc);
    for (long k = 0; k < 4 * chProc; ++k) o[k] = syms.data() + k * n;
    BitReader br{words, bitSize, 0};
    decodeRLHuff(br, o, u32(n), cb, log2Max);
    std::vector<float> lp(n);
    for (long c = 0; c < chProc; ++c) {
        orc_unquantize_difference_2d(lp.data(), o[c], step, lpRef, chTotal, c, hx, hy, hx, 0);
        const u16* bands[3] = {o[chProc + 3 * c], o[chProc + 3 * c + 1], o[chProc + 3 * c + 2]};
        orc_dwt_float_inv_from_symbols_to_byte(lp.data(), bands, step, image + c, chTotal, nx, ny, 1);
    }
    return 0;
}

// compressHeightfieldOneLevel (CompressHeightfield.cpp:82-141)
int orc_compress_heightfield_one_level(const i16* image, long nx, long ny, i16* lowpass, i16 shift, u32 cb,
                                       u32 log2Max, u32* words, u32 cap, u32* bitSize) {
    const long hx = nx / 2, hy = ny / 2, n = hx * hy;
    std::vector<i16> c(nx * ny);
    dwtInt(image, c.data(), nx, ny, 1, false);
    for (long y = 0; y < hy; ++y)
        for (long x = 0; x < hx; ++x) lowpass[y * hx + x] = c[y * nx + x];
    std::vector<u32> bits((n + 31) / 32);
    orc_lsb(1, lowpass, bits.data(), u32(n), shift);
    std::vector<u16> bands(3 * n);
    std::vector<const u16*> s(3);
    for (int b = 1; b < 4; ++b) {
        for (long y = 0; y < hy; ++y)
            for (long x = 0; x < hx; ++x)
                bands[(b - 1) * n + y * hx + x] = u16(symbolize(c[(y + (b / 2) * hy) * nx + x + (b % 2) * hx]));
        s[b - 1] = bands.data() + (b - 1) * n;
    }
    BitStream bs;
    bs.writeAligned(bits.data(), 4, u32(bits.size()));
    int r = encodeRLHuff(bs, s, u32(n), cb, log2Max);
    if (r) return r;
    u32 pos;
    return finishBits(bs, words, cap, bitSize, &pos);
}

// decompressHeightfieldOneLevel (CompressHeightfield.cpp:148-216): lowpass is
// restored in place, then the image rebuilt.
int orc_decompress_heightfield_one_level(const u32* words, u32 bitSize, i16* image, long nx, long ny, i16* lowpass,
                                         i16 shift, u32 cb, u32 log2Max) {
    const long hx = nx / 2, hy = ny / 2, n = hx * hy;
    const u32 bitWords = u32((n + 31) / 32);
    if (bitSize < bitWords * 32) return -1;
    std::vector<u32> bits(words, words + bitWords);
    orc_lsb(2, lowpass, bits.data(), u32(n), shift);
    BitReader br{words, bitSize, bitWords * 32};
    std::vector<u16> bands(3 * n);
    std::vector<u16*> ob(3);
    for (int b = 0; b < 3; ++b) ob[b] = bands.data() + b * n;
    decodeRLHuff(br, ob, u32(n), cb, log2Max);
    std::vector<i16> c(nx * ny);
    for (long y = 0; y < hy; ++y)
        for (long x = 0; x < hx; ++x) c[y * nx + x] = lowpass[y * hx + x];
    for (int b = 1; b < 4; ++b)
        for (long y = 0; y < hy; ++y)
            for (long x = 0; x < hx; ++x)
                c[(y + (b / 2) * hy) * nx + x + (b % 2) * hx] = i16(unsymbolize(ob[b - 1][y * hx + x]));
    dwtInt(c.data(), image, nx, ny, 1, true);
    return 0;
}

}  // extern "C"
