// ref_cpu_harness.cpp - drives the reference's own CPU run-length + Huffman
// coder (src/CPU/RunLengthCPU.cpp, HuffmanTableCPU.cpp, HuffmanCPU.cpp) the
// way encodeRLHuffCPU does (src/CPU/EncodeCPU.cpp:98-200), one stream per
// OpenMP task.  Built by oracle/ref/Makefile into oracle/_ref/libref_cpu.so.
// TEST / BASELINE INFRASTRUCTURE ONLY: bench.py's reference arm times it.
#include <cstdint>
#include <cstring>
#include <vector>
#include <omp.h>
#include "RunLengthCPU.h"
#include "HuffmanTableCPU.h"
#include "HuffmanCPU.h"

using namespace cudaCompress;

static void encodeOne(BitStream& bs, const std::vector<Symbol16>& symbols, uint cb) {
    std::vector<Symbol16> compact;
    std::vector<ushort> zeroCounts;
    runLengthZeroesEncodeCPU(compact, zeroCounts, symbols, ZERO_COUNT_MAX);
    uint compactCount = (uint)compact.size();
    bs.writeAligned(&compactCount, 1);
    for (int pass = 0; pass < 2; ++pass) {
        const std::vector<Symbol16>& s = pass == 0 ? compact : zeroCounts;
        HuffmanTableCPU table;
        table.design(s);
        table.writeToBitStream(bs);
        HuffmanDecodeTableCPU dec;
        dec.build(table);
        HuffmanEncodeTableCPU enc;
        enc.build(dec);
        bs.writeAlign<uint>();
        uint sizeIndex = bs.getBitPosition() / 32;
        uint bits = 0;
        bs.writeAligned(&bits, 1);
        std::vector<uint> offsets;
        uint start = bs.getBitPosition();
        huffmanEncodeCPU(bs, s, enc, offsets, cb);
        bs.getRaw()[sizeIndex] = bs.getBitPosition() - start;
        bs.writeAlign<uint>();
        std::vector<ushort> inc(offsets.size());
        for (size_t i = 1; i < offsets.size(); ++i) inc[i] = ushort(offsets[i] - offsets[i - 1]);
        bs.writeAligned(inc.data(), (uint)inc.size());
    }
}

static void decodeOne(BitStreamReadOnly& bs, std::vector<Symbol16>& out, uint n, uint cb) {
    uint compactCount = 0;
    bs.readAligned(&compactCount, 1);
    std::vector<Symbol16> streams[2];
    for (int pass = 0; pass < 2; ++pass) {
        HuffmanTableCPU table;
        table.readFromBitStream(bs);
        HuffmanDecodeTableCPU dec;
        dec.build(table);
        uint bits = 0;
        bs.readAligned(&bits, 1);
        uint start = bs.getBitPosition();
        huffmanDecodeCPU(bs, compactCount, streams[pass], dec);
        bs.setBitPosition(start + bits);
        bs.align<uint>();
        bs.skipAligned<ushort>((compactCount + cb - 1) / cb);
    }
    runLengthZeroesDecodeCPU(streams[0], streams[1], out, n);
}

extern "C" {

// Encode S streams of n symbols (contiguous); per-stream bit sizes returned.
// Returns total words written into `words` (each stream word-aligned, packed
// back to back) or -1 if cap is too small.
long refcpu_encode_rlhuff(const uint16_t* symbols, uint32_t S, uint32_t n, uint32_t cb, int threads,
                          uint32_t* words, long cap, uint32_t* streamWords) {
    std::vector<std::vector<uint>> out(S);
    if (threads > 0) omp_set_num_threads(threads);
    #pragma omp parallel for schedule(dynamic, 1)
    for (int i = 0; i < int(S); ++i) {
        std::vector<Symbol16> s(symbols + size_t(i) * n, symbols + size_t(i + 1) * n);
        BitStream bs(&out[i]);
        encodeOne(bs, s, cb);
    }
    long total = 0;
    for (uint32_t i = 0; i < S; ++i) {
        streamWords[i] = (uint32_t)out[i].size();
        if (total + long(out[i].size()) > cap) return -1;
        std::memcpy(words + total, out[i].data(), out[i].size() * 4);
        total += long(out[i].size());
    }
    return total;
}

int refcpu_decode_rlhuff(const uint32_t* words, const uint32_t* streamWords, uint32_t S, uint32_t n, uint32_t cb,
                         int threads, uint16_t* out) {
    std::vector<size_t> start(S + 1, 0);
    for (uint32_t i = 0; i < S; ++i) start[i + 1] = start[i] + streamWords[i];
    if (threads > 0) omp_set_num_threads(threads);
    #pragma omp parallel for schedule(dynamic, 1)
    for (int i = 0; i < int(S); ++i) {
        BitStreamReadOnly bs(words + start[i], streamWords[i] * 32);
        std::vector<Symbol16> o;
        decodeOne(bs, o, n, cb);
        std::memcpy(out + size_t(i) * n, o.data(), size_t(n) * 2);
    }
    return 0;
}

}
