// selftest_host.cpp - host build of the table constructor in huffman_build.cuh,
// exported for the CPU unit tests (tests/test_table_build_host.py), which
// compare it with the oracle on many histograms.  Not part of the product
// library: it is built into _lib/libcc_selftest.so and loaded only by tests.
#include <cstring>
#include <vector>
#include "huffman_build.cuh"

using namespace ccb;

extern "C" int ccst_huffman_build(const u32* hist, u32 bins, u32 symbolMax, u32 log2Max, u32* codewords,
                                  u32* lengths, u32* tableWords, u32 cap, u32* tableBits) {
    std::vector<u32> leafSym, leafProb;
    for (u32 s = 0; s < bins; ++s)
        if (hist[s]) { leafSym.push_back(s); leafProb.push_back(hist[s]); }
    int L = int(leafSym.size());
    for (u32 i = 0; i < bins; ++i) { codewords[i] = 0; lengths[i] = 0xFFFFFFFFu; }
    u32 lenCount[32] = {0};
    int maxLen = 0;
    std::vector<u32> sorted(L);
    if (L > 0) {
        std::vector<u64> heap(L);
        std::vector<u32> parent(2 * L);
        std::vector<u8> depth(2 * L);
        for (int i = 0; i < L; ++i) heap[i] = (u64(leafProb[i]) << 32) | u32(i);
        hb::buildTree(heap.data(), parent.data(), L);
        hb::nodeDepths(parent.data(), depth.data(), L);
        std::vector<u32> order(L);
        for (int i = 0; i < L; ++i) {
            order[i] = (u32(depth[i]) << 27) | u32(i);
            if (depth[i] > maxLen) maxLen = depth[i];
        }
        if (maxLen > 31) return -5;
        hb::introsort(order.data(), L, hb::LenLess());
        u32 code = 0, prevLen = 0;
        for (int k = 0; k < L; ++k) {
            u32 len = order[k] >> 27;
            u32 sym = leafSym[order[k] & hb::kLeafMask];
            if (k > 0) code = (code + 1) << (len - prevLen);
            prevLen = len;
            if (len) lenCount[len - 1]++;
            sorted[k] = sym;
            codewords[sym] = code;
            lengths[sym] = len;
        }
    }
    // serialization as HuffmanTable.cu:470-485
    std::vector<u32> w;
    u32 pos = 0;
    auto put = [&](u32 v, u32 n) {
        for (u32 b = 0; b < n; ++b, ++pos) {
            if (pos / 32 >= w.size()) w.push_back(0);
            if ((v >> (n - 1 - b)) & 1u) w[pos / 32] |= 1u << (31 - pos % 32);
        }
    };
    bool longSym = log2Max > 16;
    put(u32(maxLen), 5);
    for (int l = 0; l < maxLen; ++l) put(lenCount[l], log2Max);
    put(u32(L), log2Max);
    u32 symbolBits = requiredBits(symbolMax);
    put(symbolBits, longSym ? 5 : 4);
    for (int k = 0; k < L; ++k) put(sorted[k], symbolBits);
    *tableBits = pos;
    if (w.size() > cap) return -2;
    std::memcpy(tableWords, w.data(), w.size() * 4);
    return maxLen;
}
