// cxx_api.cu - the reference's C++ API (namespace cudaCompress) over the C ABI.
// Signatures follow include/cudaCompress/*.h of the reference exactly; bool /
// void results map the C status codes (cc_last_error() keeps the message).
#include <cstdio>
#include <map>
#include <vector>

#include <cudaCompress/BitStream.h>
#include <cudaCompress/Encode.h>
#include <cudaCompress/Instance.h>
#include <cudaCompress/Timing.h>
#include <cudaCompress/util/Bits.h>
#include <cudaCompress/util/DWT.h>
#include <cudaCompress/util/Quantize.h>
#include <cudaCompress/util/YCoCg.h>

#include "../../include/cudacompress_b200.h"

namespace cudaCompress {

class Instance {
public:
    cc_instance* h = nullptr;
};

// Grants the coder access to the word storage of a BitStream.
struct BitStreamAccess {
    static std::vector<uint>& vec(BitStream& b) { return *b.m_pVector; }
    static void place(BitStream& b, uint pos, uint size) {
        b.m_pBuffer = b.m_pVector->data();
        b.m_bitSize = size;
        b.m_bufferPos = pos / 32;
        b.m_bitPos = pos % 32;
    }
};

static bool report(int rc, const char* what) {
    if (rc == CC_OK) return true;
    std::fprintf(stderr, "cudaCompress: %s failed: %s\n", what, cc_last_error());
    return false;
}

Instance* createInstance(int cudaDevice, uint streamCountMax, uint elemCountPerStreamMax, uint codingBlockSize,
                         uint log2HuffmanDistinctSymbolCountMax) {
    cc_instance* h = nullptr;
    if (!report(cc_create_instance(&h, cudaDevice, streamCountMax, elemCountPerStreamMax, codingBlockSize,
                                   log2HuffmanDistinctSymbolCountMax), "createInstance"))
        return nullptr;
    Instance* p = new Instance();
    p->h = h;
    return p;
}

void destroyInstance(Instance* p) {
    if (!p) return;
    cc_destroy_instance(p->h);
    delete p;
}

int getInstanceCudaDevice(const Instance* p) { return cc_get_instance_cuda_device(p->h); }
uint getInstanceStreamCountMax(const Instance* p) { return cc_get_instance_stream_count_max(p->h); }
uint getInstanceElemCountPerStreamMax(const Instance* p) { return cc_get_instance_elem_count_per_stream_max(p->h); }
uint getInstanceCodingBlockSize(const Instance* p) { return cc_get_instance_coding_block_size(p->h); }
uint getInstanceLog2HuffmanDistinctSymbolCountMax(const Instance* p) { return cc_get_instance_log2_huffman_distinct_symbol_count_max(p->h); }
bool getInstanceUseLongSymbols(const Instance* p) { return cc_get_instance_use_long_symbols(p->h) != 0; }
void setInstanceCudaStream(Instance* p, cudaStream_t s) { cc_set_instance_stream(p->h, s); }
cudaStream_t getInstanceCudaStream(const Instance* p) { return static_cast<cudaStream_t>(cc_get_instance_stream(p->h)); }
void setInstanceStream(Instance* p, cudaStream_t s) { cc_set_instance_stream(p->h, s); }
cudaStream_t getInstanceStream(const Instance* p) { return static_cast<cudaStream_t>(cc_get_instance_stream(p->h)); }

size_t encodeGetRequiredMemory(const Instance* p) { return cc_encode_get_required_memory(p->h); }
bool encodeInit(Instance*) { return true; }
bool encodeShutdown(Instance*) { return true; }

// ---- encode ----
// Appends segment `i` of the last encode to `bs` (BitStream.h semantics:
// RLHuff segments begin word aligned, Huff segments at the current bit).
static void appendSegment(Instance* inst, BitStream& bs, uint i, int kind) {
    const uint* words;
    uint wordCount, startBit, bitLength;
    cc_encoded_segment(inst->h, i, &words, &wordCount, &startBit, &bitLength);
    const uint pos = bs.getBitPosition();
    const uint w0 = kind == CC_KIND_RLHUFF ? (pos + 31) / 32 : pos / 32;
    std::vector<uint>& v = BitStreamAccess::vec(bs);
    const uint endWord = w0 + wordCount;
    if (v.size() < endWord) v.resize(endWord, 0u);
    const uint r = kind == CC_KIND_RLHUFF ? 0u : (pos & 31u);
    const uint keep = r ? (0xffffffffu << (32 - r)) : 0u;
    v[w0] = (v[w0] & keep) | (words[0] & ~keep);
    for (uint k = 1; k < wordCount; ++k) v[w0 + k] = words[k];
    const uint end = w0 * 32 + bitLength;
    BitStreamAccess::place(bs, end, std::max(end, bs.getBitSize()));
}

template <typename Symbol>
static bool encodeImpl(Instance* inst, BitStream* const* bss, bool single, const Symbol* const* streams, uint count,
                       uint n, int kind) {
    std::vector<uint> startBits(count, 0);
    if (kind == CC_KIND_HUFF) {
        std::map<BitStream*, bool> seen;
        for (uint i = 0; i < count; ++i) {
            BitStream* b = bss[single ? 0 : i];
            if (!seen[b]) {
                startBits[i] = b->getBitPosition() & 31u;
                seen[b] = true;
            }
        }
    }
    std::vector<const void*> ptrs(streams, streams + count);
    if (!report(cc_encode(inst->h, kind, int(sizeof(Symbol)), ptrs.data(), count, n, startBits.data()),
                kind == CC_KIND_RLHUFF ? "encodeRLHuff" : "encodeHuff"))
        return false;
    for (uint i = 0; i < count; ++i) appendSegment(inst, *bss[single ? 0 : i], i, kind);
    return true;
}

template <typename Symbol>
static bool decodeImpl(Instance* inst, BitStreamReadOnly* const* bss, bool single, Symbol* const* streams, uint count,
                       uint n, int kind) {
    std::vector<BitStreamReadOnly*> uniq;
    std::vector<uint> idx(count);
    for (uint i = 0; i < count; ++i) {
        BitStreamReadOnly* b = bss[single ? 0 : i];
        uint k = 0;
        while (k < uniq.size() && uniq[k] != b) ++k;
        if (k == uniq.size()) uniq.push_back(b);
        idx[i] = k;
    }
    std::vector<const uint32_t*> words(uniq.size());
    std::vector<uint32_t> sizes(uniq.size()), pos(uniq.size());
    for (size_t k = 0; k < uniq.size(); ++k) {
        words[k] = uniq[k]->getRaw();
        sizes[k] = uniq[k]->getBitSize();
        pos[k] = uniq[k]->getBitPosition();
    }
    std::vector<void*> outs(streams, streams + count);
    if (!report(cc_decode(inst->h, kind, int(sizeof(Symbol)), words.data(), sizes.data(), pos.data(), uint(uniq.size()),
                          idx.data(), outs.data(), count, n),
                kind == CC_KIND_RLHUFF ? "decodeRLHuff" : "decodeHuff"))
        return false;
    for (size_t k = 0; k < uniq.size(); ++k) uniq[k]->setBitPosition(pos[k]);
    return true;
}

#define CC_DEFINE_CODEC(Sym)                                                                                          \
    bool encodeRLHuff(Instance* i, BitStream& b, const Sym* const s[], uint c, uint n) {                             \
        BitStream* p = &b;                                                                                            \
        return encodeImpl<Sym>(i, &p, true, s, c, n, CC_KIND_RLHUFF);                                                 \
    }                                                                                                                 \
    bool decodeRLHuff(Instance* i, BitStreamReadOnly& b, Sym* s[], uint c, uint n) {                                  \
        BitStreamReadOnly* p = &b;                                                                                    \
        return decodeImpl<Sym>(i, &p, true, s, c, n, CC_KIND_RLHUFF);                                                 \
    }                                                                                                                 \
    bool encodeHuff(Instance* i, BitStream& b, Sym* const s[], uint c, uint n) {                                     \
        BitStream* p = &b;                                                                                            \
        return encodeImpl<Sym>(i, &p, true, s, c, n, CC_KIND_HUFF);                                                   \
    }                                                                                                                 \
    bool decodeHuff(Instance* i, BitStreamReadOnly& b, Sym* s[], uint c, uint n) {                                    \
        BitStreamReadOnly* p = &b;                                                                                    \
        return decodeImpl<Sym>(i, &p, true, s, c, n, CC_KIND_HUFF);                                                   \
    }                                                                                                                 \
    bool encodeRLHuff(Instance* i, BitStream* b[], const Sym* const s[], uint c, uint n) {                           \
        return encodeImpl<Sym>(i, b, false, s, c, n, CC_KIND_RLHUFF);                                                 \
    }                                                                                                                 \
    bool decodeRLHuff(Instance* i, BitStreamReadOnly* b[], Sym* s[], uint c, uint n) {                                \
        return decodeImpl<Sym>(i, b, false, s, c, n, CC_KIND_RLHUFF);                                                 \
    }                                                                                                                 \
    bool encodeHuff(Instance* i, BitStream* b[], Sym* const s[], uint c, uint n) {                                   \
        return encodeImpl<Sym>(i, b, false, s, c, n, CC_KIND_HUFF);                                                   \
    }                                                                                                                 \
    bool decodeHuff(Instance* i, BitStreamReadOnly* b[], Sym* s[], uint c, uint n) {                                  \
        return decodeImpl<Sym>(i, b, false, s, c, n, CC_KIND_HUFF);                                                   \
    }

CC_DEFINE_CODEC(Symbol16)
CC_DEFINE_CODEC(Symbol32)
#undef CC_DEFINE_CODEC

// ---- timing: CUDA-event sections per kernel, accumulated by name ----
void setTimingDetail(Instance* p, ETimingDetail detail) { cc_set_timing(p->h, detail != TIMING_DETAIL_NONE); }
void getTimings(Instance* p, std::vector<std::string>& names, std::vector<float>& times) {
    names.clear();
    times.clear();
    const int n = cc_timing_count(p->h);
    for (int i = 0; i < n; ++i) {
        const char* name;
        double ms;
        uint32_t count;
        cc_timing_entry(p->h, uint32_t(i), &name, &ms, &count);
        names.push_back(name);
        times.push_back(float(ms));
    }
}
void printTimings(Instance* p) {
    std::vector<std::string> names;
    std::vector<float> times;
    getTimings(p, names, times);
    for (size_t i = 0; i < names.size(); ++i) std::printf("%-32s %10.3f ms\n", names[i].c_str(), times[i]);
}
void resetTimings(Instance* p) { cc_reset_timings(p->h); }

namespace util {

void dwtFloat2DForward(float* d, float* b, const float* s, int sx, int sy, int ch, int dr, int sr, cudaStream_t st) {
    report(cc_dwt_float_forward(d, nullptr, b, s, sx, sy, 1, ch, dr, 0, sr, 0, st), "dwtFloat2DForward");
}
void dwtFloat3DForward(float* d, float* b2, float* b1, const float* s, int sx, int sy, int sz, int ch, int dr, int ds,
                       int sr, int ss, cudaStream_t st) {
    report(cc_dwt_float_forward(d, b2, b1, s, sx, sy, sz, ch, dr, ds, sr, ss, st), "dwtFloat3DForward");
}
void dwtFloat2DInverse(float* d, float* b, const float* s, int sx, int sy, int ch, int dr, int sr, cudaStream_t st) {
    report(cc_dwt_float_inverse(d, nullptr, b, s, sx, sy, 1, ch, dr, 0, sr, 0, st), "dwtFloat2DInverse");
}
void dwtFloat3DInverse(float* d, float* b2, float* b1, const float* s, int sx, int sy, int sz, int ch, int dr, int ds,
                       int sr, int ss, cudaStream_t st) {
    report(cc_dwt_float_inverse(d, b2, b1, s, sx, sy, sz, ch, dr, ds, sr, ss, st), "dwtFloat3DInverse");
}
void dwtFloat2DInverseFromSymbols(float* d, float* b, const float* lp, const ushort* const* hp, float q, int sx, int sy,
                                  int ch, int dr, int lr, cudaStream_t st) {
    report(cc_dwt_float_inverse_from_symbols(d, nullptr, b, lp, reinterpret_cast<const void* const*>(hp), 2, q, sx, sy, 1,
                                             ch, dr, 0, lr, 0, st), "dwtFloat2DInverseFromSymbols");
}
void dwtFloat3DInverseFromSymbols(float* d, float* b2, float* b1, const float* lp, const ushort* const* hp, float q, int sx,
                                  int sy, int sz, int ch, int dr, int ds, int lr, int ls, cudaStream_t st) {
    report(cc_dwt_float_inverse_from_symbols(d, b2, b1, lp, reinterpret_cast<const void* const*>(hp), 2, q, sx, sy, sz,
                                             ch, dr, ds, lr, ls, st), "dwtFloat3DInverseFromSymbols");
}
void dwtFloat2DInverseFromSymbols(float* d, float* b, const float* lp, const uint* const* hp, float q, int sx, int sy,
                                  int ch, int dr, int lr, cudaStream_t st) {
    report(cc_dwt_float_inverse_from_symbols(d, nullptr, b, lp, reinterpret_cast<const void* const*>(hp), 4, q, sx, sy, 1,
                                             ch, dr, 0, lr, 0, st), "dwtFloat2DInverseFromSymbols");
}
void dwtFloat3DInverseFromSymbols(float* d, float* b2, float* b1, const float* lp, const uint* const* hp, float q, int sx,
                                  int sy, int sz, int ch, int dr, int ds, int lr, int ls, cudaStream_t st) {
    report(cc_dwt_float_inverse_from_symbols(d, b2, b1, lp, reinterpret_cast<const void* const*>(hp), 4, q, sx, sy, sz,
                                             ch, dr, ds, lr, ls, st), "dwtFloat3DInverseFromSymbols");
}
void dwtFloat2DForwardFromByte(float* d, float* b, const byte* s, int sx, int sy, int ch, int dr, int sr, cudaStream_t st) {
    report(cc_dwt_float_forward_from_byte(d, nullptr, b, s, sx, sy, 1, ch, dr, 0, sr, 0, st), "dwtFloat2DForwardFromByte");
}
void dwtFloat3DForwardFromByte(float* d, float* b2, float* b1, const byte* s, int sx, int sy, int sz, int ch, int dr,
                               int ds, int sr, int ss, cudaStream_t st) {
    report(cc_dwt_float_forward_from_byte(d, b2, b1, s, sx, sy, sz, ch, dr, ds, sr, ss, st), "dwtFloat3DForwardFromByte");
}
void dwtFloat2DInverseToByte(byte* d, float* b, const float* s, int sx, int sy, int ch, int dr, int sr, cudaStream_t st) {
    report(cc_dwt_float_inverse_to_byte(d, nullptr, b, s, sx, sy, 1, ch, dr, 0, sr, 0, st), "dwtFloat2DInverseToByte");
}
void dwtFloat3DInverseToByte(byte* d, float* b2, float* b1, const float* s, int sx, int sy, int sz, int ch, int dr,
                             int ds, int sr, int ss, cudaStream_t st) {
    report(cc_dwt_float_inverse_to_byte(d, b2, b1, s, sx, sy, sz, ch, dr, ds, sr, ss, st), "dwtFloat3DInverseToByte");
}
void dwtFloat2DInverseFromSymbolsToByte(byte* d, float* b, const float* lp, const ushort* const* hp, float q, int sx,
                                        int sy, int ch, int dr, int lr, cudaStream_t st) {
    report(cc_dwt_float_inverse_from_symbols_to_byte(d, nullptr, b, lp, reinterpret_cast<const void* const*>(hp), 2, q,
                                                     sx, sy, 1, ch, dr, 0, lr, 0, st),
           "dwtFloat2DInverseFromSymbolsToByte");
}
void dwtFloat3DInverseFromSymbolsToByte(byte* d, float* b2, float* b1, const float* lp, const ushort* const* hp, float q,
                                        int sx, int sy, int sz, int ch, int dr, int ds, int lr, int ls, cudaStream_t st) {
    report(cc_dwt_float_inverse_from_symbols_to_byte(d, b2, b1, lp, reinterpret_cast<const void* const*>(hp), 2, q, sx,
                                                     sy, sz, ch, dr, ds, lr, ls, st),
           "dwtFloat3DInverseFromSymbolsToByte");
}
void dwtFloat2DForwardLowpassOnlyFromByte(float* d, float* b, const byte* s, int sx, int sy, int ch, int dr, int sr,
                                          cudaStream_t st) {
    report(cc_dwt_float2d_forward_lowpass_only_from_byte(d, b, s, sx, sy, ch, dr, sr, st),
           "dwtFloat2DForwardLowpassOnlyFromByte");
}
void dwtIntForwardLowpassOnly(short* d, short* b, const short* s, int sx, int sy, int dr, int sr, cudaStream_t st) {
    report(cc_dwt_int_forward_lowpass_only(d, b, s, sx, sy, dr, sr, st), "dwtIntForwardLowpassOnly");
}
void dwtIntForward(short* d, short* b, const short* s, int sx, int sy, int sz, int dr, int ds, int sr, int ss,
                   cudaStream_t st) {
    report(cc_dwt_int_forward(d, b, s, sx, sy, sz, dr, ds, sr, ss, st), "dwtIntForward");
}
void dwtIntInverse(short* d, short* b, const short* s, int sx, int sy, int sz, int dr, int ds, int sr, int ss,
                   cudaStream_t st) {
    report(cc_dwt_int_inverse(d, b, s, sx, sy, sz, dr, ds, sr, ss, st), "dwtIntInverse");
}

void symbolize(ushort* o, const short* i, uint sx, uint sy, uint sz, uint r, uint s) {
    report(cc_symbolize(o, i, sx, sy, sz, r, s, nullptr), "symbolize");
}
void unsymbolize(short* o, const ushort* i, uint sx, uint sy, uint sz, uint r, uint s) {
    report(cc_unsymbolize(o, i, sx, sy, sz, r, s, nullptr), "unsymbolize");
}
void quantizeToSymbols(ushort* o, const float* i, uint sx, uint sy, uint sz, float q, uint r, uint s, EQuantizeType t) {
    report(cc_quantize_to_symbols(o, 2, i, sx, sy, sz, q, r, s, int(t), nullptr), "quantizeToSymbols");
}
void quantizeToSymbolsRoundtrip(ushort* o, float* i, uint sx, uint sy, uint sz, float q, uint r, uint s, EQuantizeType t) {
    report(cc_quantize_to_symbols_roundtrip(o, 2, i, sx, sy, sz, q, r, s, int(t), nullptr), "quantizeToSymbolsRoundtrip");
}
void unquantizeFromSymbols(float* o, const ushort* i, uint sx, uint sy, uint sz, float q, uint r, uint s, EQuantizeType t) {
    report(cc_unquantize_from_symbols(o, i, 2, sx, sy, sz, q, r, s, int(t), nullptr), "unquantizeFromSymbols");
}
void quantizeToSymbols(uint* o, const float* i, uint sx, uint sy, uint sz, float q, uint r, uint s, EQuantizeType t) {
    report(cc_quantize_to_symbols(o, 4, i, sx, sy, sz, q, r, s, int(t), nullptr), "quantizeToSymbols");
}
void quantizeToSymbolsRoundtrip(uint* o, float* i, uint sx, uint sy, uint sz, float q, uint r, uint s, EQuantizeType t) {
    report(cc_quantize_to_symbols_roundtrip(o, 4, i, sx, sy, sz, q, r, s, int(t), nullptr), "quantizeToSymbolsRoundtrip");
}
void unquantizeFromSymbols(float* o, const uint* i, uint sx, uint sy, uint sz, float q, uint r, uint s, EQuantizeType t) {
    report(cc_unquantize_from_symbols(o, i, 4, sx, sy, sz, q, r, s, int(t), nullptr), "unquantizeFromSymbols");
}
void quantizeToSymbols2D(ushort* o, const float* i, uint sx, uint sy, float q, uint r, EQuantizeType t) { quantizeToSymbols(o, i, sx, sy, 1, q, r, 0, t); }
void quantizeToSymbolsRoundtrip2D(ushort* o, float* i, uint sx, uint sy, float q, uint r, EQuantizeType t) { quantizeToSymbolsRoundtrip(o, i, sx, sy, 1, q, r, 0, t); }
void unquantizeFromSymbols2D(float* o, const ushort* i, uint sx, uint sy, float q, uint r, EQuantizeType t) { unquantizeFromSymbols(o, i, sx, sy, 1, q, r, 0, t); }
void quantizeToSymbols2D(uint* o, const float* i, uint sx, uint sy, float q, uint r, EQuantizeType t) { quantizeToSymbols(o, i, sx, sy, 1, q, r, 0, t); }
void quantizeToSymbolsRoundtrip2D(uint* o, float* i, uint sx, uint sy, float q, uint r, EQuantizeType t) { quantizeToSymbolsRoundtrip(o, i, sx, sy, 1, q, r, 0, t); }
void unquantizeFromSymbols2D(float* o, const uint* i, uint sx, uint sy, float q, uint r, EQuantizeType t) { unquantizeFromSymbols(o, i, sx, sy, 1, q, r, 0, t); }
void quantizeToShort(short* o, const float* i, uint sx, uint sy, uint sz, float q, uint r, uint s, EQuantizeType t) {
    report(cc_quantize_to_short(o, i, sx, sy, sz, q, r, s, int(t), nullptr), "quantizeToShort");
}
void unquantizeFromShort(float* o, const short* i, uint sx, uint sy, uint sz, float q, uint r, uint s, EQuantizeType t) {
    report(cc_unquantize_from_short(o, i, sx, sy, sz, q, r, s, int(t), nullptr), "unquantizeFromShort");
}
void getMaxAbs(Instance* p, const float* d, uint n, float* m) { report(cc_get_max_abs(p->h, d, n, m), "getMaxAbs"); }

void floatToByte2D(byte* o, uint cc, uint c, const float* i, uint sx, uint sy, uint r) {
    report(cc_float_to_byte_2d(o, cc, c, i, sx, sy, r, nullptr), "floatToByte2D");
}
void byteToFloat2D(float* o, const byte* i, uint cc, uint c, uint sx, uint sy, uint r) {
    report(cc_byte_to_float_2d(o, i, cc, c, sx, sy, r, nullptr), "byteToFloat2D");
}
void quantizeDifferenceToSymbols2D(ushort* o, const float* i, float q, const byte* ref, uint cc, uint c, uint sx, uint sy,
                                   uint r, EQuantizeType t) {
    report(cc_quantize_difference_to_symbols_2d(o, i, q, ref, cc, c, sx, sy, r, int(t), nullptr),
           "quantizeDifferenceToSymbols2D");
}
void quantizeDifferenceToSymbolsRoundtrip2D(ushort* o, float* i, float q, const byte* ref, uint cc, uint c, uint sx,
                                            uint sy, uint r, EQuantizeType t) {
    report(cc_quantize_difference_to_symbols_roundtrip_2d(o, i, q, ref, cc, c, sx, sy, r, int(t), nullptr),
           "quantizeDifferenceToSymbolsRoundtrip2D");
}
void unquantizeDifferenceFromSymbols2D(float* o, const ushort* i, float q, const byte* ref, uint cc, uint c, uint sx,
                                       uint sy, uint r, EQuantizeType t, cudaStream_t st) {
    report(cc_unquantize_difference_from_symbols_2d(o, i, q, ref, cc, c, sx, sy, r, int(t), st),
           "unquantizeDifferenceFromSymbols2D");
}

void convertRGBtoYCoCg(uchar3* d, const uchar3* s, int n) {
    report(cc_convert_rgb_to_ycocg(reinterpret_cast<uint8_t*>(d), reinterpret_cast<const uint8_t*>(s), n, 3, nullptr),
           "convertRGBtoYCoCg");
}
void convertYCoCgtoRGB(uchar3* d, const uchar3* s, int n) {
    report(cc_convert_ycocg_to_rgb(reinterpret_cast<uint8_t*>(d), reinterpret_cast<const uint8_t*>(s), n, 3, nullptr),
           "convertYCoCgtoRGB");
}
void convertRGBtoYCoCg(uchar4* d, const uchar4* s, int n) {
    report(cc_convert_rgb_to_ycocg(reinterpret_cast<uint8_t*>(d), reinterpret_cast<const uint8_t*>(s), n, 4, nullptr),
           "convertRGBtoYCoCg");
}
void convertYCoCgtoRGB(uchar4* d, const uchar4* s, int n) {
    report(cc_convert_ycocg_to_rgb(reinterpret_cast<uint8_t*>(d), reinterpret_cast<const uint8_t*>(s), n, 4, nullptr),
           "convertYCoCgtoRGB");
}

bool getLSB(const short* d, uint* b, uint n) { return report(cc_get_lsb(d, b, n, nullptr), "getLSB"); }
bool removeLSB(short* d, uint* b, uint n, short s) { return report(cc_remove_lsb(d, b, n, s, nullptr), "removeLSB"); }
bool appendLSB(short* d, const uint* b, uint n, short s) { return report(cc_append_lsb(d, b, n, s, nullptr), "appendLSB"); }
bool shiftElems(short* d, uint n, short s) { return report(cc_shift_elems(d, n, s, nullptr), "shiftElems"); }

}  // namespace util
}  // namespace cudaCompress
