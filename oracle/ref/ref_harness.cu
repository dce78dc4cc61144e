// ref_harness.cu - C entry points over the reference cudaCompress library,
// compiled from the reference's own sources by oracle/ref/Makefile into
// oracle/_ref/libref_gpu.so.  TEST INFRASTRUCTURE ONLY: it lets the tests pin
// the CPU oracle against the reference's table design (CPU-only entry points)
// and, on a GPU, produce reference bitstreams and DWT outputs.
#include <cstdint>
#include <cstring>
#include <deque>
#include <map>
#include <queue>
#include <string>
#include <vector>
#include <cuda_runtime.h>

// HuffmanEncodeTable::build and the decode table internals are private in the
// reference; expose them to this harness only.
#define private public
#include <cudaCompress/Instance.h>
#include <cudaCompress/InstanceImpl.h>
#include <cudaCompress/HuffmanTable.h>
#include <cudaCompress/Encode.h>
#include <cudaCompress/util/Bits.h>
#include <cudaCompress/util/DWT.h>
#include <cudaCompress/util/Quantize.h>
#include <cudaCompress/util/YCoCg.h>
#undef private

using namespace cudaCompress;

extern "C" {

// Reference table build + serialization (HuffmanTable.cu:470-596) on the CPU.
int ref_huffman_build(const uint32_t* hist, uint32_t bins, uint32_t symbolMax, uint32_t log2Max,
                      uint32_t* codewords, uint32_t* lengths, uint32_t* tableWords, uint32_t cap,
                      uint32_t* tableBits) {
    Instance inst;
    inst.m_log2HuffmanDistinctSymbolCountMax = log2Max;
    int maxLen;
    {
        HuffmanEncodeTable t(&inst);
        t.build(hist, bins);
        t.m_symbolMax = symbolMax;
        for (uint32_t i = 0; i < t.m_codewordTableSize; ++i) {
            codewords[i] = t.m_pCodewords[i];
            lengths[i] = t.m_pCodewordLengths[i];
        }
        std::vector<uint> v;
        BitStream bs(&v);
        t.writeToBitStream(&inst, bs);
        *tableBits = bs.getBitSize();
        if (v.size() > cap) return -2;
        std::memcpy(tableWords, v.data(), v.size() * 4);
        maxLen = int(t.m_codewordCountPerLength.size());
    }
    return maxLen;
}

void* ref_create(int dev, uint32_t streamCountMax, uint32_t elemMax, uint32_t cb, uint32_t log2Max) {
    return createInstance(dev, streamCountMax, elemMax, cb, log2Max);
}
void ref_destroy(void* p) { destroyInstance(static_cast<Instance*>(p)); }

// kind 0 = encodeRLHuff, 1 = encodeHuff; streams contiguous on the device.
int ref_encode(void* p, int kind, int symBytes, void* dSymbols, uint32_t S, uint32_t n,
               uint32_t* words, uint32_t cap, uint32_t* bitSize, uint32_t* bitPos) {
    Instance* inst = static_cast<Instance*>(p);
    std::vector<uint> v(words, words + (*bitSize + 31) / 32);
    BitStream bs(&v);
    bs.setBitSize(*bitSize);
    bs.setBitPosition(*bitPos);
    bool ok;
    if (symBytes == 2) {
        std::vector<Symbol16*> s(S);
        for (uint32_t i = 0; i < S; ++i) s[i] = static_cast<Symbol16*>(dSymbols) + size_t(i) * n;
        ok = kind == 0 ? encodeRLHuff(inst, bs, s.data(), S, n) : encodeHuff(inst, bs, s.data(), S, n);
    } else {
        std::vector<Symbol32*> s(S);
        for (uint32_t i = 0; i < S; ++i) s[i] = static_cast<Symbol32*>(dSymbols) + size_t(i) * n;
        ok = kind == 0 ? encodeRLHuff(inst, bs, s.data(), S, n) : encodeHuff(inst, bs, s.data(), S, n);
    }
    cudaDeviceSynchronize();
    if (!ok) return -1;
    if (v.size() > cap) return -2;
    std::memcpy(words, v.data(), v.size() * 4);
    *bitSize = bs.getBitSize();
    *bitPos = bs.getBitPosition();
    return 0;
}

// As ref_encode with stream i at dSymbols + i * stride elements: encodeHuff
// pads each input stream with 0xFFFF up to a multiple of 8 symbols
// (Histogram.cu:90-106), so the generator leaves that slack between streams.
int ref_encode_strided(void* p, int kind, int symBytes, void* dSymbols, uint32_t S, uint32_t n, uint32_t stride,
                       uint32_t* words, uint32_t cap, uint32_t* bitSize, uint32_t* bitPos) {
    Instance* inst = static_cast<Instance*>(p);
    std::vector<uint> v(words, words + (*bitSize + 31) / 32);
    BitStream bs(&v);
    bs.setBitSize(*bitSize);
    bs.setBitPosition(*bitPos);
    bool ok;
    if (symBytes == 2) {
        std::vector<Symbol16*> s(S);
        for (uint32_t i = 0; i < S; ++i) s[i] = static_cast<Symbol16*>(dSymbols) + size_t(i) * stride;
        ok = kind == 0 ? encodeRLHuff(inst, bs, s.data(), S, n) : encodeHuff(inst, bs, s.data(), S, n);
    } else {
        std::vector<Symbol32*> s(S);
        for (uint32_t i = 0; i < S; ++i) s[i] = static_cast<Symbol32*>(dSymbols) + size_t(i) * stride;
        ok = kind == 0 ? encodeRLHuff(inst, bs, s.data(), S, n) : encodeHuff(inst, bs, s.data(), S, n);
    }
    cudaDeviceSynchronize();
    if (!ok) return -1;
    if (v.size() > cap) return -2;
    std::memcpy(words, v.data(), v.size() * 4);
    *bitSize = bs.getBitSize();
    *bitPos = bs.getBitPosition();
    return 0;
}

void ref_dwt_float3d_fwd(float* dst, float* buf2, float* buf1, const float* src, int nx, int ny, int nz) {
    util::dwtFloat3DForward(dst, buf2, buf1, src, nx, ny, nz);
    cudaDeviceSynchronize();
}
void ref_dwt_float3d_inv(float* dst, float* buf2, float* buf1, const float* src, int nx, int ny, int nz) {
    util::dwtFloat3DInverse(dst, buf2, buf1, src, nx, ny, nz);
    cudaDeviceSynchronize();
}
void ref_dwt_int_fwd(short* dst, short* buf, const short* src, int nx, int ny, int nz) {
    util::dwtIntForward(dst, buf, src, nx, ny, nz);
    cudaDeviceSynchronize();
}
void ref_dwt_int_inv(short* dst, short* buf, const short* src, int nx, int ny, int nz) {
    util::dwtIntInverse(dst, buf, src, nx, ny, nz);
    cudaDeviceSynchronize();
}
void ref_quantize_to_symbols(uint16_t* out, const float* src, uint32_t nx, uint32_t ny, uint32_t nz, float step,
                             uint32_t rowPitch, uint32_t slicePitch) {
    util::quantizeToSymbols(out, src, nx, ny, nz, step, rowPitch, slicePitch);
    cudaDeviceSynchronize();
}

// ---- the 2D image side of util (DWT byte / lowpass-only variants, byte
// quantizers, YCoCg, Bits); all on the default stream as the reference runs
// them, synchronized before returning.
void ref_dwt_float_fwd_from_byte(float* dst, float* buf2, float* buf1, const uint8_t* src, int nx, int ny, int nz,
                                 int ch) {
    if (nz > 1) util::dwtFloat3DForwardFromByte(dst, buf2, buf1, src, nx, ny, nz, ch);
    else util::dwtFloat2DForwardFromByte(dst, buf1, src, nx, ny, ch);
    cudaDeviceSynchronize();
}
void ref_dwt_float_inv_to_byte(uint8_t* dst, float* buf2, float* buf1, const float* src, int nx, int ny, int nz,
                               int ch) {
    if (nz > 1) util::dwtFloat3DInverseToByte(dst, buf2, buf1, src, nx, ny, nz, ch);
    else util::dwtFloat2DInverseToByte(dst, buf1, src, nx, ny, ch);
    cudaDeviceSynchronize();
}
void ref_dwt_float_inv_from_symbols_to_byte(uint8_t* dst, float* buf2, float* buf1, const float* lowpass,
                                            const uint16_t* const* dHighpass, float step, int nx, int ny, int nz,
                                            int ch) {
    const ushort* const* hp = reinterpret_cast<const ushort* const*>(dHighpass);
    if (nz > 1) util::dwtFloat3DInverseFromSymbolsToByte(dst, buf2, buf1, lowpass, hp, step, nx, ny, nz, ch);
    else util::dwtFloat2DInverseFromSymbolsToByte(dst, buf1, lowpass, hp, step, nx, ny, ch);
    cudaDeviceSynchronize();
}
void ref_dwt_float2d_lowpass_from_byte(float* dst, float* buf, const uint8_t* src, int nx, int ny, int ch) {
    util::dwtFloat2DForwardLowpassOnlyFromByte(dst, buf, src, nx, ny, ch);
    cudaDeviceSynchronize();
}
void ref_dwt_int_lowpass(short* dst, short* buf, const short* src, int nx, int ny) {
    util::dwtIntForwardLowpassOnly(dst, buf, src, nx, ny);
    cudaDeviceSynchronize();
}
void ref_float_to_byte_2d(uint8_t* out, uint32_t chCount, uint32_t ch, const float* in, uint32_t nx, uint32_t ny,
                          uint32_t rowPitch) {
    util::floatToByte2D(out, chCount, ch, in, nx, ny, rowPitch);
    cudaDeviceSynchronize();
}
void ref_byte_to_float_2d(float* out, const uint8_t* in, uint32_t chCount, uint32_t ch, uint32_t nx, uint32_t ny,
                          uint32_t rowPitch) {
    util::byteToFloat2D(out, in, chCount, ch, nx, ny, rowPitch);
    cudaDeviceSynchronize();
}
void ref_quantize_difference_2d(uint16_t* sym, float* data, float step, const uint8_t* ref, uint32_t chCount,
                                uint32_t ch, uint32_t nx, uint32_t ny, uint32_t rowPitch, int type, int roundtrip) {
    const util::EQuantizeType t = type ? util::QUANTIZE_UNIFORM : util::QUANTIZE_DEADZONE;
    if (roundtrip) util::quantizeDifferenceToSymbolsRoundtrip2D(sym, data, step, ref, chCount, ch, nx, ny, rowPitch, t);
    else util::quantizeDifferenceToSymbols2D(sym, data, step, ref, chCount, ch, nx, ny, rowPitch, t);
    cudaDeviceSynchronize();
}
void ref_unquantize_difference_2d(float* data, const uint16_t* sym, float step, const uint8_t* ref, uint32_t chCount,
                                  uint32_t ch, uint32_t nx, uint32_t ny, uint32_t rowPitch, int type) {
    const util::EQuantizeType t = type ? util::QUANTIZE_UNIFORM : util::QUANTIZE_DEADZONE;
    util::unquantizeDifferenceFromSymbols2D(data, sym, step, ref, chCount, ch, nx, ny, rowPitch, t);
    cudaDeviceSynchronize();
}
void ref_ycocg(uint8_t* dst, const uint8_t* src, int n, int channels, int toYCoCg) {
    if (channels == 3) {
        if (toYCoCg) util::convertRGBtoYCoCg(reinterpret_cast<uchar3*>(dst), reinterpret_cast<const uchar3*>(src), n);
        else util::convertYCoCgtoRGB(reinterpret_cast<uchar3*>(dst), reinterpret_cast<const uchar3*>(src), n);
    } else {
        if (toYCoCg) util::convertRGBtoYCoCg(reinterpret_cast<uchar4*>(dst), reinterpret_cast<const uchar4*>(src), n);
        else util::convertYCoCgtoRGB(reinterpret_cast<uchar4*>(dst), reinterpret_cast<const uchar4*>(src), n);
    }
    cudaDeviceSynchronize();
}
// The lossless 2D heightfield codec of the scope, composed from the
// reference library's own calls: per level util::dwtIntForward (2D, sizeZ 1),
// the three detail bands symbolized in x + 2y order (util::symbolize with the
// level's pitch, CompressHeightfield.cpp:119-126) and coded with one
// encodeRLHuff; the last lowpass band symbolized and coded with encodeHuff.
// Stream order as compressVolumeLossless (CompressVolume.cpp:234-272): the
// lowpass segment first, then the levels coarse to fine, each appended at a
// word boundary.  dImg is the device image (nx * ny shorts, dense).
int ref_heightfield_compress(const short* dImg, uint32_t nx, uint32_t ny, uint32_t levels, uint32_t* words,
                             uint32_t cap, uint32_t* nWords) {
    Instance* inst = createInstance(0, 3, (nx / 2) * (ny / 2), 128, 14);
    if (!inst) return -1;
    const size_t n = size_t(nx) * ny;
    short *cur = nullptr, *coef = nullptr, *buf = nullptr;
    Symbol16* sym = nullptr;
    const size_t bandCap = n / 4 + 64;          // encode pads each stream by up to 8 symbols
    cudaMalloc(&cur, n * sizeof(short));
    cudaMalloc(&coef, n * sizeof(short));
    cudaMalloc(&buf, n * sizeof(short));
    cudaMalloc(&sym, 3 * bandCap * sizeof(Symbol16));
    cudaMemcpy(cur, dImg, n * sizeof(short), cudaMemcpyDeviceToDevice);
    std::vector<std::vector<uint>> levelBits(levels);
    bool ok = true;
    uint32_t sx = nx, sy = ny;
    for (uint32_t l = 0; l < levels && ok; ++l) {
        util::dwtIntForward(coef, buf, cur, int(sx), int(sy), 1);
        const uint32_t hx = sx / 2, hy = sy / 2;
        std::vector<Symbol16*> s(3);
        for (uint32_t b = 1; b < 4; ++b) {
            s[b - 1] = sym + (b - 1) * bandCap;
            const short* src = coef + (b % 2) * hx + (b / 2) * size_t(hy) * sx;
            util::symbolize(s[b - 1], src, hx, hy, 1, sx, sx * sy);
        }
        BitStream bs(&levelBits[l]);
        ok = encodeRLHuff(inst, bs, s.data(), 3, hx * hy);
        cudaMemcpy2D(cur, hx * sizeof(short), coef, sx * sizeof(short), hx * sizeof(short), hy,
                     cudaMemcpyDeviceToDevice);
        sx = hx;
        sy = hy;
    }
    std::vector<uint> bits;
    if (ok) {
        util::symbolize(sym, cur, sx, sy, 1, sx, sx * sy);
        BitStream bs(&bits);
        ok = encodeHuff(inst, bs, &sym, 1, sx * sy);
    }
    cudaDeviceSynchronize();
    if (ok) {
        for (int l = int(levels) - 1; l >= 0; --l) bits.insert(bits.end(), levelBits[l].begin(), levelBits[l].end());
    }
    cudaFree(cur);
    cudaFree(coef);
    cudaFree(buf);
    cudaFree(sym);
    destroyInstance(inst);
    if (!ok) return -2;
    if (bits.size() > cap) return -3;
    std::memcpy(words, bits.data(), bits.size() * 4);
    *nWords = uint32_t(bits.size());
    return 0;
}

// mode 0 getLSB, 1 removeLSB (bits may be null), 2 appendLSB, 3 shiftElems
void ref_lsb(int mode, short* data, uint32_t* bits, uint32_t n, short shift) {
    if (mode == 0) util::getLSB(data, bits, n);
    else if (mode == 1) util::removeLSB(data, bits, n, shift);
    else if (mode == 2) util::appendLSB(data, bits, n, shift);
    else util::shiftElems(data, n, shift);
    cudaDeviceSynchronize();
}

}  // extern "C"
