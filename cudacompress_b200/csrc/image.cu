// image.cu - the 2D image side of the library: the byte-image quantizers of
// util::Quantize (Quantize.h:24-26, 58-61), the YCoCg colour transform
// (util/YCoCg.cu), the least-significant-bit planes of util::Bits
// (util/Bits.cu), and the one-level image and heightfield codecs of the
// reference's examples (CompressImage.cpp:71-340, CompressHeightfield.cpp:82-216)
// built on them and on the library's DWT, quantizer and entropy coder.
#include <cstring>
#include <vector>

#include "capi_internal.cuh"

namespace ccb {
namespace {

// ---- byte images (Quantize.cuh:15-23, QuantizeKernels.cui:11-34, 227-285) ----
__device__ __forceinline__ u8 floatToByte(float v) { return u8(fminf(fmaxf(v + 128.5f, 0.0f), 255.0f)); }
__device__ __forceinline__ float byteToFloat(u8 v) { return float(v) - 128.0f; }

// 2D index of thread i in a size_x x size_y image (false past the end).
__device__ __forceinline__ bool pixelOf(u32 sx, u32 sy, u32& x, u32& y) {
    const u64 i = u64(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= u64(sx) * sy) return false;
    y = u32(i / sx);
    x = u32(i - u64(y) * sx);
    return true;
}

__global__ void k_floatToByte2D(u8* __restrict__ out, u32 stride, const float* __restrict__ in, u32 sx, u32 sy,
                                u32 rowPitch) {
    u32 x, y;
    if (!pixelOf(sx, sy, x, y)) return;
    out[(u64(y) * sx + x) * stride] = floatToByte(in[u64(y) * rowPitch + x]);
}

__global__ void k_byteToFloat2D(float* __restrict__ out, const u8* __restrict__ in, u32 stride, u32 sx, u32 sy,
                                u32 rowPitch) {
    u32 x, y;
    if (!pixelOf(sx, sy, x, y)) return;
    out[u64(y) * rowPitch + x] = byteToFloat(in[(u64(y) * sx + x) * stride]);
}

// Difference to a byte reference, quantized to 16-bit symbols; the round trip
// writes back reference + the value of the STORED (16-bit) symbol.
template <bool kRoundtrip>
__global__ void k_quantizeDifference2D(u16* __restrict__ sym, float* data, float step, float inv,
                                       const u8* __restrict__ ref, u32 stride, u32 sx, u32 sy, u32 rowPitch, int type) {
    u32 x, y;
    if (!pixelOf(sx, sy, x, y)) return;
    const u64 d = u64(y) * sx + x, s = u64(y) * rowPitch + x;
    const float r = byteToFloat(ref[d * stride]);
    const u16 q = u16(symbolizeI(quantizeV(data[s] - r, inv, type)));
    sym[d] = q;
    if (kRoundtrip) data[s] = unquantizeV(unsymbolizeI(q), step, type) + r;
}

__global__ void k_unquantizeDifference2D(float* __restrict__ data, const u16* __restrict__ sym, float step,
                                         const u8* __restrict__ ref, u32 stride, u32 sx, u32 sy, u32 rowPitch, int type) {
    u32 x, y;
    if (!pixelOf(sx, sy, x, y)) return;
    const u64 d = u64(y) * sx + x;
    data[u64(y) * rowPitch + x] = unquantizeV(unsymbolizeI(sym[d]), step, type) + byteToFloat(ref[d * stride]);
}

// ---- YCoCg (YCoCg.cu:6-88): the non-reversible transform, integer math ----
template <int kCh, bool kToYCoCg>
__global__ void k_ycocg(u8* dst, const u8* src, u32 n) {
    for (u64 i = u64(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += u64(gridDim.x) * blockDim.x) {
        int a, b, c, w = 0;
        if (kCh == 4) {
            const uchar4 p = reinterpret_cast<const uchar4*>(src)[i];
            a = p.x; b = p.y; c = p.z; w = p.w;
        } else {
            a = src[3 * i]; b = src[3 * i + 1]; c = src[3 * i + 2];
        }
        int o0, o1, o2;
        if (kToYCoCg) {
            o0 = (a + b * 2 + c + 2) / 4;
            o1 = (a - c + 1) / 2 + 127;
            o2 = (-a + b * 2 - c + 2) / 4 + 127;
        } else {
            o0 = min(max(a + b - c, 0), 255);
            o1 = min(max(a + c - 127, 0), 255);
            o2 = min(max(a - b - c + 254, 0), 255);
        }
        if (kCh == 4) {
            reinterpret_cast<uchar4*>(dst)[i] = make_uchar4(u8(o0), u8(o1), u8(o2), u8(w));
        } else {
            dst[3 * i] = u8(o0); dst[3 * i + 1] = u8(o1); dst[3 * i + 2] = u8(o2);
        }
    }
}

// ---- least significant bits (Bits.cu:13-174) ----
// Bit j of word w belongs to element 32 w + j.  A warp walks 32 words
// (1024 elements): one coalesced 64-byte load per word, the word's bits
// gathered with one ballot (get / remove) or spread with one shuffle
// (append).  Elements past elem_count are neither read nor written; their
// bits are 0.
enum LsbMode { kLsbGet = 0, kLsbRemove = 1, kLsbAppend = 2 };

template <int kMode>
__global__ void __launch_bounds__(256) k_lsb(i16* data, u32* bits, u32 n, i16 shift) {
    const u32 lane = threadIdx.x & 31u;
    const u64 warp = (u64(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const u64 warps = (u64(gridDim.x) * blockDim.x) >> 5;
    const u64 nWords = ceilDiv(n, 32);
    for (u64 w0 = warp * 32; w0 < nWords; w0 += warps * 32) {
        u32 mine = 0;   // word w0 + lane
        if (kMode == kLsbAppend && w0 + lane < nWords) mine = bits[w0 + lane];
        for (u32 j = 0; j < 32 && w0 + j < nWords; ++j) {
            const u64 e = (w0 + j) * 32 + lane;
            const bool in = e < n;
            const i16 v = in ? data[e] : i16(0);
            if (kMode == kLsbAppend) {
                const u32 wj = __shfl_sync(0xffffffffu, mine, int(j));
                const i16 t = i16((int(v) * 2) | int((wj >> lane) & 1u));
                if (in) data[e] = i16(t + shift);
            } else {
                const i16 t = kMode == kLsbRemove ? i16(v + shift) : v;
                const u32 b = __ballot_sync(0xffffffffu, in && (t & 1));
                if (lane == j) mine = b;
                if (kMode == kLsbRemove && in) data[e] = i16((int(t) + (t < 0 ? -1 : 0)) / 2);
            }
        }
        if (kMode != kLsbAppend && bits && w0 + lane < nWords) bits[w0 + lane] = mine;
    }
}

__global__ void k_shiftElems(i16* data, u32 n, i16 shift) {
    for (u64 i = u64(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += u64(gridDim.x) * blockDim.x)
        data[i] = i16(data[i] + shift);
}

unsigned pixelGrid(u64 n) { return unsigned(ceilDiv(n, 256)); }
// grid-stride kernels: enough CTAs to fill the GPU, no more than the work
unsigned strideGrid(u64 items, u64 perCta) { return unsigned(std::max<u64>(1, std::min<u64>(ceilDiv(items, perCta), 148 * 8))); }

int lsbLaunch(int mode, i16* data, u32* bits, u32 n, i16 shift, cudaStream_t st, const char* what) {
    if (!data || (mode != kLsbRemove && !bits)) { setError("%s: null argument", what); return CC_ERR_INVALID_ARGUMENT; }
    if (!n) return CC_OK;
    const unsigned g = strideGrid(ceilDiv(n, 32), 8 * 32);   // 8 warps x 32 words per CTA
    if (mode == kLsbGet) k_lsb<kLsbGet><<<g, 256, 0, st>>>(data, bits, n, shift);
    else if (mode == kLsbRemove) k_lsb<kLsbRemove><<<g, 256, 0, st>>>(data, bits, n, shift);
    else k_lsb<kLsbAppend><<<g, 256, 0, st>>>(data, bits, n, shift);
    countLaunch();
    CC_TRY_CUDA(cudaGetLastError(), what);
    return CC_OK;
}

bool imageArgsOk(u32 sx, u32 sy, u32 chTotal, u32 chProc, const char* what) {
    if (sx < 8 || sy < 8 || sx % 2 || sy % 2) {
        setError("%s: sizes must be even and >= 8 (got %u x %u)", what, sx, sy);
        return false;
    }
    if (chTotal < 1 || chTotal > 4 || chProc < 1 || chProc > chTotal) {
        setError("%s: channel counts must satisfy 1 <= channelCountToProcess <= channelCountTotal <= 4", what);
        return false;
    }
    return true;
}

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

// Host copy of device words (the bit stream walk happens on the host).
int downloadWords(cc_instance* I, const u32* d, u64 words, std::vector<u32>& host, const char* what) {
    if (words > I->hostWordsMax) { setError("%s: stream larger than instance staging", what); return CC_ERR_CAPACITY; }
    host.resize(words);
    if (!words) return CC_OK;
    CC_TRY_CUDA(cudaMemcpyAsync(I->hostWords, d, words * 4, cudaMemcpyDeviceToHost, I->stream), "download stream");
    CC_TRY_CUDA(cudaStreamSynchronize(I->stream), "download stream");
    std::memcpy(host.data(), I->hostWords, words * 4);
    return CC_OK;
}

// ---- image codec (CompressImage.cpp:71-340) ----
// Per image: for each processed channel the 9/7 DWT of the byte channel; the
// LL band minus the lowpass reference (the decoded next-coarser image) and
// the three highpass bands round-trip quantized to 16-bit symbols; the image
// overwritten with its reconstruction.  Streams of an image: the LL
// differences of all channels, then each channel's 3 highpass bands (x + 2y
// order); all of them coded by one encodeRLHuff call.  Images share one
// encode call (and one decode call) here as in compressImagesOneLevel.
int compressImages(cc_instance* I, cc_image* imgs, u32 count, u32 sx, u32 sy, u32 chTotal, u32 chProc, bool oneOut,
                   const char* what) {
    if (!I || (count && !imgs)) { setError("%s: bad argument", what); return CC_ERR_INVALID_ARGUMENT; }
    if (!imageArgsOk(sx, sy, chTotal, chProc, what)) return CC_ERR_INVALID_ARGUMENT;
    if (I->symBytes != 2) { setError("%s: needs a 16-bit-symbol instance", what); return CC_ERR_INVALID_ARGUMENT; }
    const u32 perImage = 4 * chProc, hx = sx / 2, hy = sy / 2;
    const u64 n = u64(hx) * hy;
    if (I->streamCountMax < perImage || I->elemCountPerStreamMax < n) {
        setError("%s: instance needs >= %u streams of >= %llu symbols", what, perImage, (unsigned long long)n);
        return CC_ERR_CAPACITY;
    }
    for (u32 i = 0; i < count; ++i)
        if (!imgs[i].d_image || !imgs[i].d_lowpass_reference || !imgs[i].d_words) {
            setError("%s: image %u has a null pointer", what, i);
            return CC_ERR_INVALID_ARGUMENT;
        }
    if (!count) return CC_OK;
    DeviceGuard deviceGuard(I->device);
    cudaStream_t st = I->stream;
    const u64 pixels = u64(sx) * sy, streams = u64(perImage) * count;
    // scratch words of all images when they are copied out one by one
    u64 scratchWords = 0;
    if (!oneOut) for (u32 i = 0; i < count; ++i) scratchWords += imgs[i].capacity_words;
    Bump b{nullptr};
    b.take<float>(pixels);
    b.take<float>(pixels);
    b.take<u16>(streams * n + 64);
    b.take<u32>(scratchWords);
    int rc = ensurePipelineWork(I, b.off + 1024);
    if (rc) return rc;
    Bump w{I->pipeWork};
    float* dwt0 = w.take<float>(pixels);
    float* dwt1 = w.take<float>(pixels);
    u16* syms = w.take<u16>(streams * n + 64);
    u32* scratch = w.take<u32>(scratchWords);
    std::vector<EncStream> es;
    std::vector<EncGroup> groups;
    for (u32 i = 0; i < count; ++i) {
        const cc_image& im = imgs[i];
        u16* s0 = syms + u64(i) * perImage * n;
        for (u32 c = 0; c < chProc; ++c) {
            u16* lp = s0 + u64(c) * n;
            u16* hp = s0 + (chProc + 3 * u64(c)) * n;
            if ((rc = cc_dwt_float_forward_from_byte(dwt1, nullptr, dwt0, im.d_image + c, int(sx), int(sy), 1,
                                                     int(chTotal), 0, 0, 0, 0, st))) return rc;
            if ((rc = cc_quantize_difference_to_symbols_roundtrip_2d(lp, dwt1, im.quant_step, im.d_lowpass_reference,
                                                                     chTotal, c, hx, hy, sx, 0, st))) return rc;
            for (u32 k = 1; k < 4; ++k) {
                const u64 off = u64(k % 2) * hx + u64(k / 2) * hy * sx;
                if ((rc = cc_quantize_to_symbols_roundtrip(hp + (k - 1) * n, 2, dwt1 + off, hx, hy, 1, im.quant_step,
                                                           sx, 0, 0, st))) return rc;
            }
            if ((rc = cc_dwt_float_inverse_to_byte(im.d_image + c, nullptr, dwt0, dwt1, int(sx), int(sy), 1,
                                                   int(chTotal), 0, 0, 0, 0, st))) return rc;
        }
        const u32 first = u32(es.size());
        for (u32 k = 0; k < perImage; ++k) es.push_back(EncStream{s0 + u64(k) * n, u32(n), 0, first, perImage, KIND_RLHUFF});
        groups.push_back(EncGroup{first, perImage});
    }
    u64 total = 0;
    if (oneOut) {
        if ((rc = encodeGroups(I, es, groups, imgs[0].d_words, imgs[0].capacity_words, &total))) return rc;
        CC_TRY_CUDA(cudaStreamSynchronize(st), what);
        if (total * 32 > 0xffffffffull) { setError("%s: stream exceeds 2^32 bits", what); return CC_ERR_CAPACITY; }
        imgs[0].bit_size = u32(total * 32);
        return CC_OK;
    }
    std::vector<u64> at;
    if ((rc = encodeGroups(I, es, groups, scratch, scratchWords, &total, &at))) return rc;
    for (u32 i = 0; i < count; ++i) {
        const u64 words = at[i + 1] - at[i];
        if (words > imgs[i].capacity_words) {
            setError("%s: image %u needs %llu words", what, i, (unsigned long long)words);
            return CC_ERR_CAPACITY;
        }
        if (words * 32 > 0xffffffffull) { setError("%s: stream exceeds 2^32 bits", what); return CC_ERR_CAPACITY; }
        CC_TRY_CUDA(cudaMemcpyAsync(imgs[i].d_words, scratch + at[i], words * 4, cudaMemcpyDeviceToDevice, st),
                    "copy image stream");
        imgs[i].bit_size = u32(words * 32);
    }
    CC_TRY_CUDA(cudaStreamSynchronize(st), what);
    return CC_OK;
}

int decompressImages(cc_instance* I, const cc_image* imgs, u32 count, u32 sx, u32 sy, u32 chTotal, u32 chProc,
                     const char* what) {
    if (!I || (count && !imgs)) { setError("%s: bad argument", what); return CC_ERR_INVALID_ARGUMENT; }
    if (!imageArgsOk(sx, sy, chTotal, chProc, what)) return CC_ERR_INVALID_ARGUMENT;
    if (I->symBytes != 2) { setError("%s: needs a 16-bit-symbol instance", what); return CC_ERR_INVALID_ARGUMENT; }
    const u32 perImage = 4 * chProc, hx = sx / 2, hy = sy / 2;
    const u64 n = u64(hx) * hy;
    if (u64(perImage) * count > I->streamCountMax || I->elemCountPerStreamMax < n) {
        setError("%s: instance needs >= %llu streams of >= %llu symbols", what, (unsigned long long)perImage * count,
                 (unsigned long long)n);
        return CC_ERR_CAPACITY;
    }
    for (u32 i = 0; i < count; ++i)
        if (!imgs[i].d_image || !imgs[i].d_lowpass_reference || (imgs[i].bit_size && !imgs[i].d_words)) {
            setError("%s: image %u has a null pointer", what, i);
            return CC_ERR_INVALID_ARGUMENT;
        }
    if (!count) return CC_OK;
    DeviceGuard deviceGuard(I->device);
    cudaStream_t st = I->stream;
    const u64 pixels = u64(sx) * sy, streams = u64(perImage) * count;
    Bump b{nullptr};
    b.take<float>(pixels);
    b.take<float>(pixels);
    b.take<u16>(streams * n + 64);
    b.take<const void*>(3 * u64(chProc) * count);
    int rc = ensurePipelineWork(I, b.off + 1024);
    if (rc) return rc;
    Bump w{I->pipeWork};
    float* dwt0 = w.take<float>(pixels);
    float* dwt1 = w.take<float>(pixels);
    u16* syms = w.take<u16>(streams * n + 64);
    const void** dPtrs = w.take<const void*>(3 * u64(chProc) * count);
    std::vector<std::vector<u32>> host(count);
    std::vector<const u32*> hw(count);
    std::vector<u32> bits(count), pos(count, 0), bsIndex(streams);
    std::vector<void*> outs(streams);
    std::vector<const void*> hostPtrs(3 * u64(chProc) * count);
    for (u32 i = 0; i < count; ++i) {
        if ((rc = downloadWords(I, imgs[i].d_words, ceilDiv(imgs[i].bit_size, 32), host[i], what))) return rc;
        hw[i] = host[i].data();
        bits[i] = imgs[i].bit_size;
        u16* s0 = syms + u64(i) * perImage * n;
        for (u32 k = 0; k < perImage; ++k) {
            outs[u64(i) * perImage + k] = s0 + u64(k) * n;
            bsIndex[u64(i) * perImage + k] = i;
        }
        for (u32 c = 0; c < chProc; ++c)
            for (u32 k = 0; k < 3; ++k) hostPtrs[(u64(i) * chProc + c) * 3 + k] = s0 + (chProc + 3 * u64(c) + k) * n;
    }
    CC_TRY_CUDA(cudaMemcpyAsync(dPtrs, hostPtrs.data(), hostPtrs.size() * sizeof(void*), cudaMemcpyHostToDevice, st),
                "upload band pointers");
    if ((rc = decodeDevice(I, KIND_RLHUFF, hw.data(), bits.data(), pos.data(), count, bsIndex.data(), outs.data(),
                           u32(streams), u32(n)))) return rc;
    for (u32 i = 0; i < count; ++i) {
        const cc_image& im = imgs[i];
        const u16* s0 = syms + u64(i) * perImage * n;
        for (u32 c = 0; c < chProc; ++c) {
            if ((rc = cc_unquantize_difference_from_symbols_2d(dwt0, s0 + u64(c) * n, im.quant_step,
                                                               im.d_lowpass_reference, chTotal, c, hx, hy, sx, 0, st)))
                return rc;
            if ((rc = cc_dwt_float_inverse_from_symbols_to_byte(im.d_image + c, nullptr, dwt1, dwt0,
                                                                dPtrs + (u64(i) * chProc + c) * 3, 2, im.quant_step,
                                                                int(sx), int(sy), 1, int(chTotal), 0, 0, 0, 0, st)))
                return rc;
        }
    }
    CC_TRY_CUDA(cudaStreamSynchronize(st), what);
    return cc_decode_status(I);
}

}  // namespace
}  // namespace ccb

using namespace ccb;

extern "C" {

int cc_float_to_byte_2d(uint8_t* out, uint32_t chCount, uint32_t ch, const float* in, uint32_t sx, uint32_t sy,
                        uint32_t rowPitch, void* stream) {
    if (!rowPitch) rowPitch = sx;
    if (!u64(sx) * sy) return CC_OK;
    k_floatToByte2D<<<pixelGrid(u64(sx) * sy), 256, 0, static_cast<cudaStream_t>(stream)>>>(out + ch, chCount, in, sx,
                                                                                            sy, rowPitch);
    countLaunch();
    CC_TRY_CUDA(cudaGetLastError(), "floatToByte2D");
    return CC_OK;
}

int cc_byte_to_float_2d(float* out, const uint8_t* in, uint32_t chCount, uint32_t ch, uint32_t sx, uint32_t sy,
                        uint32_t rowPitch, void* stream) {
    if (!rowPitch) rowPitch = sx;
    if (!u64(sx) * sy) return CC_OK;
    k_byteToFloat2D<<<pixelGrid(u64(sx) * sy), 256, 0, static_cast<cudaStream_t>(stream)>>>(out, in + ch, chCount, sx,
                                                                                            sy, rowPitch);
    countLaunch();
    CC_TRY_CUDA(cudaGetLastError(), "byteToFloat2D");
    return CC_OK;
}

int cc_quantize_difference_to_symbols_2d(uint16_t* sym, const float* data, float step, const uint8_t* ref,
                                         uint32_t chCount, uint32_t ch, uint32_t sx, uint32_t sy, uint32_t rowPitch,
                                         int type, void* stream) {
    if (!rowPitch) rowPitch = sx;
    if (!u64(sx) * sy) return CC_OK;
    const float inv = 1.0f / step;   // Quantize.cu:289: reciprocal on the host
    k_quantizeDifference2D<false><<<pixelGrid(u64(sx) * sy), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        sym, const_cast<float*>(data), step, inv, ref + ch, chCount, sx, sy, rowPitch, type);
    countLaunch();
    CC_TRY_CUDA(cudaGetLastError(), "quantizeDifferenceToSymbols2D");
    return CC_OK;
}

int cc_quantize_difference_to_symbols_roundtrip_2d(uint16_t* sym, float* data, float step, const uint8_t* ref,
                                                   uint32_t chCount, uint32_t ch, uint32_t sx, uint32_t sy,
                                                   uint32_t rowPitch, int type, void* stream) {
    if (!rowPitch) rowPitch = sx;
    if (!u64(sx) * sy) return CC_OK;
    const float inv = 1.0f / step;
    k_quantizeDifference2D<true><<<pixelGrid(u64(sx) * sy), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        sym, data, step, inv, ref + ch, chCount, sx, sy, rowPitch, type);
    countLaunch();
    CC_TRY_CUDA(cudaGetLastError(), "quantizeDifferenceToSymbolsRoundtrip2D");
    return CC_OK;
}

int cc_unquantize_difference_from_symbols_2d(float* data, const uint16_t* sym, float step, const uint8_t* ref,
                                             uint32_t chCount, uint32_t ch, uint32_t sx, uint32_t sy,
                                             uint32_t rowPitch, int type, void* stream) {
    if (!rowPitch) rowPitch = sx;
    if (!u64(sx) * sy) return CC_OK;
    k_unquantizeDifference2D<<<pixelGrid(u64(sx) * sy), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        data, sym, step, ref + ch, chCount, sx, sy, rowPitch, type);
    countLaunch();
    CC_TRY_CUDA(cudaGetLastError(), "unquantizeDifferenceFromSymbols2D");
    return CC_OK;
}

static int ycocg(uint8_t* dst, const uint8_t* src, int n, int channels, bool toYCoCg, void* stream, const char* what) {
    if (channels != 3 && channels != 4) { setError("%s: pixels have 3 or 4 bytes", what); return CC_ERR_INVALID_ARGUMENT; }
    if (n <= 0) return CC_OK;
    if (!dst || !src) { setError("%s: null argument", what); return CC_ERR_INVALID_ARGUMENT; }
    if (channels == 4 && ((reinterpret_cast<uintptr_t>(dst) | reinterpret_cast<uintptr_t>(src)) & 3)) {
        setError("%s: uchar4 pixels must be 4-byte aligned", what);
        return CC_ERR_INVALID_ARGUMENT;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const unsigned g = strideGrid(u32(n), 256);
    if (channels == 3) {
        if (toYCoCg) k_ycocg<3, true><<<g, 256, 0, st>>>(dst, src, u32(n));
        else k_ycocg<3, false><<<g, 256, 0, st>>>(dst, src, u32(n));
    } else {
        if (toYCoCg) k_ycocg<4, true><<<g, 256, 0, st>>>(dst, src, u32(n));
        else k_ycocg<4, false><<<g, 256, 0, st>>>(dst, src, u32(n));
    }
    countLaunch();
    CC_TRY_CUDA(cudaGetLastError(), what);
    return CC_OK;
}

int cc_convert_rgb_to_ycocg(uint8_t* dst, const uint8_t* src, int n, int channels, void* stream) {
    return ycocg(dst, src, n, channels, true, stream, "convertRGBtoYCoCg");
}
int cc_convert_ycocg_to_rgb(uint8_t* dst, const uint8_t* src, int n, int channels, void* stream) {
    return ycocg(dst, src, n, channels, false, stream, "convertYCoCgtoRGB");
}

int cc_get_lsb(const int16_t* data, uint32_t* bits, uint32_t n, void* stream) {
    return lsbLaunch(kLsbGet, const_cast<int16_t*>(data), bits, n, 0, static_cast<cudaStream_t>(stream), "getLSB");
}
int cc_remove_lsb(int16_t* data, uint32_t* bits, uint32_t n, int16_t shift, void* stream) {
    return lsbLaunch(kLsbRemove, data, bits, n, shift, static_cast<cudaStream_t>(stream), "removeLSB");
}
int cc_append_lsb(int16_t* data, const uint32_t* bits, uint32_t n, int16_t shift, void* stream) {
    return lsbLaunch(kLsbAppend, data, const_cast<uint32_t*>(bits), n, shift, static_cast<cudaStream_t>(stream),
                     "appendLSB");
}
int cc_shift_elems(int16_t* data, uint32_t n, int16_t shift, void* stream) {
    if (!n) return CC_OK;
    if (!data) { setError("shiftElems: null argument"); return CC_ERR_INVALID_ARGUMENT; }
    k_shiftElems<<<strideGrid(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(data, n, shift);
    countLaunch();
    CC_TRY_CUDA(cudaGetLastError(), "shiftElems");
    return CC_OK;
}

int cc_compress_image_one_level(cc_instance* I, uint8_t* image, uint32_t sx, uint32_t sy, uint32_t chTotal,
                                uint32_t chProc, const uint8_t* lowpassRef, float step, uint32_t* words,
                                uint64_t capacity, uint32_t* bitSize) {
    if (!bitSize) { setError("compressImageOneLevel: bad argument"); return CC_ERR_INVALID_ARGUMENT; }
    cc_image im{image, lowpassRef, words, capacity, 0, step};
    const int rc = compressImages(I, &im, 1, sx, sy, chTotal, chProc, true, "compressImageOneLevel");
    if (rc == CC_OK) *bitSize = im.bit_size;
    return rc;
}

int cc_decompress_image_one_level(cc_instance* I, uint8_t* image, uint32_t sx, uint32_t sy, uint32_t chTotal,
                                  uint32_t chProc, const uint8_t* lowpassRef, float step, const uint32_t* words,
                                  uint32_t bitSize) {
    cc_image im{image, lowpassRef, const_cast<uint32_t*>(words), 0, bitSize, step};
    return decompressImages(I, &im, 1, sx, sy, chTotal, chProc, "decompressImageOneLevel");
}

int cc_compress_images_one_level(cc_instance* I, cc_image* images, uint32_t count, uint32_t sx, uint32_t sy,
                                 uint32_t chTotal, uint32_t chProc) {
    return compressImages(I, images, count, sx, sy, chTotal, chProc, false, "compressImagesOneLevel");
}

int cc_decompress_images_one_level(cc_instance* I, const cc_image* images, uint32_t count, uint32_t sx, uint32_t sy,
                                   uint32_t chTotal, uint32_t chProc) {
    return decompressImages(I, images, count, sx, sy, chTotal, chProc, "decompressImagesOneLevel");
}

// ---- one heightfield level (CompressHeightfield.cpp:82-216) ----
// Stream: the least significant bits of (LL + shift), ceil(n/32) words, then
// one encodeRLHuff call over the 3 symbolized highpass bands (x + 2y order).
// The caller's lowpass receives (LL + shift) without its least significant
// bit (floor division by 2); decompress restores it in place and then
// reconstructs the image.
int cc_compress_heightfield_one_level(cc_instance* I, const int16_t* image, uint32_t sx, uint32_t sy,
                                      int16_t* lowpass, int16_t shift, uint32_t* words, uint64_t capacity,
                                      uint32_t* bitSize) {
    const char* what = "compressHeightfieldOneLevel";
    if (!I || !image || !lowpass || !words || !bitSize) { setError("%s: bad argument", what); return CC_ERR_INVALID_ARGUMENT; }
    if (!imageArgsOk(sx, sy, 1, 1, what)) return CC_ERR_INVALID_ARGUMENT;
    if (I->symBytes != 2) { setError("%s: needs a 16-bit-symbol instance", what); return CC_ERR_INVALID_ARGUMENT; }
    const u32 hx = sx / 2, hy = sy / 2;
    const u64 n = u64(hx) * hy, bitsWords = ceilDiv(n, 32);
    if (I->streamCountMax < 3 || I->elemCountPerStreamMax < n) {
        setError("%s: instance needs >= 3 streams of >= %llu symbols", what, (unsigned long long)n);
        return CC_ERR_CAPACITY;
    }
    if (capacity < bitsWords) { setError("%s: needs more than %llu words", what, (unsigned long long)capacity); return CC_ERR_CAPACITY; }
    DeviceGuard deviceGuard(I->device);
    cudaStream_t st = I->stream;
    const u64 pixels = u64(sx) * sy;
    Bump b{nullptr};
    b.take<i16>(pixels);
    b.take<i16>(pixels);
    b.take<u16>(3 * n + 64);
    int rc = ensurePipelineWork(I, b.off + 1024);
    if (rc) return rc;
    Bump w{I->pipeWork};
    i16* dwt0 = w.take<i16>(pixels);
    i16* dwt1 = w.take<i16>(pixels);
    u16* syms = w.take<u16>(3 * n + 64);
    if ((rc = cc_dwt_int_forward(dwt1, dwt0, image, int(sx), int(sy), 1, 0, 0, 0, 0, st))) return rc;
    CC_TRY_CUDA(cudaMemcpy2DAsync(lowpass, hx * sizeof(i16), dwt1, sx * sizeof(i16), hx * sizeof(i16), hy,
                                  cudaMemcpyDeviceToDevice, st), "copy lowpass");
    if ((rc = cc_remove_lsb(lowpass, words, u32(n), shift, st))) return rc;
    std::vector<EncStream> es;
    for (u32 k = 1; k < 4; ++k) {
        const u64 off = u64(k % 2) * hx + u64(k / 2) * hy * sx;
        if ((rc = cc_symbolize(syms + (k - 1) * n, dwt1 + off, hx, hy, 1, sx, 0, st))) return rc;
        es.push_back(EncStream{syms + (k - 1) * n, u32(n), 0, 0, 3, KIND_RLHUFF});
    }
    u64 at = 0;
    if ((rc = encodeGroups(I, es, {EncGroup{0, 3}}, words + bitsWords, capacity - bitsWords, &at))) return rc;
    CC_TRY_CUDA(cudaStreamSynchronize(st), what);
    if ((bitsWords + at) * 32 > 0xffffffffull) { setError("%s: stream exceeds 2^32 bits", what); return CC_ERR_CAPACITY; }
    *bitSize = u32((bitsWords + at) * 32);
    return CC_OK;
}

int cc_decompress_heightfield_one_level(cc_instance* I, int16_t* image, uint32_t sx, uint32_t sy, int16_t* lowpass,
                                        int16_t shift, const uint32_t* words, uint32_t bitSize) {
    const char* what = "decompressHeightfieldOneLevel";
    if (!I || !image || !lowpass || !words) { setError("%s: bad argument", what); return CC_ERR_INVALID_ARGUMENT; }
    if (!imageArgsOk(sx, sy, 1, 1, what)) return CC_ERR_INVALID_ARGUMENT;
    if (I->symBytes != 2) { setError("%s: needs a 16-bit-symbol instance", what); return CC_ERR_INVALID_ARGUMENT; }
    const u32 hx = sx / 2, hy = sy / 2;
    const u64 n = u64(hx) * hy, bitsWords = ceilDiv(n, 32);
    if (I->streamCountMax < 3 || I->elemCountPerStreamMax < n) {
        setError("%s: instance needs >= 3 streams of >= %llu symbols", what, (unsigned long long)n);
        return CC_ERR_CAPACITY;
    }
    if (u64(bitSize) < bitsWords * 32) { setError("%s: stream shorter than the lowpass bits", what); return CC_ERR_CORRUPT_STREAM; }
    DeviceGuard deviceGuard(I->device);
    cudaStream_t st = I->stream;
    const u64 pixels = u64(sx) * sy;
    Bump b{nullptr};
    b.take<i16>(pixels);
    b.take<i16>(pixels);
    b.take<u16>(3 * n + 64);
    int rc = ensurePipelineWork(I, b.off + 1024);
    if (rc) return rc;
    Bump w{I->pipeWork};
    i16* dwt0 = w.take<i16>(pixels);
    i16* dwt1 = w.take<i16>(pixels);
    u16* syms = w.take<u16>(3 * n + 64);
    std::vector<u32> host;
    if ((rc = downloadWords(I, words, ceilDiv(bitSize, 32), host, what))) return rc;
    if ((rc = cc_append_lsb(lowpass, words, u32(n), shift, st))) return rc;
    CC_TRY_CUDA(cudaMemcpy2DAsync(dwt1, sx * sizeof(i16), lowpass, hx * sizeof(i16), hx * sizeof(i16), hy,
                                  cudaMemcpyDeviceToDevice, st), "place lowpass");
    const u32* hw = host.data();
    u32 pos = u32(bitsWords * 32);
    void* outs[3] = {syms, syms + n, syms + 2 * n};
    if ((rc = decodeDevice(I, KIND_RLHUFF, &hw, &bitSize, &pos, 1, nullptr, outs, 3, u32(n)))) return rc;
    for (u32 k = 1; k < 4; ++k) {
        const u64 off = u64(k % 2) * hx + u64(k / 2) * hy * sx;
        if ((rc = cc_unsymbolize(dwt1 + off, syms + (k - 1) * n, hx, hy, 1, sx, 0, st))) return rc;
    }
    if ((rc = cc_dwt_int_inverse(image, dwt0, dwt1, int(sx), int(sy), 1, 0, 0, 0, 0, st))) return rc;
    CC_TRY_CUDA(cudaStreamSynchronize(st), what);
    return cc_decode_status(I);
}

}  // extern "C"
