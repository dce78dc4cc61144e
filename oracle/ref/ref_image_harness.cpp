// Test-infrastructure harness: the reference's own example image and
// heightfield codecs (examples/CompressImage.cpp, CompressHeightfield.cpp,
// compiled unmodified from the reference tree by oracle/ref/Makefile) behind a
// C ABI, so that tests/golden/make_golden.py can record their bit streams and
// reconstructions as fixtures.  Never shipped.
#include <cstdint>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

#include "CompressHeightfield.h"
#include "CompressImage.h"

namespace {

// GPUResources sized by the codec's own estimate plus slack: the decoders pad
// every stream to 32 coding blocks, and runLengthDecode asks for per-stream
// capacity of 32 coding blocks of 128 symbols.
GPUResources::Config padded(GPUResources::Config cfg) {
    cfg.bufferSize += size_t(64) << 20;
    if (cfg.elemCountPerBlockMax < 32u * 128u) cfg.elemCountPerBlockMax = 32u * 128u;
    return cfg;
}

struct ImageSession {
    GPUResources shared;
    CompressImageResources res;
    bool ok = false;
    ImageSession(uint32_t nx, uint32_t ny, uint32_t channels, uint32_t images) {
        ok = shared.create(padded(CompressImageResources::getRequiredResources(nx, ny, channels, images))) &&
             res.create(shared.getConfig());
    }
    ~ImageSession() {
        cudaDeviceSynchronize();
        res.destroy();
        shared.destroy();
    }
};

struct HeightfieldSession {
    GPUResources shared;
    CompressHeightfieldResources res;
    bool ok = false;
    HeightfieldSession(uint32_t nx, uint32_t ny) {
        ok = shared.create(padded(CompressHeightfieldResources::getRequiredResources(nx, ny))) &&
             res.create(shared.getConfig());
    }
    ~HeightfieldSession() {
        cudaDeviceSynchronize();
        res.destroy();
        shared.destroy();
    }
};

}  // namespace

extern "C" {

// compressImagesOneLevel over `count` device images (each overwritten with its
// reconstruction); image i's words go to words + offsets[i], offsets[count]
// the total.
int ref_images_compress(uint8_t* const* dImages, const uint8_t* const* dRefs, const float* q, uint32_t count,
                        uint32_t nx, uint32_t ny, uint32_t chTotal, uint32_t chProc, uint32_t* words, uint32_t cap,
                        uint32_t* offsets) {
    ImageSession s(nx, ny, chProc, count);
    if (!s.ok) return -1;
    std::vector<ImageV> images(count);
    for (uint32_t i = 0; i < count; ++i) {
        images[i].dpImage = dImages[i];
        images[i].dpLowpassReference = const_cast<uint8_t*>(dRefs[i]);
        images[i].quantizationStep = q[i];
    }
    const bool ok = count == 1 ? compressImageOneLevel(s.shared, s.res, dImages[0], nx, ny, chTotal, chProc, dRefs[0],
                                                       images[0].highpassBitStream, q[0])
                               : compressImagesOneLevel(s.shared, s.res, images, nx, ny, chTotal, chProc);
    cudaDeviceSynchronize();
    if (!ok) return -2;
    uint32_t at = 0;
    for (uint32_t i = 0; i < count; ++i) {
        offsets[i] = at;
        const size_t n = images[i].highpassBitStream.size();
        if (at + n > cap) return -3;
        std::memcpy(words + at, images[i].highpassBitStream.data(), n * sizeof(uint32_t));
        at += uint32_t(n);
    }
    offsets[count] = at;
    return 0;
}

// decompressImageOneLevel (count 1) / decompressImagesOneLevel: image i's
// stream is words + offsets[i] .. offsets[i + 1].
int ref_images_decompress(uint8_t* const* dImages, const uint8_t* const* dRefs, const float* q, uint32_t count,
                          uint32_t nx, uint32_t ny, uint32_t chTotal, uint32_t chProc, const uint32_t* words,
                          const uint32_t* offsets) {
    ImageSession s(nx, ny, chProc, count);
    if (!s.ok) return -1;
    std::vector<ImageV> images(count);
    for (uint32_t i = 0; i < count; ++i) {
        images[i].dpImage = dImages[i];
        images[i].dpLowpassReference = const_cast<uint8_t*>(dRefs[i]);
        images[i].quantizationStep = q[i];
        images[i].highpassBitStream.assign(words + offsets[i], words + offsets[i + 1]);
    }
    if (count == 1)
        decompressImageOneLevel(s.shared, s.res, dImages[0], nx, ny, chTotal, chProc, dRefs[0],
                                images[0].highpassBitStream, q[0]);
    else
        decompressImagesOneLevel(s.shared, s.res, images, nx, ny, chTotal, chProc);
    cudaDeviceSynchronize();
    return 0;
}

int ref_get_lowpass_image(const uint8_t* dImage, uint32_t nx, uint32_t ny, uint32_t chTotal, uint32_t chProc,
                          uint8_t* dLowpass) {
    ImageSession s(nx, ny, chProc, 1);
    if (!s.ok) return -1;
    getLowpassImage(s.shared, s.res, dImage, nx, ny, chTotal, chProc, dLowpass);
    cudaDeviceSynchronize();
    return 0;
}

int ref_heightfield_compress_one_level(const short* dImage, uint32_t nx, uint32_t ny, short* dLowpass, short shift,
                                       uint32_t* words, uint32_t cap, uint32_t* nWords) {
    HeightfieldSession s(nx, ny);
    if (!s.ok) return -1;
    std::vector<uint> bits;
    const bool ok = compressHeightfieldOneLevel(s.shared, s.res, dImage, nx, ny, dLowpass, shift, bits);
    cudaDeviceSynchronize();
    if (!ok) return -2;
    if (bits.size() > cap) return -3;
    std::memcpy(words, bits.data(), bits.size() * sizeof(uint32_t));
    *nWords = uint32_t(bits.size());
    return 0;
}

int ref_heightfield_decompress_one_level(short* dImage, uint32_t nx, uint32_t ny, short* dLowpass, short shift,
                                         const uint32_t* words, uint32_t nWords) {
    HeightfieldSession s(nx, ny);
    if (!s.ok) return -1;
    std::vector<uint> bits(words, words + nWords);
    decompressHeightfieldOneLevel(s.shared, s.res, dImage, nx, ny, dLowpass, shift, bits);
    cudaDeviceSynchronize();
    return 0;
}

int ref_get_lowpass_heightfield(const short* dImage, uint32_t nx, uint32_t ny, short* dLowpass, short shift) {
    HeightfieldSession s(nx, ny);
    if (!s.ok) return -1;
    getLowpassHeightfield(s.shared, s.res, dImage, nx, ny, dLowpass, shift);
    cudaDeviceSynchronize();
    return 0;
}

}  // extern "C"
