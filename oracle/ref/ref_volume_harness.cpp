// Test-infrastructure harness: the reference's own example volume codec
// (examples/CompressVolume.cpp, compiled unmodified from the reference tree
// by oracle/ref/Makefile) behind a C ABI, so that tests/golden/make_golden.py
// can record its bit streams and reconstructions as fixtures.  Never shipped.
#include <chrono>
#include <cstdint>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

#include "CompressVolume.h"

namespace {

struct Session {
    GPUResources shared;
    CompressVolumeResources res;
    bool ok = false;
    Session(uint32_t nx, uint32_t ny, uint32_t nz, uint32_t channels) {
        GPUResources::Config cfg = CompressVolumeResources::getRequiredResources(nx, ny, nz, channels);
        // the decoders pad every band to 32 coding blocks, which the estimate
        // leaves out; small volumes need the slack
        cfg.bufferSize += size_t(64) << 20;
        // runLengthDecode (RunLength.cu:261) asks for per-stream capacity of
        // the stride padded to whole groups of 32 coding blocks of 128 symbols
        cfg.elemCountPerBlockMax = (cfg.elemCountPerBlockMax + 32u * 128u - 1) / (32u * 128u) * (32u * 128u);
        ok = shared.create(cfg) && res.create(shared.getConfig());
    }
    ~Session() {
        cudaDeviceSynchronize();
        res.destroy();
        shared.destroy();
    }
};

}  // namespace

extern "C" {

// compressVolumeFloat (quantFirst 0) or compressVolumeFloatQuantFirst
// (quantFirst 1) of one device volume; the stream's words go to `words`.
int ref_volume_compress(const float* dVol, uint32_t nx, uint32_t ny, uint32_t nz, uint32_t levels, float q,
                        int rleOnlyLevel0, int quantFirst, uint32_t* words, uint32_t cap, uint32_t* nWords) {
    Session s(nx, ny, nz, 1);
    if (!s.ok) return -1;
    std::vector<uint> bits;
    bool ok = quantFirst
                  ? compressVolumeFloatQuantFirst(s.shared, s.res, dVol, nx, ny, nz, levels, bits, q, rleOnlyLevel0 != 0)
                  : compressVolumeFloat(s.shared, s.res, dVol, nx, ny, nz, levels, bits, q, rleOnlyLevel0 != 0);
    cudaDeviceSynchronize();
    if (!ok) return -2;
    if (bits.size() > cap) return -3;
    std::memcpy(words, bits.data(), bits.size() * sizeof(uint32_t));
    *nWords = uint32_t(bits.size());
    return 0;
}

int ref_volume_decompress(float* dOut, uint32_t nx, uint32_t ny, uint32_t nz, uint32_t levels, float q,
                          int rleOnlyLevel0, int quantFirst, const uint32_t* words, uint32_t nWords) {
    Session s(nx, ny, nz, 1);
    if (!s.ok) return -1;
    std::vector<uint> bits(words, words + nWords);
    if (quantFirst)
        decompressVolumeFloatQuantFirst(s.shared, s.res, dOut, nx, ny, nz, levels, bits, q, rleOnlyLevel0 != 0);
    else
        decompressVolumeFloat(s.shared, s.res, dOut, nx, ny, nz, levels, bits, q, rleOnlyLevel0 != 0);
    cudaDeviceSynchronize();
    return 0;
}

// decompressVolumeFloat(QuantFirst)MultiChannel: channel c's stream is
// words[c] (host, nWords[c] words), its step q[c], its output dOuts[c].
int ref_volume_decompress_multichannel(float* const* dOuts, const uint32_t* const* words, const uint32_t* nWords,
                                       const float* q, uint32_t channels, uint32_t nx, uint32_t ny, uint32_t nz,
                                       uint32_t levels, int rleOnlyLevel0, int quantFirst) {
    Session s(nx, ny, nz, channels);
    if (!s.ok) return -1;
    std::vector<VolumeChannel> ch(channels);
    for (uint32_t c = 0; c < channels; ++c) {
        ch[c].dpImage = dOuts[c];
        ch[c].pBits = words[c];
        ch[c].bitCount = nWords[c] * 32u;
        ch[c].quantizationStepLevel0 = q[c];
    }
    if (quantFirst)
        decompressVolumeFloatQuantFirstMultiChannel(s.shared, s.res, ch.data(), channels, nx, ny, nz, levels,
                                                    rleOnlyLevel0 != 0);
    else
        decompressVolumeFloatMultiChannel(s.shared, s.res, ch.data(), channels, nx, ny, nz, levels,
                                                    rleOnlyLevel0 != 0);
    cudaDeviceSynchronize();
    return 0;
}

// Timing of the reference's own codec on one device volume (baseline
// infrastructure, oracle/ref/time_ref_gpu.py): one session, one untimed call
// of each direction, then `reps` calls of compressVolumeFloat (device volume
// -> host bit stream, its own API) and of decompressVolumeFloat (host bit
// stream -> device volume), each followed by a device synchronize; msEnc /
// msDec get the mean wall time of one call.
int ref_volume_time(const float* dVol, float* dOut, uint32_t nx, uint32_t ny, uint32_t nz, uint32_t levels, float q,
                    uint32_t reps, double* msEnc, double* msDec, uint32_t* nWords) {
    Session s(nx, ny, nz, 1);
    if (!s.ok) return -1;
    using clk = std::chrono::steady_clock;
    std::vector<uint> bits;
    double enc = 0.0, dec = 0.0;
    for (uint32_t r = 0; r <= reps; ++r) {
        bits.clear();
        const auto t0 = clk::now();
        if (!compressVolumeFloat(s.shared, s.res, dVol, nx, ny, nz, levels, bits, q, false)) return -2;
        cudaDeviceSynchronize();
        const auto t1 = clk::now();
        decompressVolumeFloat(s.shared, s.res, dOut, nx, ny, nz, levels, bits, q, false);
        cudaDeviceSynchronize();
        const auto t2 = clk::now();
        if (r > 0) {
            enc += std::chrono::duration<double, std::milli>(t1 - t0).count();
            dec += std::chrono::duration<double, std::milli>(t2 - t1).count();
        }
    }
    *msEnc = reps ? enc / reps : 0.0;
    *msDec = reps ? dec / reps : 0.0;
    *nWords = uint32_t(bits.size());
    return cudaGetLastError() == cudaSuccess ? 0 : -4;
}

}  // extern "C"
