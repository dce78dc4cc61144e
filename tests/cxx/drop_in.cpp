// A program written against the reference's C++ API (include/cudaCompress/*.h)
// only, built and linked against this library: the drop-in check.  It codes a
// volume the way the reference's examples do (one DWT level, quantized
// bands, encodeRLHuff / encodeHuff into a BitStream, decode, inverse from
// symbols), runs the image-side util helpers and the CUDA-event timers, and
// prints DROPIN OK when every check holds.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include <cuda_runtime.h>

#include <cudaCompress/BitStream.h>
#include <cudaCompress/Encode.h>
#include <cudaCompress/Instance.h>
#include <cudaCompress/Timing.h>
#include <cudaCompress/util/Bits.h>
#include <cudaCompress/util/CudaTimer.h>
#include <cudaCompress/util/DWT.h>
#include <cudaCompress/util/Quantize.h>
#include <cudaCompress/util/YCoCg.h>

using namespace cudaCompress;

static int failures = 0;
#define CHECK(cond)                                                      \
    do {                                                                 \
        if (!(cond)) {                                                   \
            std::printf("FAILED %s:%d: %s\n", __FILE__, __LINE__, #cond); \
            ++failures;                                                  \
        }                                                                \
    } while (0)

template <class T>
static T* dalloc(size_t n) {
    T* p = nullptr;
    cudaMalloc(&p, n * sizeof(T) + 256);
    cudaMemset(p, 0, n * sizeof(T) + 256);
    return p;
}

static void volumeRoundTrip() {
    const int n = 32, h = n / 2, nb = h * h * h;
    const float step = 0.02f;
    std::vector<float> host(n * n * n);
    for (int z = 0; z < n; ++z)
        for (int y = 0; y < n; ++y)
            for (int x = 0; x < n; ++x)
                host[(z * n + y) * n + x] = std::sin(0.3f * x) * std::cos(0.2f * y) + 0.1f * std::sin(0.5f * z + x);
    float* dVol = dalloc<float>(host.size());
    float* dDwt = dalloc<float>(host.size());
    float* dBuf1 = dalloc<float>(host.size());
    float* dBuf2 = dalloc<float>(host.size());
    cudaMemcpy(dVol, host.data(), host.size() * 4, cudaMemcpyHostToDevice);

    Instance* inst = createInstance(0, 7, nb, 0, 0);
    CHECK(inst != nullptr);
    CHECK(getInstanceCodingBlockSize(inst) == 128);
    CHECK(getInstanceLog2HuffmanDistinctSymbolCountMax(inst) == 14);
    CHECK(getInstanceStreamCountMax(inst) == 7);

    util::dwtFloat3DForward(dDwt, dBuf2, dBuf1, dVol, n, n, n);
    std::vector<Symbol16*> bands(7);
    for (int b = 0; b < 7; ++b) bands[b] = dalloc<Symbol16>(nb);
    Symbol16* lp = dalloc<Symbol16>(nb);
    for (int b = 1; b < 8; ++b) {
        const int off = (b & 1) * h + ((b >> 1) & 1) * h * n + (b >> 2) * h * n * n;
        util::quantizeToSymbols(bands[b - 1], dDwt + off, h, h, h, step, n, n * n);
    }
    util::quantizeToSymbols(lp, dDwt, h, h, h, step, n, n * n);

    std::vector<uint> words;
    BitStream bs(&words);
    CHECK(encodeHuff(inst, bs, &lp, 1, nb));
    CHECK(encodeRLHuff(inst, bs, bands.data(), 7, nb));
    CHECK(!words.empty());

    // decode into fresh (zeroed) buffers
    Symbol16* lpOut = dalloc<Symbol16>(nb);
    std::vector<Symbol16*> out(7);
    for (int b = 0; b < 7; ++b) out[b] = dalloc<Symbol16>(nb);
    BitStreamReadOnly rd(words.data(), uint(words.size() * 32));
    CHECK(decodeHuff(inst, rd, &lpOut, 1, nb));
    CHECK(decodeRLHuff(inst, rd, out.data(), 7, nb));
    cudaDeviceSynchronize();

    float* dLp = dalloc<float>(host.size());
    util::unquantizeFromSymbols(dLp, lpOut, h, h, h, step, n, n * n);
    Symbol16** dBands = dalloc<Symbol16*>(7);
    cudaMemcpy(dBands, out.data(), 7 * sizeof(Symbol16*), cudaMemcpyHostToDevice);
    float* dRec = dalloc<float>(host.size());
    util::dwtFloat3DInverseFromSymbols(dRec, dBuf2, dBuf1, dLp, dBands, step, n, n, n);
    std::vector<float> rec(host.size());
    cudaMemcpy(rec.data(), dRec, rec.size() * 4, cudaMemcpyDeviceToHost);
    double maxErr = 0;
    for (size_t i = 0; i < rec.size(); ++i) maxErr = std::fmax(maxErr, std::fabs(double(rec[i]) - host[i]));
    CHECK(maxErr < 8 * step);

    // the per-stream overload of the same call writes the same segments: the
    // single stream's words are bit stream 1's followed by bit stream 2's
    // (an RLHuff segment starts word aligned)
    std::vector<uint> w1, w2, wAll;
    BitStream b1(&w1), b2(&w2), bAll(&wAll);
    BitStream* ptrs[7] = {&b1, &b1, &b1, &b1, &b2, &b2, &b2};
    CHECK(encodeRLHuff(inst, ptrs, bands.data(), 7, nb));
    CHECK(encodeRLHuff(inst, bAll, bands.data(), 7, nb));
    std::vector<uint> joined(w1);
    joined.insert(joined.end(), w2.begin(), w2.end());
    CHECK(!w1.empty() && !w2.empty() && joined == wAll);
    destroyInstance(inst);
}

static void imageHelpers() {
    const int nx = 64, ny = 48, px = nx * ny;
    std::vector<unsigned char> rgb(3 * px);
    for (int i = 0; i < 3 * px; ++i) rgb[i] = (unsigned char)((i * 37 + (i / 3) % 11) & 255);
    uchar3* dRgb = dalloc<uchar3>(px);
    cudaMemcpy(dRgb, rgb.data(), rgb.size(), cudaMemcpyHostToDevice);
    util::convertRGBtoYCoCg(dRgb, dRgb, px);
    util::convertYCoCgtoRGB(dRgb, dRgb, px);
    std::vector<unsigned char> back(rgb.size());
    cudaMemcpy(back.data(), dRgb, back.size(), cudaMemcpyDeviceToHost);
    int worst = 0;
    for (size_t i = 0; i < back.size(); ++i) worst = std::max(worst, std::abs(int(back[i]) - int(rgb[i])));
    CHECK(worst <= 2);

    // byte DWT forward of channel 1, inverse into channel 1: within one grey level
    byte* dImg = reinterpret_cast<byte*>(dRgb);
    cudaMemcpy(dImg, rgb.data(), rgb.size(), cudaMemcpyHostToDevice);
    float* dDwt = dalloc<float>(px);
    float* dBuf = dalloc<float>(px);
    util::dwtFloat2DForwardFromByte(dDwt, dBuf, dImg + 1, nx, ny, 3);
    util::dwtFloat2DInverseToByte(dImg + 1, dBuf, dDwt, nx, ny, 3);
    cudaMemcpy(back.data(), dImg, back.size(), cudaMemcpyDeviceToHost);
    worst = 0;
    for (int i = 0; i < px; ++i) {
        worst = std::max(worst, std::abs(int(back[3 * i + 1]) - int(rgb[3 * i + 1])));
        CHECK(back[3 * i] == rgb[3 * i] && back[3 * i + 2] == rgb[3 * i + 2]);
    }
    CHECK(worst <= 1);

    // lowpass only equals the LL band of the full transform
    float* dLL = dalloc<float>(px / 4);
    util::dwtFloat2DForwardLowpassOnlyFromByte(dLL, dBuf, dImg, nx, ny, 3);
    util::dwtFloat2DForwardFromByte(dDwt, dBuf, dImg, nx, ny, 3);
    std::vector<float> ll(px / 4), full(px);
    cudaMemcpy(ll.data(), dLL, ll.size() * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(full.data(), dDwt, full.size() * 4, cudaMemcpyDeviceToHost);
    for (int y = 0; y < ny / 2; ++y)
        for (int x = 0; x < nx / 2; ++x) CHECK(ll[y * (nx / 2) + x] == full[y * nx + x]);

    // LSB planes: remove then append restores the data (with opposite shifts)
    const uint n = 4096;
    std::vector<short> v(n);
    for (uint i = 0; i < n; ++i) v[i] = short(int(i * 7919) % 20001 - 10000);
    short* dV = dalloc<short>(n);
    uint* dBits = dalloc<uint>(n / 32);
    cudaMemcpy(dV, v.data(), n * 2, cudaMemcpyHostToDevice);
    CHECK(util::removeLSB(dV, dBits, n, 3));
    CHECK(util::appendLSB(dV, dBits, n, -3));
    std::vector<short> w(n);
    cudaMemcpy(w.data(), dV, n * 2, cudaMemcpyDeviceToHost);
    CHECK(w == v);
}

static void timers() {
    util::CudaTimerResources res(true);
    {
        util::CudaScopedTimer timer(res);
        timer("first");
        float* d = dalloc<float>(1 << 20);
        timer("second");
        cudaMemset(d, 1, 4 << 20);
        timer();
    }
    std::vector<std::string> names;
    std::vector<float> times;
    res.getAccumulatedTimes(names, times, true);
    CHECK(names.size() == 2 && names[0] == "first" && names[1] == "second");
    for (float t : times) CHECK(t >= 0.0f);
    util::CudaTimerResources off;
    off.record("x");
    CHECK(off.getAccumulatedTimes(true).empty());
}

int main() {
    int devices = 0;
    if (cudaGetDeviceCount(&devices) != cudaSuccess || devices == 0) {
        std::printf("no CUDA device\n");
        return 2;
    }
    volumeRoundTrip();
    imageHelpers();
    timers();
    if (failures) {
        std::printf("%d check(s) failed\n", failures);
        return 1;
    }
    std::printf("DROPIN OK\n");
    return 0;
}
