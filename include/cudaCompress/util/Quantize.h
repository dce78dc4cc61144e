// util/Quantize.h - quantization to/from symbols (drop-in for the
// reference's include/cudaCompress/util/Quantize.h:24-65).
// Like the reference, these launch on the default stream.
#ifndef CUDACOMPRESS_B200_QUANTIZE_H
#define CUDACOMPRESS_B200_QUANTIZE_H

#include <cudaCompress/global.h>

#include <cuda_runtime.h>

namespace cudaCompress {

class Instance;

namespace util {

enum EQuantizeType {
    QUANTIZE_DEADZONE = 0,  // midtread quantizer with a zero bin twice as wide
    QUANTIZE_UNIFORM,       // plain midtread quantizer
    QUANTIZE_COUNT
};

// float <-> one channel of an interleaved byte image (quantization step 1,
// shifted by 128 to be unsigned)
CUCOMP_DLL void floatToByte2D(byte* dpQuant, uint channelCount, uint channel, const float* dpData, uint sizeX, uint sizeY, uint rowPitchSrc = 0);
CUCOMP_DLL void byteToFloat2D(float* dpData, const byte* dpQuant, uint channelCount, uint channel, uint sizeX, uint sizeY, uint rowPitchDst = 0);

// signed shorts <-> symbols (>= 0 -> even, < 0 -> odd)
CUCOMP_DLL void symbolize(ushort* dpSymbols, const short* dpData, uint sizeX, uint sizeY, uint sizeZ, uint rowPitchSrc = 0, uint slicePitchSrc = 0);
CUCOMP_DLL void unsymbolize(short* dpData, const ushort* dpSymbols, uint sizeX, uint sizeY, uint sizeZ, uint rowPitchDst = 0, uint slicePitchDst = 0);

// floats <-> symbols
CUCOMP_DLL void quantizeToSymbols(ushort* dpSymbols, const float* dpData, uint sizeX, uint sizeY, uint sizeZ, float quantizationStep, uint rowPitchSrc = 0, uint slicePitchSrc = 0, EQuantizeType quantType = QUANTIZE_DEADZONE);
CUCOMP_DLL void quantizeToSymbolsRoundtrip(ushort* dpSymbols, float* dpData, uint sizeX, uint sizeY, uint sizeZ, float quantizationStep, uint rowPitchSrc = 0, uint slicePitchSrc = 0, EQuantizeType quantType = QUANTIZE_DEADZONE);
CUCOMP_DLL void unquantizeFromSymbols(float* dpData, const ushort* dpSymbols, uint sizeX, uint sizeY, uint sizeZ, float quantizationStep, uint rowPitchDst = 0, uint slicePitchDst = 0, EQuantizeType quantType = QUANTIZE_DEADZONE);
CUCOMP_DLL void quantizeToSymbols(uint* dpSymbols, const float* dpData, uint sizeX, uint sizeY, uint sizeZ, float quantizationStep, uint rowPitchSrc = 0, uint slicePitchSrc = 0, EQuantizeType quantType = QUANTIZE_DEADZONE);
CUCOMP_DLL void quantizeToSymbolsRoundtrip(uint* dpSymbols, float* dpData, uint sizeX, uint sizeY, uint sizeZ, float quantizationStep, uint rowPitchSrc = 0, uint slicePitchSrc = 0, EQuantizeType quantType = QUANTIZE_DEADZONE);
CUCOMP_DLL void unquantizeFromSymbols(float* dpData, const uint* dpSymbols, uint sizeX, uint sizeY, uint sizeZ, float quantizationStep, uint rowPitchDst = 0, uint slicePitchDst = 0, EQuantizeType quantType = QUANTIZE_DEADZONE);

// 2D convenience forms
CUCOMP_DLL void quantizeToSymbols2D(ushort* dpSymbols, const float* dpData, uint sizeX, uint sizeY, float quantizationStep, uint rowPitchSrc = 0, EQuantizeType quantType = QUANTIZE_DEADZONE);
CUCOMP_DLL void quantizeToSymbolsRoundtrip2D(ushort* dpSymbols, float* dpData, uint sizeX, uint sizeY, float quantizationStep, uint rowPitchSrc = 0, EQuantizeType quantType = QUANTIZE_DEADZONE);
CUCOMP_DLL void unquantizeFromSymbols2D(float* dpData, const ushort* dpSymbols, uint sizeX, uint sizeY, float quantizationStep, uint rowPitchDst = 0, EQuantizeType quantType = QUANTIZE_DEADZONE);
CUCOMP_DLL void quantizeToSymbols2D(uint* dpSymbols, const float* dpData, uint sizeX, uint sizeY, float quantizationStep, uint rowPitchSrc = 0, EQuantizeType quantType = QUANTIZE_DEADZONE);
CUCOMP_DLL void quantizeToSymbolsRoundtrip2D(uint* dpSymbols, float* dpData, uint sizeX, uint sizeY, float quantizationStep, uint rowPitchSrc = 0, EQuantizeType quantType = QUANTIZE_DEADZONE);
CUCOMP_DLL void unquantizeFromSymbols2D(float* dpData, const uint* dpSymbols, uint sizeX, uint sizeY, float quantizationStep, uint rowPitchDst = 0, EQuantizeType quantType = QUANTIZE_DEADZONE);

// floats <-> signed shorts
CUCOMP_DLL void quantizeToShort(short* dpQuant, const float* dpData, uint sizeX, uint sizeY, uint sizeZ, float quantizationStep, uint rowPitchSrc = 0, uint slicePitchSrc = 0, EQuantizeType quantType = QUANTIZE_DEADZONE);
CUCOMP_DLL void unquantizeFromShort(float* dpData, const short* dpQuant, uint sizeX, uint sizeY, uint sizeZ, float quantizationStep, uint rowPitchDst = 0, uint slicePitchDst = 0, EQuantizeType quantType = QUANTIZE_DEADZONE);

// float minus a byte reference channel (b - 128), quantized to symbols; the
// round trip writes back reference + dequantized symbol
CUCOMP_DLL void quantizeDifferenceToSymbols2D(ushort* dpSymbols, const float* dpData, float quantizationStep, const byte* dpReference, uint channelCount, uint channel, uint sizeX, uint sizeY, uint rowPitchSrc = 0, EQuantizeType quantType = QUANTIZE_DEADZONE);
CUCOMP_DLL void quantizeDifferenceToSymbolsRoundtrip2D(ushort* dpSymbols, float* dpData, float quantizationStep, const byte* dpReference, uint channelCount, uint channel, uint sizeX, uint sizeY, uint rowPitchSrc = 0, EQuantizeType quantType = QUANTIZE_DEADZONE);
CUCOMP_DLL void unquantizeDifferenceFromSymbols2D(float* dpData, const ushort* dpSymbols, float quantizationStep, const byte* dpReference, uint channelCount, uint channel, uint sizeX, uint sizeY, uint rowPitchDst = 0, EQuantizeType quantType = QUANTIZE_DEADZONE, cudaStream_t stream = 0);

// max |x| over elemCount floats, written to device memory
CUCOMP_DLL void getMaxAbs(Instance* pInstance, const float* dpImage, uint elemCount, float* dpValMax);

}
}

#endif
