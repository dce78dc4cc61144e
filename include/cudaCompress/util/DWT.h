// util/DWT.h - one-level wavelet transforms on device arrays (drop-in for the
// reference's include/cudaCompress/util/DWT.h:21-157).
// All sizes even (>= 8); pitches in elements, 0 = tight; channel counts 1..4
// (interleaved channels, the pointer addressing the wanted channel).
#ifndef CUDACOMPRESS_B200_DWT_H
#define CUDACOMPRESS_B200_DWT_H

#include <cudaCompress/global.h>

#include <cuda_runtime.h>

namespace cudaCompress {
namespace util {

// CDF 9/7, float.  Results land in [L|H] halves along each axis.
CUCOMP_DLL void dwtFloat2DForward(float* dpDest, float* dpBuffer, const float* dpSource, int sizeX, int sizeY,
                                  int srcChannelCount = 1, int dstRowPitch = 0, int srcRowPitch = 0, cudaStream_t stream = 0);
CUCOMP_DLL void dwtFloat3DForward(float* dpDest, float* dpBuffer2, float* dpBuffer1, const float* dpSource, int sizeX,
                                  int sizeY, int sizeZ, int srcChannelCount = 1, int dstRowPitch = 0, int dstSlicePitch = 0,
                                  int srcRowPitch = 0, int srcSlicePitch = 0, cudaStream_t stream = 0);
CUCOMP_DLL void dwtFloat2DInverse(float* dpDest, float* dpBuffer, const float* dpSource, int sizeX, int sizeY,
                                  int dstChannelCount = 1, int dstRowPitch = 0, int srcRowPitch = 0, cudaStream_t stream = 0);
CUCOMP_DLL void dwtFloat3DInverse(float* dpDest, float* dpBuffer2, float* dpBuffer1, const float* dpSource, int sizeX,
                                  int sizeY, int sizeZ, int dstChannelCount = 1, int dstRowPitch = 0, int dstSlicePitch = 0,
                                  int srcRowPitch = 0, int srcSlicePitch = 0, cudaStream_t stream = 0);

// Inverse that dequantizes the highpass bands on the fly.  dppHighpass is a
// device array of 3 (2D) or 7 (3D) device pointers to the band symbols, band
// index x + 2y + 4z - 1.
CUCOMP_DLL void dwtFloat2DInverseFromSymbols(float* dpDest, float* dpBuffer, const float* dpLowpass,
                                             const ushort* const* dppHighpass, float quantStep, int sizeX, int sizeY,
                                             int dstChannelCount = 1, int dstRowPitch = 0, int lowpassRowPitch = 0,
                                             cudaStream_t stream = 0);
CUCOMP_DLL void dwtFloat3DInverseFromSymbols(float* dpDest, float* dpBuffer2, float* dpBuffer1, const float* dpLowpass,
                                             const ushort* const* dppHighpass, float quantStep, int sizeX, int sizeY,
                                             int sizeZ, int dstChannelCount = 1, int dstRowPitch = 0, int dstSlicePitch = 0,
                                             int lowpassRowPitch = 0, int lowpassSlicePitch = 0, cudaStream_t stream = 0);
CUCOMP_DLL void dwtFloat2DInverseFromSymbols(float* dpDest, float* dpBuffer, const float* dpLowpass,
                                             const uint* const* dppHighpass, float quantStep, int sizeX, int sizeY,
                                             int dstChannelCount = 1, int dstRowPitch = 0, int lowpassRowPitch = 0,
                                             cudaStream_t stream = 0);
CUCOMP_DLL void dwtFloat3DInverseFromSymbols(float* dpDest, float* dpBuffer2, float* dpBuffer1, const float* dpLowpass,
                                             const uint* const* dppHighpass, float quantStep, int sizeX, int sizeY,
                                             int sizeZ, int dstChannelCount = 1, int dstRowPitch = 0, int dstSlicePitch = 0,
                                             int lowpassRowPitch = 0, int lowpassSlicePitch = 0, cudaStream_t stream = 0);

// Byte variants: the forward reads one channel of a byte array with
// srcChannelCount interleaved channels (b -> b - 128), the inverses write one
// channel of one (clamp(v + 128.5, 0, 255)); the pointer addresses the channel.
CUCOMP_DLL void dwtFloat2DForwardFromByte(float* dpDest, float* dpBuffer, const byte* dpSource, int sizeX, int sizeY,
                                          int srcChannelCount = 1, int dstRowPitch = 0, int srcRowPitch = 0,
                                          cudaStream_t stream = 0);
CUCOMP_DLL void dwtFloat3DForwardFromByte(float* dpDest, float* dpBuffer2, float* dpBuffer1, const byte* dpSource,
                                          int sizeX, int sizeY, int sizeZ, int srcChannelCount = 1, int dstRowPitch = 0,
                                          int dstSlicePitch = 0, int srcRowPitch = 0, int srcSlicePitch = 0,
                                          cudaStream_t stream = 0);
CUCOMP_DLL void dwtFloat2DInverseToByte(byte* dpDest, float* dpBuffer, const float* dpSource, int sizeX, int sizeY,
                                        int dstChannelCount = 1, int dstRowPitch = 0, int srcRowPitch = 0,
                                        cudaStream_t stream = 0);
CUCOMP_DLL void dwtFloat3DInverseToByte(byte* dpDest, float* dpBuffer2, float* dpBuffer1, const float* dpSource,
                                        int sizeX, int sizeY, int sizeZ, int dstChannelCount = 1, int dstRowPitch = 0,
                                        int dstSlicePitch = 0, int srcRowPitch = 0, int srcSlicePitch = 0,
                                        cudaStream_t stream = 0);
CUCOMP_DLL void dwtFloat2DInverseFromSymbolsToByte(byte* dpDest, float* dpBuffer, const float* dpLowpass,
                                                   const ushort* const* dppHighpass, float quantStep, int sizeX,
                                                   int sizeY, int dstChannelCount = 1, int dstRowPitch = 0,
                                                   int lowpassRowPitch = 0, cudaStream_t stream = 0);
CUCOMP_DLL void dwtFloat3DInverseFromSymbolsToByte(byte* dpDest, float* dpBuffer2, float* dpBuffer1,
                                                   const float* dpLowpass, const ushort* const* dppHighpass,
                                                   float quantStep, int sizeX, int sizeY, int sizeZ,
                                                   int dstChannelCount = 1, int dstRowPitch = 0, int dstSlicePitch = 0,
                                                   int lowpassRowPitch = 0, int lowpassSlicePitch = 0,
                                                   cudaStream_t stream = 0);
// Only the lowpass (LL) band of one 2D level; dpBuffer is not used.
CUCOMP_DLL void dwtFloat2DForwardLowpassOnlyFromByte(float* dpDest, float* dpBuffer, const byte* dpSource, int sizeX,
                                                     int sizeY, int srcChannelCount = 1, int dstRowPitch = 0,
                                                     int srcRowPitch = 0, cudaStream_t stream = 0);

// CDF 5/3 integer lifting on shorts.
CUCOMP_DLL void dwtIntForward(short* dpDest, short* dpBuffer, const short* dpSource, int sizeX, int sizeY, int sizeZ,
                              int dstRowPitch = 0, int dstSlicePitch = 0, int srcRowPitch = 0, int srcSlicePitch = 0,
                              cudaStream_t stream = 0);
CUCOMP_DLL void dwtIntInverse(short* dpDest, short* dpBuffer, const short* dpSource, int sizeX, int sizeY, int sizeZ,
                              int dstRowPitch = 0, int dstSlicePitch = 0, int srcRowPitch = 0, int srcSlicePitch = 0,
                              cudaStream_t stream = 0);
// Only the lowpass (LL) band of one 2D level; dpBuffer is not used.
CUCOMP_DLL void dwtIntForwardLowpassOnly(short* dpDest, short* dpBuffer, const short* dpSource, int sizeX, int sizeY,
                                         int dstRowPitch = 0, int srcRowPitch = 0, cudaStream_t stream = 0);

}
}

#endif
