// Instance.h - coder instance (drop-in for reference Instance.h:26-45).
#ifndef CUDACOMPRESS_B200_INSTANCE_H
#define CUDACOMPRESS_B200_INSTANCE_H

#include <cudaCompress/global.h>

#include <cuda_runtime.h>

namespace cudaCompress {

// Owns every device buffer and host staging area the coder needs; sized at
// creation from the limits below, so coding calls do not allocate.
class Instance;

// cudaDevice: device index, or -1 for the current device.
// streamCountMax: most symbol streams coded in one call.
// elemCountPerStreamMax: most symbols per stream.
// codingBlockSize: Huffman parallelization granularity, 32/64/128/256 (0 -> 128).
// log2HuffmanDistinctSymbolCountMax: symbol alphabet is [0, 2^this) (0 -> 14, max 24).
// Returns nullptr on failure.
CUCOMP_DLL Instance* createInstance(int cudaDevice, uint streamCountMax, uint elemCountPerStreamMax,
                                    uint codingBlockSize = 0, uint log2HuffmanDistinctSymbolCountMax = 0);
CUCOMP_DLL void destroyInstance(Instance* pInstance);

CUCOMP_DLL int getInstanceCudaDevice(const Instance* pInstance);
CUCOMP_DLL uint getInstanceStreamCountMax(const Instance* pInstance);
CUCOMP_DLL uint getInstanceElemCountPerStreamMax(const Instance* pInstance);
CUCOMP_DLL uint getInstanceCodingBlockSize(const Instance* pInstance);
CUCOMP_DLL uint getInstanceLog2HuffmanDistinctSymbolCountMax(const Instance* pInstance);
CUCOMP_DLL bool getInstanceUseLongSymbols(const Instance* pInstance);

// Stream used by every kernel of the instance.  Both spellings are provided:
// the reference declares the *CudaStream names and defines the *Stream ones.
CUCOMP_DLL void setInstanceCudaStream(Instance* pInstance, cudaStream_t str);
CUCOMP_DLL cudaStream_t getInstanceCudaStream(const Instance* pInstance);
CUCOMP_DLL void setInstanceStream(Instance* pInstance, cudaStream_t str);
CUCOMP_DLL cudaStream_t getInstanceStream(const Instance* pInstance);

}

#endif
