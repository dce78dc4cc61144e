// Encode.h - run-length + Huffman coding of device symbol streams
// (drop-in for reference Encode.h:17-52).
#ifndef CUDACOMPRESS_B200_ENCODE_H
#define CUDACOMPRESS_B200_ENCODE_H

#include <cstddef>

#include <cudaCompress/global.h>
#include <cudaCompress/BitStream.h>
#include <cudaCompress/EncodeCommon.h>

namespace cudaCompress {

class Instance;

// Device bytes held by the instance; init/shutdown are no-ops kept for
// source compatibility (the instance sets itself up at creation).
size_t encodeGetRequiredMemory(const Instance* pInstance);
bool encodeInit(Instance* pInstance);
bool encodeShutdown(Instance* pInstance);

// Notes on the contract (same as the reference):
// - encode* appends to the bit stream(s) and returns once it is complete.
// - decode* reads from the current position, advances it, and returns once
//   the work is queued on the instance stream.
// - decodeRLHuff outputs must be zeroed by the caller in the reference;
//   here every output symbol is written, so zeroing is not needed.
// - Symbol16 calls need log2HuffmanDistinctSymbolCountMax <= 16, Symbol32
//   calls need > 16 (the reference silently misreads the buffers otherwise;
//   here the call returns false).
// - Unlike the reference, inputs are not modified and outputs need no
//   padding beyond the symbol count.

// one bit stream for all streams
CUCOMP_DLL bool encodeRLHuff(Instance* pInstance, BitStream& bitStream, const Symbol16* const pdpSymbolStreams[], uint streamCount, uint symbolCountPerBlock);
CUCOMP_DLL bool decodeRLHuff(Instance* pInstance, BitStreamReadOnly& bitStream, Symbol16* pdpSymbolStreams[], uint streamCount, uint symbolCountPerBlock);
CUCOMP_DLL bool encodeHuff(Instance* pInstance, BitStream& bitStream, /*const*/ Symbol16* const pdpSymbolStreams[], uint streamCount, uint symbolCountPerBlock);
CUCOMP_DLL bool decodeHuff(Instance* pInstance, BitStreamReadOnly& bitStream, Symbol16* pdpSymbolStreams[], uint streamCount, uint symbolCountPerBlock);

CUCOMP_DLL bool encodeRLHuff(Instance* pInstance, BitStream& bitStream, const Symbol32* const pdpSymbolStreams[], uint streamCount, uint symbolCountPerBlock);
CUCOMP_DLL bool decodeRLHuff(Instance* pInstance, BitStreamReadOnly& bitStream, Symbol32* pdpSymbolStreams[], uint streamCount, uint symbolCountPerBlock);
CUCOMP_DLL bool encodeHuff(Instance* pInstance, BitStream& bitStream, /*const*/ Symbol32* const pdpSymbolStreams[], uint streamCount, uint symbolCountPerBlock);
CUCOMP_DLL bool decodeHuff(Instance* pInstance, BitStreamReadOnly& bitStream, Symbol32* pdpSymbolStreams[], uint streamCount, uint symbolCountPerBlock);

// one bit stream per stream (entries may repeat; repeated streams are appended in order)
CUCOMP_DLL bool encodeRLHuff(Instance* pInstance, BitStream* ppBitStreams[], const Symbol16* const pdpSymbolStreams[], uint streamCount, uint symbolCountPerBlock);
CUCOMP_DLL bool decodeRLHuff(Instance* pInstance, BitStreamReadOnly* ppBitStreams[], Symbol16* pdpSymbolStreams[], uint streamCount, uint symbolCountPerBlock);
CUCOMP_DLL bool encodeHuff(Instance* pInstance, BitStream* ppBitStreams[], /*const*/ Symbol16* const pdpSymbolStreams[], uint streamCount, uint symbolCountPerBlock);
CUCOMP_DLL bool decodeHuff(Instance* pInstance, BitStreamReadOnly* ppBitStreams[], Symbol16* pdpSymbolStreams[], uint streamCount, uint symbolCountPerBlock);

CUCOMP_DLL bool encodeRLHuff(Instance* pInstance, BitStream* ppBitStreams[], const Symbol32* const pdpSymbolStreams[], uint streamCount, uint symbolCountPerBlock);
CUCOMP_DLL bool decodeRLHuff(Instance* pInstance, BitStreamReadOnly* ppBitStreams[], Symbol32* pdpSymbolStreams[], uint streamCount, uint symbolCountPerBlock);
CUCOMP_DLL bool encodeHuff(Instance* pInstance, BitStream* ppBitStreams[], /*const*/ Symbol32* const pdpSymbolStreams[], uint streamCount, uint symbolCountPerBlock);
CUCOMP_DLL bool decodeHuff(Instance* pInstance, BitStreamReadOnly* ppBitStreams[], Symbol32* pdpSymbolStreams[], uint streamCount, uint symbolCountPerBlock);

}

#endif
