// util/Bits.h - least-significant-bit planes of short arrays (drop-in for the
// reference's include/cudaCompress/util/Bits.h:14-27).  Bit j of word w of
// dpBits belongs to element 32 w + j.  The reference processes whole blocks
// of 4096 elements (its callers pad); these touch exactly elemCount elements.
// All return true unless a launch fails.  Default stream.
#ifndef CUDACOMPRESS_B200_BITS_H
#define CUDACOMPRESS_B200_BITS_H

#include <cudaCompress/global.h>

namespace cudaCompress {
namespace util {

// the least significant bit of each element into dpBits
CUCOMP_DLL bool getLSB(const short* dpData, uint* dpBits, uint elemCount);
// v -> (v + shift) without its least significant bit (floor of half); the
// removed bits into dpBits if non-null
CUCOMP_DLL bool removeLSB(short* dpData, uint* dpBits, uint elemCount, short shift = 0);
// v -> 2v + bit + shift
CUCOMP_DLL bool appendLSB(short* dpData, const uint* dpBits, uint elemCount, short shift = 0);
// v -> v + shift
CUCOMP_DLL bool shiftElems(short* dpData, uint elemCount, short shift);

}
}

#endif
