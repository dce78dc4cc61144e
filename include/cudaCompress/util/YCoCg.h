// util/YCoCg.h - RGB <-> YCoCg colour conversion (drop-in for the reference's
// include/cudaCompress/util/YCoCg.h:14-20).  The non-reversible transform:
// it keeps the dynamic range and loses one bit in the chroma channels.
// dpTarget and dpData may point to the same memory.  Default stream.
#ifndef CUDACOMPRESS_B200_YCOCG_H
#define CUDACOMPRESS_B200_YCOCG_H

#include <cudaCompress/global.h>

#include <vector_types.h>

namespace cudaCompress {
namespace util {

CUCOMP_DLL void convertRGBtoYCoCg(uchar3* dpTarget, const uchar3* dpData, int pixelCount);
CUCOMP_DLL void convertYCoCgtoRGB(uchar3* dpTarget, const uchar3* dpData, int pixelCount);

CUCOMP_DLL void convertRGBtoYCoCg(uchar4* dpTarget, const uchar4* dpData, int pixelCount);
CUCOMP_DLL void convertYCoCgtoRGB(uchar4* dpTarget, const uchar4* dpData, int pixelCount);

}
}

#endif
