// global.h - basic integer types of the cudaCompress C++ API
// (drop-in for include/cudaCompress/global.h of the reference).
#ifndef CUDACOMPRESS_B200_GLOBAL_H
#define CUDACOMPRESS_B200_GLOBAL_H

namespace cudaCompress {

typedef unsigned char byte;
typedef unsigned char uchar;
typedef unsigned short ushort;
typedef unsigned int uint;
typedef long long int int64;
typedef unsigned long long int uint64;

}

// The library is built as a shared object with default visibility; the
// export macro exists for source compatibility.
#ifndef CUCOMP_DLL
#define CUCOMP_DLL
#endif

#endif
