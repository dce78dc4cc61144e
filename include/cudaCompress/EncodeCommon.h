// EncodeCommon.h - symbol types and format constants (reference EncodeCommon.h:10-31).
#ifndef CUDACOMPRESS_B200_ENCODE_COMMON_H
#define CUDACOMPRESS_B200_ENCODE_COMMON_H

#include <cudaCompress/global.h>

namespace cudaCompress {

typedef ushort Symbol16;
typedef uint Symbol32;

const Symbol16 INVALID_SYMBOL16 = Symbol16(-1);
const Symbol32 INVALID_SYMBOL32 = Symbol32(-1);

// field widths of the serialized Huffman table
const uint LOG2_MAX_SYMBOL16_BITS = 4;
const uint MAX_SYMBOL16_BITS = 1u << LOG2_MAX_SYMBOL16_BITS;
const uint LOG2_MAX_SYMBOL32_BITS = 5;
const uint MAX_SYMBOL32_BITS = 1u << LOG2_MAX_SYMBOL32_BITS;
const uint LOG2_MAX_CODEWORD_BITS = 5;
const uint MAX_CODEWORD_BITS = 1u << LOG2_MAX_CODEWORD_BITS;

const uint LOG2_HUFFMAN_LOOKUP_SIZE = 7;
const uint HUFFMAN_LOOKUP_SIZE = 1u << LOG2_HUFFMAN_LOOKUP_SIZE;

// longest zero run one (symbol, zero count) pair can describe
const uint ZERO_COUNT_MAX = 255;

}

#endif
