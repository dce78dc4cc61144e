// codec.cuh - device data structures of the entropy coder (run-length +
// Huffman) and the instance that owns their memory.
//
// Byte format (written by encode, read by decode) follows the reference
// exactly (Encode.cpp:400-463 for encodeRLHuff, :751-782 for encodeHuff):
//   RLHuff stream: u32 compactCount | table(sym) | u32 bits | codewords | u16 offsets
//                  | table(zero counts) | u32 bits | codewords | u16 offsets
//   Huff stream:   table | u32 bits | codewords | u16 offsets
// where every "u32"/codeword/offset block is word aligned before and after,
// tables are bit packed (HuffmanTable.cu:470-485) and offsets are the 16-bit
// increments of the coding-block bit offsets (PackInc.cu:210-219).
#pragma once

#include <cstddef>
#include <map>
#include <string>
#include <vector>

#include "cc_common.cuh"

namespace ccb {

enum CodecKind : int { KIND_RLHUFF = 0, KIND_HUFF = 1 };

// Tile of the run-length passes: 256 threads x 8 symbols.
constexpr u32 kRleThreads = 256;
constexpr u32 kRlePerThread = 32;
constexpr u32 kRleTile = kRleThreads * kRlePerThread;
// The Huffman block kernels take coding blocks in runs of kRunSymbols symbols
// of one table (32 per lane of a warp): 1024 / codingBlockSize blocks.
constexpr u32 kRunSymbols = 1024;

// Tables planned by one CTA of the encode's and decode's table plans (1024
// threads, four tables each); a call of more tables runs one CTA per chunk
// and a carry pass over the chunks' sums (planPart).
constexpr u32 kPlanChunk = 4096;
constexpr u64 planPartWords(u64 tables) { return 8 * ((tables + kPlanChunk - 1) / kPlanChunk + 1); }

// Leaves of a table whose Huffman build runs in shared memory (20 bytes per
// leaf: heap key, sort key, two parent links); larger tables use global memory.
constexpr u32 kBuildSmemLeaves = 8192;

// Words of a serialized table with `leaves` symbols (HuffmanTable.cu:470-485
// field sizes at their maxima: 31 codeword lengths, 24-bit symbols) plus two
// words of slack.
CC_HD u32 headerWordsFor(u32 leaves, u32 log2Max) {
    const u64 symBits = log2Max > 16 ? 24 : 16;
    const u64 bits = 5 + 31ull * log2Max + log2Max + 5 + u64(leaves) * symBits;
    return u32(ceilDiv(bits, 32) + 2);
}

// Per-stream input of one encode call (host side).
struct EncStream {
    const void* in;      // device symbols (u16 or u32)
    u32 n;               // symbol count
    u32 startBit;        // bit offset (0..31) of the segment start in its first word
    u32 groupFirst;      // first stream of the reference call this stream belongs to
    u32 groupSize;       // streams in that call
    u32 kind;            // KIND_RLHUFF or KIND_HUFF
};

// Device copy of a stream with its offsets into the call's work arrays.
struct EncStreamDev {
    const void* in;
    u32 n, kind, startBit, groupFirst, groupSize;
    u32 tileOff;         // first run-length tile of the stream
    u32 tableFirst;      // first Huffman table of the stream
    u32 pad;
    u64 compactOff;      // element offset of its compact symbols / zero counts
};

// One Huffman table of a call: the symbols of a Huff stream, or the compact
// symbols (which 0) / zero counts (which 1) of an RLHuff stream.
struct EncTableDev {
    u32 stream, which;
    u32 blockOff;        // first coding block in the call's block arrays
    u32 blocksMax;       // coding blocks if every symbol is coded (ceil(n / cb))
};

// Summary of a run of symbols for the zero-run RLE scan.  Positions are
// stored +1 so that the virtual "nonzero before the stream" sits at 0.
struct RunSum {
    u32 cnt;       // nonzero symbols
    u32 ext;       // extra (0, 255) entries for the gaps between them
    u32 firstP1;   // position+1 of the first nonzero (valid if cnt)
    u32 lastP1;    // position+1 of the last nonzero (valid if cnt)
};

CC_HD RunSum runCombine(const RunSum& a, const RunSum& b) {
    if (a.cnt == 0) return b;
    if (b.cnt == 0) return a;
    RunSum r;
    r.cnt = a.cnt + b.cnt;
    r.ext = a.ext + b.ext + (b.firstP1 - a.lastP1 - 1u) / 256u;
    r.firstP1 = a.firstP1;
    r.lastP1 = b.lastP1;
    return r;
}

// Per-tile result of the scan: where its output starts and the position+1
// of the last nonzero before the tile (0 = none).
struct TileStart {
    u32 out;
    u32 prevP1;
};

// Per-table results of an encode call (device).
struct TableMeta {
    u32 count;        // symbols coded with this table
    u32 symbolMax;    // largest symbol (0 for an empty stream)
    u32 leaves;       // distinct symbols
    u32 maxLen;       // longest codeword
    u32 headerBits;   // serialized table size
    u32 codeBits;     // total codeword bits
    u32 blocks;       // coding blocks
    u32 histSize;     // histogram bins of this table
    u32 actOff;       // first of its coding blocks in the call's list of used blocks
    u32 runOff;       // first of its runs (kRunSymbols symbols of coding blocks) in the call's run list
    u64 histOff;      // offset of its histogram and code table
    u64 leafOff;      // offset of its table-builder arrays (by leaf)
    u64 hdrOff;       // offset of its serialized header (words)
};

// Where the pieces of one stream's segment go in the device output buffer.
struct SegmentLayout {
    u64 startWord;        // first word of the segment
    u32 words;            // segment size in words
    u32 startBit;         // bit offset of the first written bit inside word 0
    u32 bitLength;        // bits from word 0 bit 0 to the end of the segment
    u32 hdrWord[2];       // relative word of each table header
    u32 cwWord[2];        // relative word of each codeword block
    u32 offWord[2];       // relative word of each offset block
    u32 countWord;        // relative word of compactCount (RLHuff)
};

// Decode-side table descriptor, filled by the host walk of a caller's bit
// stream (cc_decode) or by the device walk of a device-resident one.
struct DecTableDesc {
    u64 hdrBit;       // absolute bit of the table header in its stream's words
    u64 cwWord;       // first codeword word
    u64 offWord;      // first word of the u16 offset increments
    u32 cwBits;       // codeword bits
    u32 count;        // symbols to decode
    u32 symbolBits;   // bits per symbol in the header
    u32 nLen;         // number of codeword lengths
    u32 nSym;         // symbols in the table
    u32 stream;       // owning stream
    u32 blockOff;     // first of its coding blocks in the call's block arrays
    u32 symOff;       // first of its symbols in the decode symbol array
};

// A bit stream a decode call reads.  Device walk: words may be given as a
// base pointer plus a device array of word offsets (results of a batched
// encode), resolved by the walk.
struct DecSource {
    const u32* words;
    u64 wordCount;
    u64 bitSize;      // readable bits
    u64 startBit;     // device walk: where its first stream starts
    u64 endBit;       // device walk: where its last stream ends
    u32 firstStream;  // device walk: its streams, in stream order
    u32 streamCount;
};

struct DecStreamDesc {
    void* out;        // device output symbols
    u64 zcOff;        // RLHuff: offset of its decoded zero counts
    u32 n;            // output symbol count
    u32 m;            // compact count (RLHuff) / n (Huff)
    u32 kind;         // KIND_RLHUFF or KIND_HUFF
    u32 tableFirst;   // its first table (RLHuff: symbols, then zero counts)
    u32 source;       // index of its DecSource
    u32 blockFirst;   // first of its blocks among the streams of its kind
};

// Decode tables in device memory: canonical description + fast lookup.
constexpr u32 kLutBits = 10;
struct DecTable {
    int firstIndex[32];
    int minCode[32];
    int maxCode[32];
    u32 nSym;
    u32 single;       // symbol when nSym <= 1
    u32 pad[2];
};

}  // namespace ccb

// The instance: limits, stream, device arena and host staging.
struct cc_instance {
    int device = -1;
    unsigned streamCountMax = 0;
    unsigned elemCountPerStreamMax = 0;
    unsigned codingBlockSize = 0;
    unsigned log2Max = 0;
    cudaStream_t stream = nullptr;
    // the table build's large-table launch runs on this side stream beside
    // the small-table launch on `stream` (fork / join by the two events)
    cudaStream_t buildSide = nullptr, buildSide2 = nullptr;   // the table builders' other streams
    cudaEvent_t buildFork = nullptr, buildJoin = nullptr, buildJoin2 = nullptr;
    cudaEvent_t decFork = nullptr, decJoin = nullptr;   // the decode's Huff branch on buildSide2

    // derived sizes
    ccb::u32 bins = 0;          // 1 << log2Max
    ccb::u32 symBytes = 0;      // 2, or 4 when log2Max > 16
    ccb::u32 tilesMax = 0;      // run-length tiles per stream
    ccb::u32 blocksMax = 0;     // coding blocks per stream
    ccb::u32 hdrWordsMax = 0;   // serialized table words
    ccb::u32 leavesMax = 0;     // distinct symbols per table
    ccb::u64 outWordsMax = 0;   // device output words

    // capacities of one encode call (totals over its streams / tables)
    ccb::u32 capStreams = 0;    // streams (>= streamCountMax; batched pipelines use more)
    ccb::u64 capCompact = 0;    // run-length output symbols
    ccb::u32 capTiles = 0;      // run-length tiles
    ccb::u32 capTables = 0;     // Huffman tables
    ccb::u32 capBlocks = 0;     // coding blocks
    ccb::u64 capHist = 0;       // histogram bins
    ccb::u64 capLeaves = 0;     // table-builder leaves
    ccb::u64 capHdr = 0;        // serialized header words

    // device memory (one allocation)
    char* arena = nullptr;
    size_t arenaBytes = 0;
    void* compact = nullptr;    // encode: compact symbols; decode: staging of decoded zero counts
    void* zc = nullptr;         // zero counts
    ccb::RunSum* tiles = nullptr;
    ccb::TileStart* tileStart = nullptr;
    ccb::u32* streamMax = nullptr;     // [capStreams] largest symbol
    ccb::u32* hist = nullptr;          // [capHist]
    uint2* enc = nullptr;              // [capHist] (code, len) by symbol
    ccb::TableMeta* meta = nullptr;    // [capTables]
    ccb::u32* tierTables = nullptr;    // [4 capTables]: the tables of each leaf-count tier of a call
    ccb::u64* planPart = nullptr;      // [2 planPartWords(capTables)]: sums of each chunk of a table plan
    ccb::u32* headers = nullptr;       // [capHdr]
    ccb::u32* blockBits = nullptr;     // [capBlocks]
    ccb::u32* blockOff = nullptr;      // [capBlocks]
    ccb::u32* blockTable = nullptr;    // [capBlocks]: table of each coding block of a call
    ccb::u32* runTable = nullptr;      // [capBlocks]: table of each run of coding blocks of a call
    ccb::u32* tileStream = nullptr;    // [capTiles]: stream of each run-length tile of a call
    ccb::SegmentLayout* layout = nullptr;  // [capStreams]
    ccb::u32* out = nullptr;           // [outWordsMax]
    ccb::u32* counts = nullptr;        // [capStreams]
    ccb::u32* errors = nullptr;        // [8]
    ccb::u64* totals = nullptr;        // [8]
    void* dPlan = nullptr;             // stream + table descriptors of the current call
    ccb::u64* leafWork = nullptr;      // [capLeaves] heap keys (tables too large for shared memory)
    ccb::u32* parentWork = nullptr;    // [2 capLeaves]
    ccb::u32* orderWork = nullptr;     // [capLeaves]
    ccb::u32* leafSymWork = nullptr;   // [capLeaves]
    // decode (descriptors live in dPlan)
    ccb::DecTable* decTables = nullptr;       // [capTables]
    ccb::u32* decSyms = nullptr;              // [capLeaves]
    ccb::u32* decLut = nullptr;               // [capTables][1 << kLutBits]
    ccb::u32* stagedWords = nullptr;          // decode input words (host bit streams)
    ccb::u64 stagedWordsMax = 0;
    ccb::u32* blockSum = nullptr;             // [capBlocks]
    bool tableBuildSoloSM = false;            // table-build CTAs ask for a whole SM (calls of <= smCount tables)
    int smCount = 148;
    ccb::u64* decRlTasks = nullptr;           // [capBlocks / 32 + capStreams + 1]: run-length decode warp tasks, then their count

    // host staging: ring of slots for uploads, one buffer for downloads
    static constexpr int kRing = 8;
    char* hostRing[kRing] = {};
    size_t hostRingBytes = 0;
    cudaEvent_t ringEvent[kRing] = {};
    int ringNext = 0;
    char* hostDown = nullptr;
    size_t hostDownBytes = 0;
    ccb::u32* hostWords = nullptr;   // encoded words (host)
    ccb::u64 hostWordsMax = 0;
    std::vector<ccb::SegmentLayout> lastLayout;

    // kernel timing (cudaEvent pairs on the instance stream, resolved lazily)
    bool timing = false;
    struct Section { const char* name; cudaEvent_t a, b; };
    std::vector<Section> pendingSections;
    std::vector<cudaEvent_t> freeEvents;
    std::map<std::string, std::pair<double, unsigned>> timings;
    cudaEvent_t takeEvent();
    void resolveTimings();

    // whole-pipeline workspace (volume / heightfield codecs), grown on demand
    char* pipeWork = nullptr;
    size_t pipeWorkBytes = 0;
    // the plain volume calls' volume batches (pipeline.cu plainBatchFor):
    // two kept, by (volume count, nx, ny, nz, levels), least recently used
    // replaced; a shape gets one on its fifth consecutive call
    struct PlainBatch {
        cc_volume_batch* b = nullptr;
        ccb::u32 key[5] = {};
        ccb::u64 used = 0;
    };
    PlainBatch plainBatch[2];
    ccb::u32 plainSeenKey[5] = {};
    ccb::u32 plainSeenRun = 0;        // consecutive calls of plainSeenKey
    ccb::u64 plainCalls = 0;

    char* takeRingSlot();
};
