// batch.cuh - descriptors and launchers of the batched volume codec's
// transform kernels (dwt.cu).  Every launch covers one pass of one level for
// all volumes of a batch: its CTAs are numbered across the volumes and a
// per-launch CTA map (u32 per CTA) gives each CTA its descriptor's index.
#pragma once

#include "capi_internal.cuh"

namespace ccb {

// X pass (DWTFloatKernels.cui row kernels): rows of one volume level.
struct BRowDesc {
    const float* src;       // nullptr: the volume's entry of the input pointer table
    float* dst;             // nullptr: the volume's entry of the output pointer table
    int vol;
    int nx, ny, nz;
    int srcRow, srcSlice, dstRow, dstSlice;
    int W, R, tilesX;       // tile width, rows per CTA, tiles per row
    int vec;                // nx, W and all pitches allow float4 rows (pointers are checked per CTA)
    u32 ctaOff;
};

// Y or Z pass: kBColTileX x-columns (unit stride, float2 pairs) by
// kBColTileA axis positions per CTA.  With `bands`
// set it is the first inverse pass of dwtFloat3DInverseFromSymbols: the
// lowpass octant comes from src (lpRow, lpSlice pitches), the other seven
// from dequantized symbol bands (band b-1 at bands + (b-1) * bandStride).
struct BColDesc {
    const float* src;
    float* dst;
    int nx, na, nc;
    int sa, sc;             // source strides (axis, other); x has unit stride
    int da, dc;             // destination strides
    const u16* bands;
    u64 bandStride;
    float step;
    int hx, hy, hz, lpRow, lpSlice;
    // last forward pass of a level (axis Z) with quantization fused into the
    // store: the 7 highpass octants go to symOut (band b-1 at b-1 bandStride)
    // quantized with inv; the LLL octant stays float in dst, or - at the
    // coarsest level - goes to lpSymOut quantized with invLP
    u16* symOut;
    u16* lpSymOut;
    float inv, invLP;
    int lastLevel;
    u32 tilesX, tilesA;
    u32 ctaOff;
};

// One band: deadzone quantization to u16 symbols (src strided -> sym dense),
// or (dstF set) dequantization of dense symbols to a dense float block.
struct BQuantDesc {
    const float* src;
    u16* sym;
    float* dstF;
    int nx, ny, nz, row, slice;
    float step, inv;
    u32 ctaOff;             // kBQuantPerCta elements per CTA
};

// One forward level in one pass (k_bLevelFwd): a CTA owns kLvTX x kLvTY
// outputs of the level's XY plane (positions in the filtering domain) and
// zChunk output slices; it streams the input slices through X and Y filters
// in shared memory and a 9-slice Z window in registers, and stores the seven
// highpass octants as quantized symbols and the LLL octant as float (tight
// hx x hy x hz, the next level's input) - or, at the coarsest level, as
// symbols too.
struct BLevelDesc {
    const float* src;       // level input; nullptr: the volume's entry of the input pointer table
    int vol;
    int nx, ny, nz;         // level extents (even, >= 8)
    int srcRow, srcSlice;
    float* lpOut;           // LLL octant, tight (not the coarsest level)
    u16* symOut;            // highpass octant b at symOut + (b - 1) * bandStride, tight hx x hy x hz
    u16* lpSymOut;          // coarsest level: the LLL octant's symbols, tight
    u64 bandStride;
    float inv, invLP;       // reciprocal quantization steps (highpass, lowpass band)
    int lastLevel;
    int tilesX, tilesY, chunksZ;
    int zChunk;             // output slices per CTA (the Z extent of its tile)
    u32 ctaOff;
};
constexpr int kLvTX = 64, kLvTY = 16;
constexpr int kLvZCDefault = 32;   // default Z extent of a tile (cc_volume_batch_create_ex: 8..256)

constexpr int kBRowOutputs = 4096;    // outputs per row-pass CTA
constexpr int kBRowMaxWidth = 2048;   // row tile width
constexpr int kBRowMaxRows = 128;     // rows per row-pass CTA
constexpr int kBRowSmem = kBRowOutputs + 8 * kBRowMaxRows;   // floats: R rows of W + 8
constexpr int kBColTileX = 64;
constexpr int kBColTileA = 64;
constexpr int kBQuantPerCta = 4096;

// Descriptor arrays and CTA maps are device pointers; ctas = CTA count.
void launchBatchRows(const BRowDesc* d, const u32* map, u32 ctas, bool inverse, const float* const* inTab,
                     float* const* outTab, cudaStream_t st);
void launchBatchCols(const BColDesc* d, const u32* map, u32 ctas, bool inverse, bool fromSymbols, cudaStream_t st,
                     bool quantizeStore = false);
void launchBatchQuant(const BQuantDesc* d, const u32* map, u32 ctas, bool dequantize, cudaStream_t st);
void launchBatchLevelFwd(const BLevelDesc* d, const u32* map, u32 ctas, const float* const* inTab, cudaStream_t st);

// Row tiling of an X pass over an nx-wide level: tile width, rows per CTA.
inline void batchRowTiling(int nx, int& W, int& R) {
    W = nx < kBRowMaxWidth ? nx : kBRowMaxWidth;
    R = kBRowOutputs / W;
    if (R < 1) R = 1;
    if (R > kBRowMaxRows) R = kBRowMaxRows;
}

// New quantization steps for a batch's volumes (batch.cu).
int batchSetQuantSteps(cc_volume_batch* b, const float* q);
// The error status of the batch's last compress (decode false) or decompress
// (decode true), after synchronizing its stream (batch.cu).
int batchStatusOf(cc_volume_batch* b, bool decode);

}  // namespace ccb
