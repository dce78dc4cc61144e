// batch.cuh - descriptors and launchers of the batched volume codec's
// transform kernels (dwt.cu).  Every launch covers one pass of one level for
// all volumes of a batch: its CTAs are numbered across the volumes and each
// CTA finds its volume's descriptor by binary search over ctaOff.
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
    u32 ctaOff;
};

// Y or Z pass: 32 x-columns by 64 axis positions per CTA.  With `bands`
// set it is the first inverse pass of dwtFloat3DInverseFromSymbols: the
// lowpass octant comes from src (lpRow, lpSlice pitches), the other seven
// from dequantized symbol bands (band b-1 at bands + (b-1) * bandStride).
struct BColDesc {
    const float* src;
    float* dst;
    int nx, na, nc;
    int sx, sa, sc;         // source strides (x, axis, other)
    int dx, da, dc;         // destination strides
    const u16* bands;
    u64 bandStride;
    float step;
    int hx, hy, hz, lpRow, lpSlice;
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
    u32 ctaOff;             // 1024 elements per CTA
};

constexpr int kBRowOutputs = 512;
constexpr int kBQuantPerCta = 1024;

// Descriptor arrays are device pointers; ctas = total CTA count.
void launchBatchRows(const BRowDesc* d, u32 nd, u32 ctas, bool inverse, const float* const* inTab,
                     float* const* outTab, cudaStream_t st);
void launchBatchCols(const BColDesc* d, u32 nd, u32 ctas, bool inverse, bool fromSymbols, cudaStream_t st);
void launchBatchQuant(const BQuantDesc* d, u32 nd, u32 ctas, bool dequantize, cudaStream_t st);

// Row tiling of an X pass over an nx-wide level: tile width, rows per CTA.
inline void batchRowTiling(int nx, int& W, int& R) {
    W = nx < kBRowOutputs ? nx : kBRowOutputs;
    R = kBRowOutputs / W;
    if (R < 1) R = 1;
    if (R > 64) R = 64;
}

}  // namespace ccb
