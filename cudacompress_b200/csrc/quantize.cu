// quantize.cu - util::quantize* / symbolize (Quantize.h:25-65, Quantize.cu:46-361,
// QuantizeKernels.cui:39-285, Quantize.cuh:26-147).
//
//   symbolize(v)   = 2|v| + (v < 0 ? -1 : 0)          (>= 0 even, < 0 odd)
//   deadzone q(v)  = int(v * (1/step)), 1/step rounded on the host
//   uniform  q(v)  = int(v * (1/step) + sign(v) * 0.5)
//   deadzone v(q)  = (q + sign(q) * 0.5) * step
//   uniform  v(q)  = q * step
// Symbol16 stores truncate silently, as in the reference.
#include "capi_internal.cuh"

namespace ccb {


struct Box {
    u32 nx, ny, nz;
    u32 row, slice;    // pitches of the strided side
};

__device__ __forceinline__ bool boxIndex(const Box& b, u64& dense, u64& strided) {
    const u64 i = u64(blockIdx.x) * blockDim.x + threadIdx.x;
    const u64 plane = u64(b.nx) * b.ny;
    if (i >= plane * b.nz) return false;
    const u32 z = u32(i / plane);
    const u32 r = u32(i - u64(z) * plane);
    const u32 y = r / b.nx, x = r - y * b.nx;
    dense = i;
    strided = u64(z) * b.slice + u64(y) * b.row + x;
    return true;
}

template <class Sym>
__global__ void k_quantize(Sym* out, const float* in, Box b, float inv, int type) {
    u64 d, s;
    if (!boxIndex(b, d, s)) return;
    out[d] = Sym(symbolizeI(quantizeV(in[s], inv, type)));
}

template <class Sym>
__global__ void k_quantizeRoundtrip(Sym* out, float* data, Box b, float step, float inv, int type) {
    u64 d, s;
    if (!boxIndex(b, d, s)) return;
    int q = quantizeV(data[s], inv, type);
    out[d] = Sym(symbolizeI(q));
    data[s] = unquantizeV(q, step, type);
}

template <class Sym>
__global__ void k_unquantize(float* data, const Sym* in, Box b, float step, int type) {
    u64 d, s;
    if (!boxIndex(b, d, s)) return;
    data[s] = unquantizeV(unsymbolizeI(u32(in[d])), step, type);
}

__global__ void k_symbolize(u16* out, const i16* in, Box b) {
    u64 d, s;
    if (!boxIndex(b, d, s)) return;
    out[d] = u16(symbolizeI(int(in[s])));
}
__global__ void k_unsymbolize(i16* out, const u16* in, Box b) {
    u64 d, s;
    if (!boxIndex(b, d, s)) return;
    out[s] = i16(unsymbolizeI(u32(in[d])));
}
__global__ void k_quantizeShort(i16* out, const float* in, Box b, float inv, int type) {
    u64 d, s;
    if (!boxIndex(b, d, s)) return;
    out[d] = i16(quantizeV(in[s], inv, type));
}
__global__ void k_unquantizeShort(float* out, const i16* in, Box b, float step, int type) {
    u64 d, s;
    if (!boxIndex(b, d, s)) return;
    out[s] = unquantizeV(int(in[d]), step, type);
}

__global__ void k_maxAbs(const float* in, u32 n, float* out) {
    __shared__ float part[32];
    float m = 0.0f;
    for (u64 i = u64(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += u64(gridDim.x) * blockDim.x)
        m = fmaxf(m, fabsf(in[i]));
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32) {
        m = threadIdx.x < blockDim.x / 32 ? part[threadIdx.x] : 0.0f;
        for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
        // non-negative floats order like their bit patterns
        if (threadIdx.x == 0) atomicMax(reinterpret_cast<unsigned int*>(out), __float_as_uint(m));
    }
}

static Box makeBox(u32 nx, u32 ny, u32 nz, u32 row, u32 slice) {
    Box b{nx, ny, nz, row ? row : nx, 0};
    b.slice = slice ? slice : b.row * ny;
    return b;
}
static unsigned gridFor(const Box& b) { return unsigned(ceilDiv(u64(b.nx) * b.ny * b.nz, 256)); }

}  // namespace ccb

using namespace ccb;

extern "C" {

int cc_quantize_to_symbols(void* out, int symBytes, const float* in, uint32_t nx, uint32_t ny, uint32_t nz, float step,
                           uint32_t row, uint32_t slice, int type, void* stream) {
    if (symBytes != 2 && symBytes != 4) { setError("symbol size must be 2 or 4"); return CC_ERR_INVALID_ARGUMENT; }
    Box b = makeBox(nx, ny, nz, row, slice);
    if (!u64(nx) * ny * nz) return CC_OK;
    const float inv = 1.0f / step;   // Quantize.cu:90: reciprocal computed on the host
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (symBytes == 2) k_quantize<u16><<<gridFor(b), 256, 0, st>>>(static_cast<u16*>(out), in, b, inv, type);
    else k_quantize<u32><<<gridFor(b), 256, 0, st>>>(static_cast<u32*>(out), in, b, inv, type);
    countLaunch();
    CC_TRY_CUDA(cudaGetLastError(), "quantizeToSymbols");
    return CC_OK;
}

int cc_quantize_to_symbols_roundtrip(void* out, int symBytes, float* data, uint32_t nx, uint32_t ny, uint32_t nz,
                                     float step, uint32_t row, uint32_t slice, int type, void* stream) {
    if (symBytes != 2 && symBytes != 4) { setError("symbol size must be 2 or 4"); return CC_ERR_INVALID_ARGUMENT; }
    Box b = makeBox(nx, ny, nz, row, slice);
    if (!u64(nx) * ny * nz) return CC_OK;
    const float inv = 1.0f / step;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (symBytes == 2) k_quantizeRoundtrip<u16><<<gridFor(b), 256, 0, st>>>(static_cast<u16*>(out), data, b, step, inv, type);
    else k_quantizeRoundtrip<u32><<<gridFor(b), 256, 0, st>>>(static_cast<u32*>(out), data, b, step, inv, type);
    countLaunch();
    CC_TRY_CUDA(cudaGetLastError(), "quantizeToSymbolsRoundtrip");
    return CC_OK;
}

int cc_unquantize_from_symbols(float* data, const void* in, int symBytes, uint32_t nx, uint32_t ny, uint32_t nz,
                               float step, uint32_t row, uint32_t slice, int type, void* stream) {
    if (symBytes != 2 && symBytes != 4) { setError("symbol size must be 2 or 4"); return CC_ERR_INVALID_ARGUMENT; }
    Box b = makeBox(nx, ny, nz, row, slice);
    if (!u64(nx) * ny * nz) return CC_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (symBytes == 2) k_unquantize<u16><<<gridFor(b), 256, 0, st>>>(data, static_cast<const u16*>(in), b, step, type);
    else k_unquantize<u32><<<gridFor(b), 256, 0, st>>>(data, static_cast<const u32*>(in), b, step, type);
    countLaunch();
    CC_TRY_CUDA(cudaGetLastError(), "unquantizeFromSymbols");
    return CC_OK;
}

int cc_symbolize(uint16_t* out, const int16_t* in, uint32_t nx, uint32_t ny, uint32_t nz, uint32_t row, uint32_t slice,
                 void* stream) {
    Box b = makeBox(nx, ny, nz, row, slice);
    if (!u64(nx) * ny * nz) return CC_OK;
    k_symbolize<<<gridFor(b), 256, 0, static_cast<cudaStream_t>(stream)>>>(out, in, b); countLaunch();
    CC_TRY_CUDA(cudaGetLastError(), "symbolize");
    return CC_OK;
}

int cc_unsymbolize(int16_t* out, const uint16_t* in, uint32_t nx, uint32_t ny, uint32_t nz, uint32_t row,
                   uint32_t slice, void* stream) {
    Box b = makeBox(nx, ny, nz, row, slice);
    if (!u64(nx) * ny * nz) return CC_OK;
    k_unsymbolize<<<gridFor(b), 256, 0, static_cast<cudaStream_t>(stream)>>>(out, in, b); countLaunch();
    CC_TRY_CUDA(cudaGetLastError(), "unsymbolize");
    return CC_OK;
}

int cc_quantize_to_short(int16_t* out, const float* in, uint32_t nx, uint32_t ny, uint32_t nz, float step,
                         uint32_t row, uint32_t slice, int type, void* stream) {
    Box b = makeBox(nx, ny, nz, row, slice);
    if (!u64(nx) * ny * nz) return CC_OK;
    k_quantizeShort<<<gridFor(b), 256, 0, static_cast<cudaStream_t>(stream)>>>(out, in, b, 1.0f / step, type); countLaunch();
    CC_TRY_CUDA(cudaGetLastError(), "quantizeToShort");
    return CC_OK;
}

int cc_unquantize_from_short(float* out, const int16_t* in, uint32_t nx, uint32_t ny, uint32_t nz, float step,
                             uint32_t row, uint32_t slice, int type, void* stream) {
    Box b = makeBox(nx, ny, nz, row, slice);
    if (!u64(nx) * ny * nz) return CC_OK;
    k_unquantizeShort<<<gridFor(b), 256, 0, static_cast<cudaStream_t>(stream)>>>(out, in, b, step, type); countLaunch();
    CC_TRY_CUDA(cudaGetLastError(), "unquantizeFromShort");
    return CC_OK;
}

int cc_get_max_abs(cc_instance* I, const float* in, uint32_t n, float* dMax) {
    if (!I) { setError("getMaxAbs: null instance"); return CC_ERR_INVALID_ARGUMENT; }
    cudaStream_t st = I->stream;
    CC_TRY_CUDA(cudaMemsetAsync(dMax, 0, sizeof(float), st), "getMaxAbs");
    if (n) {
        k_maxAbs<<<std::min<u32>(1184u, u32(ceilDiv(n, 256))), 256, 0, st>>>(in, n, dMax);
        countLaunch();
    }
    CC_TRY_CUDA(cudaGetLastError(), "getMaxAbs");
    return CC_OK;
}

}  // extern "C"
