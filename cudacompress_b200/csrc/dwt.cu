// dwt.cu - separable one-level wavelet transforms (util::dwt*, DWT.h:21-157).
//
// Float: CDF 9/7 as a 9-tap FIR per axis (DWTFloatKernels.cui:13-875, taps
// DWTFloatFilters.cuh:42-49) with whole-sample symmetric extension
// (DWTCommon.cuh:54-55); the taps of an output are chosen by the parity of its
// position and accumulated as fma(c[i], v[i], sum), i = 0..8, from 0.0f, so
// results are bit-identical to the reference kernels.  Forward writes even
// positions to the low half and odd ones to the high half of each axis; the
// inverse reads the halves as one interleaved signal.  Axis order: X, Y, Z
// forward; Z, Y, X inverse; intermediates are float32 in the caller's buffers
// with the reference's pitches (DWTFloat.cu:84-463).
//
// Int: CDF 5/3 lifting on shorts (DWTIntKernels.cui:14-1188) with the
// reference's rounding (DWTCommon.cuh:133-142), including the narrowing of
// every intermediate to 16 bits.
#include "batch.cuh"

namespace ccb {

__constant__ float c_fwd[2][9] = {
    {0.0267488f, -0.0168641f, -0.0782233f, 0.2668641f, 0.6029490f, 0.2668641f, -0.0782233f, -0.0168641f, 0.0267488f},
    {0.0f, 0.0456359f, -0.0287718f, -0.2956359f, 0.5575435f, -0.2956359f, -0.0287718f, 0.0456359f, 0.0f}};
__constant__ float c_inv[2][9] = {
    {0.0f, 0.0337282f, -0.0575435f, -0.5337281f, 1.1150871f, -0.5337281f, -0.0575435f, 0.0337282f, 0.0f},
    {0.0534975f, -0.0912718f, -0.1564465f, 0.5912718f, 1.2058980f, 0.5912718f, -0.1564465f, -0.0912718f, 0.0534975f}};

// whole-sample symmetric extension (valid for n >= 5 and |overhang| < n)
__device__ __forceinline__ int mirrorIdx(int i, int n) {
    i = i < 0 ? -i : i;
    return i > n - 1 ? 2 * (n - 1) - i : i;
}
// position of interleaved index j (inverse domain) in the [L|H] layout
__device__ __forceinline__ int splitPos(int j, int n) { return (j & 1) ? (n >> 1) + (j >> 1) : (j >> 1); }

// The same taps as compile-time constants: with the parity known at compile
// time the coefficients become instruction immediates (no divergent
// constant-cache reads when neighbouring threads hold outputs of both
// parities).  Identical fmaf chain, so identical results.
template <bool kInverse, int kParity>
__device__ __forceinline__ float fir9c(const float* v) {
    constexpr float kF[2][9] = {
        {0.0267488f, -0.0168641f, -0.0782233f, 0.2668641f, 0.6029490f, 0.2668641f, -0.0782233f, -0.0168641f, 0.0267488f},
        {0.0f, 0.0456359f, -0.0287718f, -0.2956359f, 0.5575435f, -0.2956359f, -0.0287718f, 0.0456359f, 0.0f}};
    constexpr float kI[2][9] = {
        {0.0f, 0.0337282f, -0.0575435f, -0.5337281f, 1.1150871f, -0.5337281f, -0.0575435f, 0.0337282f, 0.0f},
        {0.0534975f, -0.0912718f, -0.1564465f, 0.5912718f, 1.2058980f, 0.5912718f, -0.1564465f, -0.0912718f, 0.0534975f}};
    float sum = 0.0f;
#pragma unroll
    for (int i = 0; i < 9; ++i) sum = __fmaf_rn(kInverse ? kI[kParity][i] : kF[kParity][i], v[i], sum);
    return sum;
}

// Two outputs of one parity at once, their windows at a and b: Blackwell's
// packed fma.rn.f32x2 does both lanes' fmaf in one instruction, each lane
// rounded exactly as fir9c's scalar chain.
template <bool kInverse, int kParity>
__device__ __forceinline__ float2 fir9x2(const float* a, const float* b) {
    constexpr float kF[2][9] = {
        {0.0267488f, -0.0168641f, -0.0782233f, 0.2668641f, 0.6029490f, 0.2668641f, -0.0782233f, -0.0168641f, 0.0267488f},
        {0.0f, 0.0456359f, -0.0287718f, -0.2956359f, 0.5575435f, -0.2956359f, -0.0287718f, 0.0456359f, 0.0f}};
    constexpr float kI[2][9] = {
        {0.0f, 0.0337282f, -0.0575435f, -0.5337281f, 1.1150871f, -0.5337281f, -0.0575435f, 0.0337282f, 0.0f},
        {0.0534975f, -0.0912718f, -0.1564465f, 0.5912718f, 1.2058980f, 0.5912718f, -0.1564465f, -0.0912718f, 0.0534975f}};
    float2 sum = make_float2(0.0f, 0.0f);
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        const float c = kInverse ? kI[kParity][i] : kF[kParity][i];
        sum = __ffma2_rn(make_float2(c, c), make_float2(a[i], b[i]), sum);
    }
    return sum;
}

// The same over a window of value pairs (lane x: one output, lane y: the other).
template <bool kInverse, int kParity>
__device__ __forceinline__ float2 fir9p(const float2* w) {
    constexpr float kF[2][9] = {
        {0.0267488f, -0.0168641f, -0.0782233f, 0.2668641f, 0.6029490f, 0.2668641f, -0.0782233f, -0.0168641f, 0.0267488f},
        {0.0f, 0.0456359f, -0.0287718f, -0.2956359f, 0.5575435f, -0.2956359f, -0.0287718f, 0.0456359f, 0.0f}};
    constexpr float kI[2][9] = {
        {0.0f, 0.0337282f, -0.0575435f, -0.5337281f, 1.1150871f, -0.5337281f, -0.0575435f, 0.0337282f, 0.0f},
        {0.0534975f, -0.0912718f, -0.1564465f, 0.5912718f, 1.2058980f, 0.5912718f, -0.1564465f, -0.0912718f, 0.0534975f}};
    float2 sum = make_float2(0.0f, 0.0f);
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        const float c = kInverse ? kI[kParity][i] : kF[kParity][i];
        sum = __ffma2_rn(make_float2(c, c), w[i], sum);
    }
    return sum;
}

template <bool kInverse>
__device__ __forceinline__ float fir9(const float* v, int parity) {
    const float* c = kInverse ? c_inv[parity] : c_fwd[parity];
    float sum = 0.0f;
#pragma unroll
    for (int i = 0; i < 9; ++i) sum = __fmaf_rn(c[i], v[i], sum);
    return sum;
}

// ---- element conversions (DWTCommon.cuh:14-50) ----
template <class T> __device__ __forceinline__ float toF(T v);
template <> __device__ __forceinline__ float toF<float>(float v) { return v; }
template <> __device__ __forceinline__ float toF<u8>(u8 v) { return float(v) - 128.0f; }
template <class T> __device__ __forceinline__ T fromF(float v);
template <> __device__ __forceinline__ float fromF<float>(float v) { return v; }
template <> __device__ __forceinline__ u8 fromF<u8>(float v) { return u8(fminf(fmaxf(v + 128.5f, 0.0f), 255.0f)); }

// ---------------------------------------------------------------------------
// Row pass (axis X).  Block: 256 threads, 512 outputs of one row.
// ---------------------------------------------------------------------------
constexpr int kRowTile = 512;

template <class TIn, class TOut, bool kInverse>
__global__ void __launch_bounds__(256) k_firRows(TOut* __restrict__ dst, const TIn* __restrict__ src, int nx,
                                                 int srcElem, int srcRow, int srcSlice, int dstElem, int dstRow,
                                                 int dstSlice) {
    __shared__ float s[kRowTile + 8];
    const int y = blockIdx.y, z = blockIdx.z;
    const int x0 = blockIdx.x * kRowTile;
    const TIn* in = src + size_t(z) * srcSlice + size_t(y) * srcRow;
    TOut* out = dst + size_t(z) * dstSlice + size_t(y) * dstRow;
    for (int k = threadIdx.x; k < kRowTile + 8; k += 256) {
        int j = x0 - 4 + k;
        if (j < nx + 4) {
            int m = mirrorIdx(j, nx);
            s[k] = toF<TIn>(in[size_t(kInverse ? splitPos(m, nx) : m) * srcElem]);
        }
    }
    __syncthreads();
    // one (even, odd) output pair per thread: parity-free taps
    for (int p = threadIdx.x; p < kRowTile / 2; p += 256) {
        const int x = x0 + 2 * p;
        if (x >= nx) break;
        const float e = fir9c<kInverse, 0>(s + 2 * p), o = fir9c<kInverse, 1>(s + 2 * p + 1);
        const int oe = kInverse ? x : (x >> 1), oo = kInverse ? x + 1 : (nx >> 1) + (x >> 1);
        out[size_t(oe) * dstElem] = fromF<TOut>(e);
        out[size_t(oo) * dstElem] = fromF<TOut>(o);
    }
}

// ---------------------------------------------------------------------------
// Column pass (axis Y or Z).  Block 32 x 8 threads: 32 adjacent columns, 64
// outputs along the axis.  The loader maps (x, a, c) -> value, a = axis
// position (in the [L|H] layout for the inverse), c = the remaining coordinate.
// ---------------------------------------------------------------------------
constexpr int kColTile = 64;

struct PitchLoad {
    const float* p;
    int sx, sa, sc;   // strides for x, axis, other
    __device__ __forceinline__ float operator()(int x, int a, int c) const {
        return p[size_t(x) * sx + size_t(a) * sa + size_t(c) * sc];
    }
};

// Dequantizing loader of the first inverse pass of dwtFloat*InverseFromSymbols
// (DWTFloatFromSymbolsKernels.cui:18-464): the lowpass block comes from a
// float array with pitches, every other block from a symbol band (band index
// x+2y+4z-1, dense), dequantized as Quantize.cuh:104-110.
template <class Sym>
struct SymbolLoad {
    const float* lp;
    int lpRow, lpSlice;
    const Sym* const* bands;
    float step;
    int hx, hy, hz;     // half sizes
    bool axisIsZ;       // axis Z (3D) or Y (2D)
    __device__ __forceinline__ float operator()(int x, int a, int c) const {
        int y = axisIsZ ? c : a;
        int z = axisIsZ ? a : 0;
        int bx = x >= hx, by = y >= hy, bz = axisIsZ && z >= hz;
        int lx = x - bx * hx, ly = y - by * hy, lz = z - bz * hz;
        int b = bx + 2 * by + 4 * bz;
        if (b == 0) return lp[size_t(lz) * lpSlice + size_t(ly) * lpRow + lx];
        u32 sym = u32(bands[b - 1][(size_t(lz) * hy + ly) * hx + lx]);
        int neg = int(sym & 1u);
        int q = (1 - 2 * neg) * int((sym + u32(neg)) >> 1);
        float sg = q > 0 ? 1.0f : (q < 0 ? -1.0f : 0.0f);
        return (float(q) + sg * 0.5f) * step;
    }
};

template <class Load, bool kInverse>
__global__ void __launch_bounds__(256) k_firCols(float* __restrict__ dst, Load load, int nx, int na, int dx, int da,
                                                 int dc) {
    __shared__ float s[kColTile + 8][33];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int x = blockIdx.x * 32 + tx;
    const int a0 = blockIdx.y * kColTile;
    const int c = blockIdx.z;
    if (x < nx) {
        for (int k = ty; k < kColTile + 8; k += 8) {
            int j = a0 - 4 + k;
            if (j < na + 4) {
                int m = mirrorIdx(j, na);
                s[k][tx] = load(x, kInverse ? splitPos(m, na) : m, c);
            }
        }
    }
    __syncthreads();
    if (x >= nx) return;
    for (int k = ty; k < kColTile; k += 8) {
        int a = a0 + k;
        if (a >= na) break;
        float v[9];
#pragma unroll
        for (int i = 0; i < 9; ++i) v[i] = s[k + i][tx];
        float r = fir9<kInverse>(v, a & 1);
        int o = kInverse ? a : splitPos(a, na);
        dst[size_t(x) * dx + size_t(o) * da + size_t(c) * dc] = r;
    }
}

// ---------------------------------------------------------------------------
// Integer 5/3 lifting: same tiling; the tile keeps two extra samples each side.
// ---------------------------------------------------------------------------
__device__ __forceinline__ i16 div2(i16 v) { v = i16(v + ((v >= 0) ? 1 : -1)); return i16(v / 2); }
__device__ __forceinline__ i16 div4(i16 v) { v = i16(v + ((v >= 0) ? 2 : -2)); return i16(v / 4); }

// Lifts the samples in s[0 .. len) (s[k] <-> position base + k, positions
// outside [0, na) hold mirrored samples); forward: s holds natural samples;
// inverse: s holds the interleaved L/H signal.  A position is lifted when the
// sample it mirrors lies below liftEnd.  Positions whose neighbours are
// outside s are not valid afterwards.
template <bool kInverse>
__device__ __forceinline__ void liftLine(i16* s, int len, int base, int na, int liftEnd) {
    if (!kInverse) {
        for (int k = 1; k + 1 < len; ++k)
            if (((base + k) & 1) == 1 && mirrorIdx(base + k, na) < liftEnd)
                s[k] = i16(s[k] - div2(i16(s[k - 1] + s[k + 1])));
        for (int k = 2; k + 2 < len; ++k)
            if (((base + k) & 1) == 0 && mirrorIdx(base + k, na) < liftEnd)
                s[k] = i16(s[k] + div4(i16(s[k - 1] + s[k + 1])));
    } else {
        for (int k = 1; k + 1 < len; ++k)
            if (((base + k) & 1) == 0 && mirrorIdx(base + k, na) < liftEnd)
                s[k] = i16(s[k] - div4(i16(s[k - 1] + s[k + 1])));
        for (int k = 2; k + 2 < len; ++k)
            if (((base + k) & 1) == 1 && mirrorIdx(base + k, na) < liftEnd)
                s[k] = i16(s[k] + div2(i16(s[k - 1] + s[k + 1])));
    }
}

// DWTInt.cu:111-135 with DWTIntKernels.cui:104-200 (inverse DWTInt.cu:271-310,
// DWTIntKernels.cui:596-780): the reference's X pass lifts whole 256-sample
// blocks, then the remainder in 32-sample blocks of which its predict/update
// loops cover only whole pairs.  With an odd count of remainder blocks the
// last one is not lifted (its samples are only split into L and H); results
// stay identical to the reference by lifting only below this position.
static int intDwtXLiftEnd(int n) {
    const int done = n / 256 * 256, rest = n - done, blocks = (rest + 31) / 32;
    return std::min(n, done + 64 * (blocks / 2));
}

// Generic int lifting pass along one axis: block (32, 8): 32 adjacent lines of
// the fastest non-axis coordinate (x for Y/Z passes; for the X pass the lines
// are rows and the block covers 32 rows), kColTile outputs per line.
template <bool kInverse>
__global__ void __launch_bounds__(256) k_liftAxis(i16* __restrict__ dst, const i16* __restrict__ src, int nLines,
                                                  int na, int liftEnd, int sLine, int sAxis, int sOther, int dLine,
                                                  int dAxis, int dOther) {
    __shared__ i16 s[32][kColTile + 8];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int line = blockIdx.x * 32 + tx;
    const int a0 = blockIdx.y * kColTile;
    const int c = blockIdx.z;
    // stage positions a0-4 .. a0+kColTile+3
    if (line < nLines) {
        for (int k = ty; k < kColTile + 8; k += 8) {
            int j = a0 - 4 + k;
            if (j < na + 4) {
                int m = mirrorIdx(j, na);
                int ap = kInverse ? splitPos(m, na) : m;
                s[tx][k] = src[size_t(line) * sLine + size_t(ap) * sAxis + size_t(c) * sOther];
            }
        }
    }
    __syncthreads();
    if (line >= nLines) return;
    if (ty == 0) {
        int len = min(kColTile + 8, na + 4 - (a0 - 4));
        liftLine<kInverse>(s[tx], len, a0 - 4, na, liftEnd);
    }
    __syncthreads();
    for (int k = ty; k < kColTile; k += 8) {
        int a = a0 + k;
        if (a >= na) break;
        int o = kInverse ? a : splitPos(a, na);
        dst[size_t(line) * dLine + size_t(o) * dAxis + size_t(c) * dOther] = s[tx][k + 4];
    }
}

// ---------------------------------------------------------------------------
// Host-side pass launchers.
// ---------------------------------------------------------------------------
template <class TIn, class TOut, bool kInverse>
static void rowPass(TOut* dst, const TIn* src, int nx, int ny, int nz, int srcElem, int srcRow, int srcSlice,
                    int dstElem, int dstRow, int dstSlice, cudaStream_t st) {
    dim3 g(unsigned(ceilDiv(nx, kRowTile)), ny, nz);
    k_firRows<TIn, TOut, kInverse><<<g, 256, 0, st>>>(dst, src, nx, srcElem, srcRow, srcSlice, dstElem, dstRow, dstSlice); countLaunch();
}

// axis 1 (Y, other = Z) or 2 (Z, other = Y)
template <bool kInverse, class Load>
static void colPass(float* dst, Load load, int nx, int ny, int nz, int axis, int dstRow, int dstSlice, cudaStream_t st) {
    int na = axis == 1 ? ny : nz;
    int nc = axis == 1 ? nz : ny;
    dim3 g(unsigned(ceilDiv(nx, 32)), unsigned(ceilDiv(na, kColTile)), nc);
    int da = axis == 1 ? dstRow : dstSlice;
    int dc = axis == 1 ? dstSlice : dstRow;
    k_firCols<Load, kInverse><<<g, dim3(32, 8), 0, st>>>(dst, load, nx, na, 1, da, dc); countLaunch();
}

static PitchLoad pitchLoad(const float* p, int axis, int row, int slice) {
    PitchLoad l;
    l.p = p;
    l.sx = 1;
    l.sa = axis == 1 ? row : slice;
    l.sc = axis == 1 ? slice : row;
    return l;
}

template <bool kInverse>
static void liftPass(i16* dst, const i16* src, int nx, int ny, int nz, int axis, int srcRow, int srcSlice, int dstRow,
                     int dstSlice, cudaStream_t st) {
    // lines: X pass -> rows indexed by y (other = z); Y pass -> x (other = z); Z pass -> x (other = y)
    int nLines, na, nc, sLine, sAxis, sOther, dLine, dAxis, dOther;
    if (axis == 0) {
        nLines = ny; na = nx; nc = nz;
        sLine = srcRow; sAxis = 1; sOther = srcSlice;
        dLine = dstRow; dAxis = 1; dOther = dstSlice;
    } else if (axis == 1) {
        nLines = nx; na = ny; nc = nz;
        sLine = 1; sAxis = srcRow; sOther = srcSlice;
        dLine = 1; dAxis = dstRow; dOther = dstSlice;
    } else {
        nLines = nx; na = nz; nc = ny;
        sLine = 1; sAxis = srcSlice; sOther = srcRow;
        dLine = 1; dAxis = dstSlice; dOther = dstRow;
    }
    dim3 g(unsigned(ceilDiv(nLines, 32)), unsigned(ceilDiv(na, kColTile)), nc);
    const int liftEnd = axis == 0 ? intDwtXLiftEnd(na) : na;
    k_liftAxis<kInverse><<<g, dim3(32, 8), 0, st>>>(dst, src, nLines, na, liftEnd, sLine, sAxis, sOther, dLine, dAxis,
                                                    dOther);
    countLaunch();
}

static bool checkSizes(int sx, int sy, int sz, const char* what) {
    bool ok = sx >= 8 && sy >= 8 && sz >= 1 && (sx % 2 == 0) && (sy % 2 == 0) && (sz == 1 || (sz >= 8 && sz % 2 == 0));
    if (!ok) setError("%s: sizes must be even and >= 8 (got %d x %d x %d)", what, sx, sy, sz);
    return ok;
}

// ---------------------------------------------------------------------------
// Float transforms of every element type (DWTFloat.cu:465-533): float or byte
// source (byte b -> b - 128, DWTCommon.cuh:14-27) and float or byte
// destination (v -> clamp(v + 128.5, 0, 255) truncated, DWTCommon.cuh:29-41).
// The byte side carries the interleaved channels; intermediates are float.
// ---------------------------------------------------------------------------
template <class TIn>
static int floatForward(float* dst, float* buf2, float* buf1, const TIn* src, int sx, int sy, int sz, int ch,
                        int dstRow, int dstSlice, int srcRow, int srcSlice, cudaStream_t st, const char* what) {
    if (!checkSizes(sx, sy, sz, what)) return CC_ERR_INVALID_ARGUMENT;
    if (ch < 1 || ch > 4) { setError("channel count must be 1..4"); return CC_ERR_INVALID_ARGUMENT; }
    if (dstRow <= 0) dstRow = sx;
    if (dstSlice <= 0) dstSlice = sy * dstRow;
    if (srcRow <= 0) srcRow = sx * ch;
    if (srcSlice <= 0) srcSlice = sy * srcRow;
    const bool do3D = sz > 1;
    rowPass<TIn, float, false>(buf1, src, sx, sy, sz, ch, srcRow, srcSlice, 1, dstRow, dstSlice, st);
    float* yDst = do3D ? buf2 : dst;
    colPass<false>(yDst, pitchLoad(buf1, 1, dstRow, dstSlice), sx, sy, sz, 1, dstRow, dstSlice, st);
    if (do3D) colPass<false>(dst, pitchLoad(buf2, 2, dstRow, dstSlice), sx, sy, sz, 2, dstRow, dstSlice, st);
    CC_TRY_CUDA(cudaGetLastError(), what);
    return CC_OK;
}

template <class TOut>
static int floatInverse(TOut* dst, float* buf2, float* buf1, const float* src, int sx, int sy, int sz, int ch,
                        int dstRow, int dstSlice, int srcRow, int srcSlice, cudaStream_t st, const char* what) {
    if (!checkSizes(sx, sy, sz, what)) return CC_ERR_INVALID_ARGUMENT;
    if (ch < 1 || ch > 4) { setError("channel count must be 1..4"); return CC_ERR_INVALID_ARGUMENT; }
    if (dstRow <= 0) dstRow = sx * ch;
    if (dstSlice <= 0) dstSlice = sy * dstRow;
    if (srcRow <= 0) srcRow = sx;
    if (srcSlice <= 0) srcSlice = sy * srcRow;
    const bool do3D = sz > 1;
    const float* ySrc = src;
    if (do3D) {
        colPass<true>(buf2, pitchLoad(src, 2, srcRow, srcSlice), sx, sy, sz, 2, srcRow, srcSlice, st);
        ySrc = buf2;
    }
    colPass<true>(buf1, pitchLoad(ySrc, 1, srcRow, srcSlice), sx, sy, sz, 1, srcRow, srcSlice, st);
    rowPass<float, TOut, true>(dst, buf1, sx, sy, sz, 1, srcRow, srcSlice, ch, dstRow, dstSlice, st);
    CC_TRY_CUDA(cudaGetLastError(), what);
    return CC_OK;
}

template <class TOut>
static int floatInverseFromSymbols(TOut* dst, float* buf2, float* buf1, const float* lowpass,
                                   const void* const* highpass, int symBytes, float step, int sx, int sy, int sz,
                                   int ch, int dstRow, int dstSlice, int lpRow, int lpSlice, cudaStream_t st,
                                   const char* what) {
    if (!checkSizes(sx, sy, sz, what)) return CC_ERR_INVALID_ARGUMENT;
    if (ch < 1 || ch > 4) { setError("channel count must be 1..4"); return CC_ERR_INVALID_ARGUMENT; }
    if (symBytes != 2 && symBytes != 4) { setError("symbol size must be 2 or 4"); return CC_ERR_INVALID_ARGUMENT; }
    if (dstRow <= 0) dstRow = sx * ch;
    if (dstSlice <= 0) dstSlice = sy * dstRow;
    if (lpRow <= 0) lpRow = sx;
    if (lpSlice <= 0) lpSlice = sy * lpRow;
    const bool do3D = sz > 1;
    const int bRow = sx, bSlice = sx * sy;   // DWTFloat.cu:354-355: tight intermediates
    auto first = [&](auto tag, float* out, int axis) {
        using Sym = decltype(tag);
        SymbolLoad<Sym> l;
        l.lp = lowpass;
        l.lpRow = lpRow;
        l.lpSlice = lpSlice;
        l.bands = reinterpret_cast<const Sym* const*>(highpass);
        l.step = step;
        l.hx = sx / 2;
        l.hy = sy / 2;
        l.hz = do3D ? sz / 2 : 1;
        l.axisIsZ = axis == 2;
        colPass<true>(out, l, sx, sy, sz, axis, bRow, bSlice, st);
    };
    if (do3D) {
        if (symBytes == 2) first(u16(), buf2, 2); else first(u32(), buf2, 2);
        colPass<true>(buf1, pitchLoad(buf2, 1, bRow, bSlice), sx, sy, sz, 1, bRow, bSlice, st);
    } else {
        if (symBytes == 2) first(u16(), buf1, 1); else first(u32(), buf1, 1);
    }
    rowPass<float, TOut, true>(dst, buf1, sx, sy, sz, 1, bRow, bSlice, ch, dstRow, dstSlice, st);
    CC_TRY_CUDA(cudaGetLastError(), what);
    return CC_OK;
}

// ---------------------------------------------------------------------------
// Lowpass-only forward transforms: the LL band of one 2D level and nothing
// else, in ONE kernel (the reference runs an X and a Y kernel through a
// buffer).  A CTA owns 32 x 32 LL outputs: it stages the (mirrored) source
// window they depend on, filters its rows along X into shared memory (the
// even outputs only), then the columns of that along Y.  Each LL sample is
// the same arithmetic as the reference's two passes, so results are
// bit-identical.
// ---------------------------------------------------------------------------
constexpr int kLpTile = 32;

// CDF 9/7 (DWTFloat2DLowpassKernels.cui:14-300): window 2L-4 .. 2L+4 per axis.
// Channel blockIdx.z of interleaved source / destination elements (element
// strides srcElem / dstElem, in elements of their type).
template <class TIn, class TOut>
__global__ void __launch_bounds__(256) k_lowpass97(TOut* __restrict__ dst, const TIn* __restrict__ src, int nx, int ny,
                                                   int srcElem, int srcRow, int dstElem, int dstRow) {
    src += blockIdx.z;
    dst += blockIdx.z;
    constexpr int kIn = 2 * kLpTile + 7;
    __shared__ float sIn[kIn][kIn + 1];
    __shared__ float sX[kIn][kLpTile + 1];
    const int lx0 = blockIdx.x * kLpTile, ly0 = blockIdx.y * kLpTile;
    const int x0 = 2 * lx0 - 4, y0 = 2 * ly0 - 4;
    // samples at or beyond n + 4 feed no output of this tile
    const int rows = min(kIn, ny + 4 - y0), cols = min(kIn, nx + 4 - x0);
    for (int k = threadIdx.x; k < rows * kIn; k += 256) {
        const int j = k / kIn, i = k - j * kIn;
        if (i < cols)
            sIn[j][i] = toF<TIn>(src[size_t(mirrorIdx(y0 + j, ny)) * srcRow + size_t(mirrorIdx(x0 + i, nx)) * srcElem]);
    }
    __syncthreads();
    const int ox = min(kLpTile, (nx >> 1) - lx0), oy = min(kLpTile, (ny >> 1) - ly0);
    for (int k = threadIdx.x; k < rows * ox; k += 256) {
        const int j = k / ox, c = k - j * ox;
        sX[j][c] = fir9c<false, 0>(&sIn[j][2 * c]);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < oy * ox; k += 256) {
        const int r = k / ox, c = k - r * ox;
        float v[9];
#pragma unroll
        for (int i = 0; i < 9; ++i) v[i] = sX[2 * r + i][c];
        dst[(size_t(ly0 + r) * dstRow + lx0 + c) * dstElem] = fromF<TOut>(fir9c<false, 0>(v));
    }
}

// CDF 5/3 lifting (DWTInt2DLowpassKernels.cui:14-196): the even sample 2L
// updated by its two predicted odd neighbours, window 2L-2 .. 2L+2.
__device__ __forceinline__ i16 lowpass53(i16 a, i16 b, i16 c, i16 d, i16 e) {
    const i16 d1 = i16(b - div2(i16(a + c)));
    const i16 d3 = i16(d - div2(i16(c + e)));
    return i16(c + div4(i16(d1 + d3)));
}

// kRemoveLsb: each LL sample v is stored as (t + (t < 0 ? -1 : 0)) / 2 with
// t = v + shift in 16 bits (removeLSB without bits, Bits.cu:62-96).
template <bool kRemoveLsb>
__global__ void __launch_bounds__(256) k_lowpass53(i16* __restrict__ dst, const i16* __restrict__ src, int nx, int ny,
                                                   int srcRow, int dstRow, i16 shift) {
    constexpr int kIn = 2 * kLpTile + 3;
    __shared__ i16 sIn[kIn][kIn + 1];
    __shared__ i16 sX[kIn][kLpTile + 1];
    const int lx0 = blockIdx.x * kLpTile, ly0 = blockIdx.y * kLpTile;
    const int x0 = 2 * lx0 - 2, y0 = 2 * ly0 - 2;
    const int rows = min(kIn, ny + 2 - y0), cols = min(kIn, nx + 2 - x0);
    for (int k = threadIdx.x; k < rows * kIn; k += 256) {
        const int j = k / kIn, i = k - j * kIn;
        if (i < cols) sIn[j][i] = src[size_t(mirrorIdx(y0 + j, ny)) * srcRow + mirrorIdx(x0 + i, nx)];
    }
    __syncthreads();
    const int ox = min(kLpTile, (nx >> 1) - lx0), oy = min(kLpTile, (ny >> 1) - ly0);
    for (int k = threadIdx.x; k < rows * ox; k += 256) {
        const int j = k / ox, c = k - j * ox;
        const i16* s = &sIn[j][2 * c];
        sX[j][c] = lowpass53(s[0], s[1], s[2], s[3], s[4]);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < oy * ox; k += 256) {
        const int r = k / ox, c = k - r * ox;
        i16 v = lowpass53(sX[2 * r][c], sX[2 * r + 1][c], sX[2 * r + 2][c], sX[2 * r + 3][c], sX[2 * r + 4][c]);
        if (kRemoveLsb) {
            const i16 t = i16(v + shift);
            v = i16((int(t) + (t < 0 ? -1 : 0)) / 2);
        }
        dst[size_t(ly0 + r) * dstRow + lx0 + c] = v;
    }
}

// ---------------------------------------------------------------------------
// Fixed scratch of cc_dwt_float_forward_static: the two intermediate volumes
// of the forward transform live in this file-scope device array instead of
// caller buffers, for callers that cannot allocate device memory (code that
// runs while a host allocator lock is held, inside a stream capture, or under
// a host application that owns the device's memory pool).  Every GPU that
// loads the library holds these 8 MiB until the process exits.
// ---------------------------------------------------------------------------
constexpr u64 kStaticScratchFloats = u64(1) << 20;   // per intermediate volume (4 MiB)
static __device__ __align__(256) float g_dwtScratch[2 * kStaticScratchFloats];

// Device address of g_dwtScratch per device, resolved once with that device
// current (a host reference to g_dwtScratch is a host-side stand-in, not a
// device address).
constexpr int kMaxDevices = 64;
static float* g_dwtScratchDev[kMaxDevices] = {};

static int dwtScratchFor(int device, float** out) {
    if (device < 0 || device >= kMaxDevices) { setError("dwtFloatForwardStatic: device %d out of range", device); return CC_ERR_INVALID_ARGUMENT; }
    float* p = __atomic_load_n(&g_dwtScratchDev[device], __ATOMIC_ACQUIRE);
    if (!p) {
        void* addr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&addr, g_dwtScratch);
        if (e != cudaSuccess) return cudaFail(e, "dwtFloatForwardStatic: cudaGetSymbolAddress");
        p = static_cast<float*>(addr);
        __atomic_store_n(&g_dwtScratchDev[device], p, __ATOMIC_RELEASE);
    }
    *out = p;
    return CC_OK;
}

// ---------------------------------------------------------------------------
// Batched passes (batch.cuh): the same arithmetic as k_firRows / k_firCols /
// k_quantize, over all volumes of a batch in one launch.  A CTA reads its
// descriptor index from the launch's CTA map (one load) and the descriptor.
// ---------------------------------------------------------------------------
// floor(k / d) for 0 <= k < 2^22 and 1 <= d < 2^13 from r = 1/d rounded to
// nearest: (k + 1/2) / d lies at least 1/(2d) from an integer, and the two
// roundings move it by at most (k/d) 2^-23 < 1/(2d).
__device__ __forceinline__ int quotient(int k, float r) {
    return int(__float2uint_rz((float(k) + 0.5f) * r));
}

template <bool kInverse>
__device__ __forceinline__ void rowPairs4(const float* w, float4& a, float4& b) {
    // four (even, odd) output pairs from the 16-sample window w[0..15]: pair
    // p is one packed chain, lane x the even output over w[2p .. 2p+8], lane y
    // the odd one over w[2p+1 .. 2p+9] (tap i: coefficients (even_i, odd_i),
    // samples (w[2p+i], w[2p+i+1])), each lane rounded as fir9c's chain
    constexpr float kF[2][9] = {
        {0.0267488f, -0.0168641f, -0.0782233f, 0.2668641f, 0.6029490f, 0.2668641f, -0.0782233f, -0.0168641f, 0.0267488f},
        {0.0f, 0.0456359f, -0.0287718f, -0.2956359f, 0.5575435f, -0.2956359f, -0.0287718f, 0.0456359f, 0.0f}};
    constexpr float kI[2][9] = {
        {0.0f, 0.0337282f, -0.0575435f, -0.5337281f, 1.1150871f, -0.5337281f, -0.0575435f, 0.0337282f, 0.0f},
        {0.0534975f, -0.0912718f, -0.1564465f, 0.5912718f, 1.2058980f, 0.5912718f, -0.1564465f, -0.0912718f, 0.0534975f}};
    float2 r[4];
#pragma unroll
    for (int p = 0; p < 4; ++p) r[p] = make_float2(0.0f, 0.0f);
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        const float2 c = kInverse ? make_float2(kI[0][i], kI[1][i]) : make_float2(kF[0][i], kF[1][i]);
#pragma unroll
        for (int p = 0; p < 4; ++p) r[p] = __ffma2_rn(c, make_float2(w[2 * p + i], w[2 * p + i + 1]), r[p]);
    }
    if (kInverse) {
        a = make_float4(r[0].x, r[0].y, r[1].x, r[1].y);
        b = make_float4(r[2].x, r[2].y, r[3].x, r[3].y);
    } else {
        a = make_float4(r[0].x, r[1].x, r[2].x, r[3].x);
        b = make_float4(r[0].y, r[1].y, r[2].y, r[3].y);
    }
}

// Row (X) pass.  A CTA transforms R rows of one W-wide tile of a row
// (R * W <= kBRowOutputs): the rows and their 4-sample mirrored halos are
// staged in shared memory, then every thread computes output pairs.  Fast
// path (descriptor flag `vec` and 16-byte aligned pointers): float4 loads of
// the tile body - the inverse reads the low and high halves separately and
// interleaves them on the way into shared memory - and float4 stores of four
// pairs per thread.  Otherwise scalar loads and stores.  The inverse, whose
// packed chains fit 32 registers, runs eight CTAs per SM (the forward six).
template <bool kInverse>
__global__ void __launch_bounds__(256, kInverse ? 8 : 6) k_bRows(const BRowDesc* __restrict__ descs, const u32* __restrict__ map,
                                               const float* const* inTab, float* const* outTab) {
    __shared__ __align__(16) float s[kBRowSmem];
    const BRowDesc D = descs[map[blockIdx.x]];
    const float* src = D.src ? D.src : inTab[D.vol];
    float* dst = D.dst ? D.dst : outTab[D.vol];
    const u32 local = blockIdx.x - D.ctaOff;
    const int xt = int(local % u32(D.tilesX)), rg = int(local / u32(D.tilesX));
    const int nx = D.nx, hn = nx >> 1;
    const int x0 = xt * D.W, Wt = min(D.W, nx - x0), Wp = Wt + 8;
    const int rows = D.ny * D.nz, r0 = rg * D.R, R = min(D.R, rows - r0);
    // row j of the tile: (y0 + j, z0) carried over slices (R <= 128 rows, so
    // at most one carry when ny >= 128)
    const int z0 = r0 / D.ny, y0 = r0 - z0 * D.ny;
    auto rowYZ = [&](int j, int& y, int& z) {
        y = y0 + j;
        z = z0;
        while (y >= D.ny) { y -= D.ny; ++z; }
    };
    auto srcRow = [&](int j) {
        int y, z;
        rowYZ(j, y, z);
        return src + size_t(z) * D.srcSlice + size_t(y) * D.srcRow;
    };
    auto dstRow = [&](int j) {
        int y, z;
        rowYZ(j, y, z);
        return dst + size_t(z) * D.dstSlice + size_t(y) * D.dstRow;
    };
    const int tid = threadIdx.x;
    const bool vec = D.vec && ((reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(dst)) & 15) == 0;
    if (vec) {
        // body: forward U = Wt/4 float4 per row; inverse U = Wt/8 (low, high) float4 pairs per row
        constexpr int kBody = kBRowOutputs / 1024;   // float4 loads per thread
        float4 body[kBody];
        float halo[kBody];
        const int U = kInverse ? Wt >> 3 : Wt >> 2;
        const float rU = __frcp_rn(float(U));
#pragma unroll
        for (int i = 0; i < kBody; ++i) {
            const int k = tid + 256 * (kInverse ? (i >> 1) : i);
            body[i] = make_float4(0.f, 0.f, 0.f, 0.f);
            if (k < R * U) {
                const int j = quotient(k, rU), q = k - j * U;
                const float* row = srcRow(j);
                if (kInverse) body[i] = *reinterpret_cast<const float4*>(row + (i & 1) * hn + (x0 >> 1) + 4 * q);
                else body[i] = *reinterpret_cast<const float4*>(row + x0 + 4 * q);
            }
        }
#pragma unroll
        for (int i = 0; i < kBody; ++i) {
            const int k = tid + 256 * i;
            halo[i] = 0.0f;
            if (k < R * 8) {
                const int j = k >> 3, h = k & 7;
                const int m = mirrorIdx(h < 4 ? x0 - 4 + h : x0 + Wt + h - 4, nx);
                halo[i] = srcRow(j)[kInverse ? splitPos(m, nx) : m];
            }
        }
#pragma unroll
        for (int i = 0; i < kBody; ++i) {
            const int k = tid + 256 * (kInverse ? (i >> 1) : i);
            if (k < R * U) {
                const int j = quotient(k, rU), q = k - j * U;
                if (kInverse) {
                    if (i & 1) {
                        const float4 l = body[i - 1], h = body[i];
                        float4* o = reinterpret_cast<float4*>(s + j * Wp + 4 + 8 * q);
                        o[0] = make_float4(l.x, h.x, l.y, h.y);
                        o[1] = make_float4(l.z, h.z, l.w, h.w);
                    }
                } else {
                    *reinterpret_cast<float4*>(s + j * Wp + 4 + 4 * q) = body[i];
                }
            }
            if (tid + 256 * i < R * 8) {
                const int k2 = tid + 256 * i, j = k2 >> 3, h = k2 & 7;
                s[j * Wp + (h < 4 ? h : Wt + h)] = halo[i];
            }
        }
        __syncthreads();
        // outputs: four pairs per thread-step
        const int Q = Wt >> 3;
        const float rQ = __frcp_rn(float(Q));
#pragma unroll
        for (int i = 0; i < kBRowOutputs / 2048; ++i) {
            const int k = tid + 256 * i;
            if (k < R * Q) {
                const int j = quotient(k, rQ), q = k - j * Q;
                const float* w4 = s + j * Wp + 8 * q;
                float w[16];
#pragma unroll
                for (int t = 0; t < 4; ++t) {
                    const float4 v = *reinterpret_cast<const float4*>(w4 + 4 * t);
                    w[4 * t] = v.x; w[4 * t + 1] = v.y; w[4 * t + 2] = v.z; w[4 * t + 3] = v.w;
                }
                float4 a, b;
                rowPairs4<kInverse>(w, a, b);
                float* row = dstRow(j);
                if (kInverse) {
                    float4* o = reinterpret_cast<float4*>(row + x0 + 8 * q);
                    o[0] = a;
                    o[1] = b;
                } else {
                    *reinterpret_cast<float4*>(row + (x0 >> 1) + 4 * q) = a;
                    *reinterpret_cast<float4*>(row + hn + (x0 >> 1) + 4 * q) = b;
                }
            }
        }
        return;
    }
    // scalar path: positions x0-4 .. x0+Wt+3 of each row, 8 loads in flight per thread
    const int total = R * Wp;
    for (int base = 0; base < total; base += 256 * 8) {
        float v[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int k = base + tid + 256 * i;
            v[i] = 0.0f;
            if (k < total) {
                const int j = k / Wp, kk = k - j * Wp;
                const int m = mirrorIdx(x0 - 4 + kk, nx);
                v[i] = srcRow(j)[kInverse ? splitPos(m, nx) : m];
            }
        }
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int k = base + tid + 256 * i;
            if (k < total) s[k] = v[i];
        }
    }
    __syncthreads();
    const int P = Wt >> 1;
    for (int k = tid; k < R * P; k += 256) {
        const int j = k / P, p = k - j * P, x = x0 + 2 * p;
        const float* w = s + j * Wp + 2 * p;
        const float e = fir9c<kInverse, 0>(w), o = fir9c<kInverse, 1>(w + 1);
        float* row = dstRow(j);
        if (kInverse) {
            row[x] = e;
            row[x + 1] = o;
        } else {
            row[x >> 1] = e;
            row[hn + (x >> 1)] = o;
        }
    }
}

// One sample of the first inverse pass of dwtFloat3DInverseFromSymbols:
// (x, y, z) in the level's interleaved-band layout; the lowpass octant comes
// from src, the other seven from dequantized symbol bands
// (DWTFloatFromSymbolsKernels.cui:18-464).
__device__ __forceinline__ float bandSample(const BColDesc& D, int x, int y, int z) {
    const int bx = x >= D.hx, by = y >= D.hy, bz = z >= D.hz;
    const int lx = x - bx * D.hx, ly = y - by * D.hy, lz = z - bz * D.hz;
    const int b = bx + 2 * by + 4 * bz;
    if (b == 0) return D.src[size_t(lz) * D.lpSlice + size_t(ly) * D.lpRow + lx];
    const u32 sym = D.bands[u64(b - 1) * D.bandStride + (u64(lz) * D.hy + ly) * D.hx + lx];
    const int q = unsymbolizeI(sym);
    return (float(q) + signI(q) * 0.5f) * D.step;   // Quantize.cuh:104-110
}

// (float(q) + sign(q) * 0.5f) * step for q = unsymbolize(s), the dequantizer
// of Quantize.cuh:104-110, without the sign selects: float(q) +- 1/2 is
// exactly float(m) / 2 with m = 0, s + 1 or -(s + 2) for s zero, even or
// odd (|m| < 2^24), so the one rounding, the product with step, is the same.
__device__ __forceinline__ float dequantSym(u32 s, float step) {
    const int m = s == 0u ? 0 : ((s & 1u) ? -int(s + 2u) : int(s + 1u));
    return (float(m) * 0.5f) * step;
}

// The samples (x, x + 1), x even, of that pass.  With an even half width hx
// both lie in one band at an even offset: one 4-byte symbol pair, or one
// float2 of the lowpass (all pitches even, bases 16-byte aligned).
__device__ __forceinline__ float2 bandPair(const BColDesc& D, int x, int y, int z) {
    if (D.hx & 1) return make_float2(bandSample(D, x, y, z), bandSample(D, x + 1, y, z));
    const int bx = x >= D.hx, by = y >= D.hy, bz = z >= D.hz;
    const int lx = x - bx * D.hx, ly = y - by * D.hy, lz = z - bz * D.hz;
    const int b = bx + 2 * by + 4 * bz;
    if (b == 0) return *reinterpret_cast<const float2*>(D.src + size_t(lz) * D.lpSlice + size_t(ly) * D.lpRow + lx);
    const u32 pair =
        *reinterpret_cast<const u32*>(D.bands + u64(b - 1) * D.bandStride + (u64(lz) * D.hy + ly) * D.hx + lx);
    const int q0 = unsymbolizeI(pair & 0xFFFFu), q1 = unsymbolizeI(pair >> 16);
    return make_float2((float(q0) + signI(q0) * 0.5f) * D.step, (float(q1) + signI(q1) * 0.5f) * D.step);
}

// One sample of the fused store (see BColDesc::symOut): (x, y, z) in the
// level's [L|H] layout.  Deadzone quantization as k_bQuant's
// (Quantize.cuh:55-59, reciprocal from the host).
__device__ __forceinline__ void quantStoreOne(const BColDesc& D, int x, int y, int z, float v) {
    const int bx = x >= D.hx, by = y >= D.hy, bz = z >= D.hz;
    const int b = bx + 2 * by + 4 * bz;
    if (b == 0 && !D.lastLevel) {
        D.dst[size_t(x) + size_t(z) * D.da + size_t(y) * D.dc] = v;
        return;
    }
    const int lx = x - bx * D.hx, ly = y - by * D.hy, lz = z - bz * D.hz;
    u16* base = b == 0 ? D.lpSymOut : D.symOut + u64(b - 1) * D.bandStride;
    base[(u64(lz) * D.hy + ly) * D.hx + lx] = u16(symbolizeI(int(v * (b == 0 ? D.invLP : D.inv))));
}

// The samples (x, x + 1), x even; with an even half width both lie in one
// octant at an even offset (one float2 or one 4-byte symbol pair).
__device__ __forceinline__ void quantStorePair(const BColDesc& D, int x, int y, int z, float2 v) {
    if (D.hx & 1) {
        quantStoreOne(D, x, y, z, v.x);
        quantStoreOne(D, x + 1, y, z, v.y);
        return;
    }
    const int bx = x >= D.hx, by = y >= D.hy, bz = z >= D.hz;
    const int b = bx + 2 * by + 4 * bz;
    if (b == 0 && !D.lastLevel) {
        *reinterpret_cast<float2*>(D.dst + size_t(x) + size_t(z) * D.da + size_t(y) * D.dc) = v;
        return;
    }
    const int lx = x - bx * D.hx, ly = y - by * D.hy, lz = z - bz * D.hz;
    u16* base = b == 0 ? D.lpSymOut : D.symOut + u64(b - 1) * D.bandStride;
    const float inv = b == 0 ? D.invLP : D.inv;
    const u32 s0 = symbolizeI(int(v.x * inv)) & 0xFFFFu, s1 = symbolizeI(int(v.y * inv)) & 0xFFFFu;
    *reinterpret_cast<u32*>(base + (u64(lz) * D.hy + ly) * D.hx + lx) = s0 | (s1 << 16);
}

// Eight consecutive outputs of a column pair per thread: the 16 staged
// samples they use are read from shared memory once into registers (a
// sliding window) instead of nine reads per output.  The tile's first row
// is even, so output j has parity j & 1 and its taps are immediates.
template <bool kInverse, bool kQuantize = false, bool kPacked = false>
__device__ __forceinline__ void colOutputs8(const BColDesc& D, const float2 (*s)[33], int tx, int ty, int x, int c,
                                            int a0) {
    static_assert(kBColTileA == 64, "eight outputs per thread row of an 8-row block");
    const int k0 = 8 * ty;
    if (a0 + k0 >= D.na) return;
    float2 w[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) w[i] = s[k0 + i][tx];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int a = a0 + k0 + j;
        if (a >= D.na) break;
        float2 r;
        if (kPacked) {
            // both columns' chains in one packed fma.rn.f32x2 each tap
            r = (j & 1) ? fir9p<kInverse, 1>(w + j) : fir9p<kInverse, 0>(w + j);
        } else {
            // two scalar chains: the passes held to 40 registers (six CTAs
            // per SM) keep the window in registers this way without spills
            float v0[9], v1[9];
#pragma unroll
            for (int i = 0; i < 9; ++i) {
                v0[i] = w[j + i].x;
                v1[i] = w[j + i].y;
            }
            r = (j & 1) ? make_float2(fir9c<kInverse, 1>(v0), fir9c<kInverse, 1>(v1))
                        : make_float2(fir9c<kInverse, 0>(v0), fir9c<kInverse, 0>(v1));
        }
        const int o = kInverse ? a : splitPos(a, D.na);
        if (kQuantize) quantStorePair(D, x, c, o, r);   // axis Z: a = z, c = y
        else *reinterpret_cast<float2*>(D.dst + size_t(x) + size_t(o) * D.da + size_t(c) * D.dc) = r;
    }
}

// The same outputs with the quantizer fused into the store (axis Z, a = z,
// c = y), for an even half width hx and hz = na / 2: the thread's x and y fix
// its octant up to bz, and output a lands in octant bz = a & 1 at lz = a >> 1
// (a's split position is a / 2 or hz + a / 2), so every store goes to one of
// two per-thread bases.  Symbols as quantStorePair computes them.
__device__ __forceinline__ void colOutputs8Quantize(const BColDesc& D, const float2 (*s)[33], int tx, int ty, int x,
                                                    int c, int a0) {
    const int k0 = 8 * ty;
    if (a0 + k0 >= D.na) return;
    float2 w[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) w[i] = s[k0 + i][tx];
    const int bx = x >= D.hx, by = c >= D.hy;
    const int lx = x - bx * D.hx, ly = c - by * D.hy, be = bx + 2 * by;
    const u64 slice = u64(D.hy) * D.hx, inPlane = u64(ly) * D.hx + lx;
    u16* const oddBase = D.symOut + u64(be + 3) * D.bandStride + inPlane;        // octant be + 4
    u16* const evenSym = be ? D.symOut + u64(be - 1) * D.bandStride + inPlane     // octant be
                            : D.lpSymOut + inPlane;                               // LLL, coarsest level
    const bool evenFloat = be == 0 && !D.lastLevel;                              // LLL kept as floats
    float* const evenF = D.dst + size_t(x) + size_t(c) * D.dc;
    const float invEven = be ? D.inv : D.invLP;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int a = a0 + k0 + j;
        if (a >= D.na) break;
        const float2 r = (j & 1) ? fir9p<false, 1>(w + j) : fir9p<false, 0>(w + j);
        const u64 lz = u64(a >> 1);
        if (j & 1) {
            const u32 s0 = symbolizeI(int(r.x * D.inv)) & 0xFFFFu, s1 = symbolizeI(int(r.y * D.inv)) & 0xFFFFu;
            *reinterpret_cast<u32*>(oddBase + lz * slice) = s0 | (s1 << 16);
        } else if (evenFloat) {
            *reinterpret_cast<float2*>(evenF + size_t(a >> 1) * D.da) = r;
        } else {
            const u32 s0 = symbolizeI(int(r.x * invEven)) & 0xFFFFu, s1 = symbolizeI(int(r.y * invEven)) & 0xFFFFu;
            *reinterpret_cast<u32*>(evenSym + lz * slice) = s0 | (s1 << 16);
        }
    }
}

// Y or Z pass: 64 x-columns (a column pair per thread, float2 accesses; all
// level extents are even and x is the unit-stride axis) by kBColTileA axis
// positions per CTA.  The CTA stages the tile's kBColTileA + 8 input rows in
// shared memory (nine loads in flight per thread; tiles away from both ends
// skip the mirroring), then every thread computes eight consecutive outputs
// (colOutputs8).  The descriptor is a register copy; the register bounds
// (six CTAs per SM for the plain passes and the one with the dequantizer -
// whose packed chains fit 40 registers - four with the quantizer) are the
// tightest that keep the 16-sample window in registers without spills.  The
// symbol pass's loads are 4-byte pairs, so its bytes in flight per SM are
// set by the CTAs resident.
static_assert(kBColTileX == 64, "a column-pass CTA has 32 threads of column pairs per row");

template <bool kInverse, bool kSymbols, bool kQuantize = false>
__global__ void __launch_bounds__(256, kQuantize ? 4 : 6) k_bCols(const BColDesc* __restrict__ descs, const u32* __restrict__ map) {
    __shared__ float2 s[kBColTileA + 8][33];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const BColDesc D = descs[map[blockIdx.x]];   // a copy: the output stores cannot alias it
    const u32 local = blockIdx.x - D.ctaOff;
    const u32 xt = local % D.tilesX, rest = local / D.tilesX;
    const int at = int(rest % D.tilesA), c = int(rest / D.tilesA);
    const int nx = D.nx, na = D.na;
    const int x = int(xt) * kBColTileX + 2 * tx;
    const int a0 = at * kBColTileA;
    // all of a thread's column loads are issued before any is used
    constexpr int kLoads = (kBColTileA + 8) / 8;
    float2 vals[kLoads];
    if (kSymbols && !(D.hx & 1) && 2 * D.hz == na) {
        // axis Z (a = z, c = y), even half width, hz = na / 2: the thread's
        // rows j = a0 - 4 + ty + 8i all have the parity of ty, and so have
        // their mirrored indices m, so all lie in octant bx + 2by + 4 (ty
        // odd) or bx + 2by (ty even), at lz = m >> 1.  Each load is one
        // float2 of the lowpass (octant 0) or one 4-byte symbol pair, issued
        // as predicated loads of raw bits; the dequantization follows once
        // all of them are in flight.
        const int bx = x >= D.hx, by = c >= D.hy;
        const int lx = x - bx * D.hx, ly = c - by * D.hy;
        const int b = bx + 2 * by + ((ty & 1) ? 4 : 0);
        const u64 slice = u64(D.hy) * D.hx;
        const u16* const band = D.bands + u64(b ? b - 1 : 0) * D.bandStride + u64(ly) * D.hx + lx;
        const float* const lpBase = D.src + size_t(ly) * D.lpRow + lx;
        uint2 raw[kLoads];
        auto loadRows = [&](auto position) {
#pragma unroll
            for (int i = 0; i < kLoads; ++i) {
                const int j = a0 - 4 + ty + 8 * i;
                raw[i] = make_uint2(0u, 0u);
                if (x < nx && j < na + 4) {
                    const int lz = position(j) >> 1;
                    if (b == 0) raw[i] = *reinterpret_cast<const uint2*>(lpBase + size_t(lz) * D.lpSlice);
                    else raw[i].x = *reinterpret_cast<const u32*>(band + u64(lz) * slice);
                }
            }
        };
        // tiles whose rows a0 - 4 .. a0 + kBColTileA + 3 all lie inside need no mirroring
        if (a0 >= 4 && a0 + kBColTileA + 4 <= na) loadRows([](int j) { return j; });
        else loadRows([na](int j) { return mirrorIdx(j, na); });
#pragma unroll
        for (int i = 0; i < kLoads; ++i) {
            if (b == 0) vals[i] = make_float2(__uint_as_float(raw[i].x), __uint_as_float(raw[i].y));
            else vals[i] = make_float2(dequantSym(raw[i].x & 0xFFFFu, D.step), dequantSym(raw[i].x >> 16, D.step));
        }
    } else {
        auto loadRows = [&](auto position) {
#pragma unroll
            for (int i = 0; i < kLoads; ++i) {
                const int j = a0 - 4 + ty + 8 * i;
                vals[i] = make_float2(0.0f, 0.0f);
                if (x < nx && j < na + 4) {
                    const int m = position(j);
                    const int a = kInverse ? splitPos(m, na) : m;
                    if (kSymbols) {
                        // axis Z: a = z, c = y
                        vals[i] = bandPair(D, x, c, a);
                    } else {
                        vals[i] = *reinterpret_cast<const float2*>(D.src + size_t(x) + size_t(a) * D.sa + size_t(c) * D.sc);
                    }
                }
            }
        };
        if (a0 >= 4 && a0 + kBColTileA + 4 <= na) loadRows([](int j) { return j; });
        else loadRows([na](int j) { return mirrorIdx(j, na); });
    }
#pragma unroll
    for (int i = 0; i < kLoads; ++i) s[ty + 8 * i][tx] = vals[i];
    __syncthreads();
    if (x >= nx) return;
    if (kQuantize && !(D.hx & 1) && 2 * D.hz == na) colOutputs8Quantize(D, s, tx, ty, x, c, a0);
    else colOutputs8<kInverse, kQuantize, kSymbols || kQuantize>(D, s, tx, ty, x, c, a0);
}

// Quantization of one band to u16 symbols (deadzone, Quantize.cuh:55-59), or
// dequantization of dense symbols (Quantize.cuh:104-110).  A CTA covers
// kBQuantPerCta elements of one band in groups of four consecutive elements;
// a group inside one row with 16-byte aligned source moves as one float4
// and one 8-byte symbol store.
template <bool kDequantize>
__global__ void __launch_bounds__(256) k_bQuant(const BQuantDesc* __restrict__ descs, const u32* __restrict__ map) {
    const BQuantDesc& D = descs[map[blockIdx.x]];
    const u32 nx = u32(D.nx), plane = nx * u32(D.ny), total = plane * u32(D.nz);
    const u32 e0 = (blockIdx.x - D.ctaOff) * u32(kBQuantPerCta);
    constexpr int kGroups = kBQuantPerCta / 1024;
    if (kDequantize) {
#pragma unroll
        for (int g = 0; g < kGroups; ++g) {
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                const u32 e = e0 + u32(g) * 1024u + u32(t) * 256u + threadIdx.x;
                if (e < total) {
                    const int q = unsymbolizeI(u32(D.sym[e]));
                    D.dstF[e] = (float(q) + signI(q) * 0.5f) * D.step;
                }
            }
        }
        return;
    }
    const bool vec = (nx & 3) == 0 && ((D.row | D.slice) & 3) == 0 && (reinterpret_cast<uintptr_t>(D.src) & 15) == 0 &&
                     (reinterpret_cast<uintptr_t>(D.sym) & 7) == 0;
    float4 v[kGroups];
    u32 eg[kGroups];
#pragma unroll
    for (int g = 0; g < kGroups; ++g) {
        eg[g] = e0 + u32(g) * 1024u + 4u * threadIdx.x;
        v[g] = make_float4(0.f, 0.f, 0.f, 0.f);
        if (eg[g] < total) {
            const u32 z = eg[g] / plane, r = eg[g] - z * plane, y = r / nx, xx = r - y * nx;
            const float* p = D.src + size_t(z) * D.slice + size_t(y) * D.row + xx;
            if (vec) {
                v[g] = *reinterpret_cast<const float4*>(p);
            } else {
                // element by element (the group may cross rows or be unaligned)
                float t[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const u32 e = eg[g] + u32(i);
                    if (e < total) {
                        const u32 zi = e / plane, ri = e - zi * plane, yi = ri / nx, xi = ri - yi * nx;
                        t[i] = D.src[size_t(zi) * D.slice + size_t(yi) * D.row + xi];
                    }
                }
                v[g] = make_float4(t[0], t[1], t[2], t[3]);
            }
        }
    }
#pragma unroll
    for (int g = 0; g < kGroups; ++g) {
        if (eg[g] >= total) continue;
        const u16 s0 = u16(symbolizeI(int(v[g].x * D.inv))), s1 = u16(symbolizeI(int(v[g].y * D.inv)));
        const u16 s2 = u16(symbolizeI(int(v[g].z * D.inv))), s3 = u16(symbolizeI(int(v[g].w * D.inv)));
        if (vec) {
            *reinterpret_cast<uint2*>(D.sym + eg[g]) = make_uint2(u32(s0) | (u32(s1) << 16), u32(s2) | (u32(s3) << 16));
        } else {
            const u16 sv[4] = {s0, s1, s2, s3};
#pragma unroll
            for (int i = 0; i < 4; ++i)
                if (eg[g] + u32(i) < total) D.sym[eg[g] + u32(i)] = sv[i];
        }
    }
}

// ---------------------------------------------------------------------------
// One forward level in one pass (BLevelDesc).  For each input slice of the
// CTA's Z chunk (with 4 slices of mirrored halo each side) the tile's rows
// y0-4 .. y0+TY+3 and columns x0-4 .. x0+TX+3 are staged in shared memory,
// filtered along X (outputs x0 .. x0+TX-1 of every staged row), then along Y
// (outputs y0 .. y0+TY-1); each thread keeps the Y outputs of its column
// pair and row pair for the last eight slices in a thread-private ring, and
// once an output slice's nine inputs are in it filters along Z, quantizes
// and stores.  The taps and fmaf chains are those of the separate X, Y and Z
// passes, in that order, so the coefficients - and symbols - are
// bit-identical.  Every filter runs on value pairs with Blackwell's packed
// fma.rn.f32x2 (each lane rounded as the scalar fmaf):
//  * the staged rows are stored interleaved in pairs (rows 2p, 2p+1 of a
//    column side by side), so X filters two rows at once;
//  * the X outputs are stored row-major, so Y and Z filter two adjacent
//    columns at once (one coefficient for both);
//  * warp w owns output rows 2w, 2w+1 and lane l columns 2l, 2l+1: its four
//    outputs of a slice are one per octant band and share the in-band
//    offset, and a warp's store to a band is 64 contiguous bytes.
// The slice loop is unrolled by eight, so ring slots and the z parity are
// constants.  The next slice's loads are issued before the current slice is
// filtered.
// ---------------------------------------------------------------------------
constexpr int kLvRows = kLvTY + 8;               // staged rows
constexpr int kLvCols = kLvTX + 8;               // staged columns
constexpr int kLvPairs = kLvRows / 2;            // staged row pairs
constexpr int kLvQuads = kLvCols / 4;            // 16-byte column groups of a staged row
// padded strides: a row pair of the stage is 37 16-byte units (odd, so two
// row pairs' groups fall in different banks), an X output row 18 units
constexpr int kLvPairStride = kLvCols + 2;       // float2
constexpr int kLvXStride = kLvTX + 8;            // float
static_assert(kLvTX == 64 && kLvTY == 16, "256 threads: a column pair and a row pair of outputs each");
static_assert(kLvPairs * kLvQuads <= 256, "one vector staging task per thread");

// Forward taps as a constexpr table (kFwdTap[parity][tap]) for the Z chains.
__device__ constexpr float kFwdTap[2][9] = {
    {0.0267488f, -0.0168641f, -0.0782233f, 0.2668641f, 0.6029490f, 0.2668641f, -0.0782233f, -0.0168641f, 0.0267488f},
    {0.0f, 0.0456359f, -0.0287718f, -0.2956359f, 0.5575435f, -0.2956359f, -0.0287718f, 0.0456359f, 0.0f}};

template <int K>
struct SliceK {
    static constexpr int value = K;
};

__global__ void __launch_bounds__(256, 4) k_bLevelFwd(const BLevelDesc* __restrict__ descs,
                                                     const u32* __restrict__ map, const float* const* inTab) {
    __shared__ __align__(16) float2 sIn[kLvPairs * kLvPairStride];   // (row 2p, row 2p+1) per staged column
    __shared__ __align__(16) float sX[kLvRows * kLvXStride];         // X outputs, row-major
    __shared__ float2 sZ[8][2][256];                           // Y outputs of the last eight slices
    // the descriptor's fields in registers (the output stores could alias it)
    const BLevelDesc& D = descs[map[blockIdx.x]];
    const float* const src = D.src ? D.src : inTab[D.vol];
    // lowpass output: symbols (last level) or floats; offsets below 2^31
    const bool lastLevel = D.lastLevel != 0;
    char* const lpBase = lastLevel ? reinterpret_cast<char*>(D.lpSymOut) : reinterpret_cast<char*>(D.lpOut);
    u16* const symOut = D.symOut;
    const u32 bandStride = u32(D.bandStride);
    const float inv = D.inv, invLP = D.invLP;
    const int srcRow = D.srcRow;
    const u32 srcSlice = u32(D.srcSlice);
    const u32 local = blockIdx.x - D.ctaOff;
    const int tilesX = D.tilesX, tilesY = D.tilesY;
    const int tX = int(local % u32(tilesX));
    const u32 rest = local / u32(tilesX);
    const int tY = int(rest % u32(tilesY)), cZ = int(rest / u32(tilesY));
    const int nx = D.nx, ny = D.ny, nz = D.nz;
    const int zChunk = D.zChunk;
    const int x0 = tX * kLvTX, y0 = tY * kLvTY, z0 = cZ * zChunk;
    const int TXe = min(kLvTX, nx - x0), TYe = min(kLvTY, ny - y0), ZCe = min(zChunk, nz - z0);
    const int colsE = TXe + 8, rowsE = TYe + 8;
    const int tid = int(threadIdx.x);
    // Staging: thread t < 216 moves the staged column group vq (four
    // columns) of the rows 2vp, 2vp+1 and interleaves them.  A group inside
    // the volume with 16-byte aligned rows is one float4 per row; a group
    // reaching over an edge (mirrored) or in unaligned rows is four floats.
    const bool task = tid < kLvPairs * kLvQuads;
    const int vp = tid / kLvQuads, vq = tid - vp * kLvQuads;
    const int xs = x0 - 4 + 4 * vq;   // first source column of the group
    const bool aligned = ((srcRow | int(srcSlice)) & 3) == 0 && (reinterpret_cast<uintptr_t>(src) & 15) == 0;
    const bool wide = aligned && xs >= 0 && xs + 3 < nx;
    int rowOff[2];   // source row offsets within a slice (-1: not needed)
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const int r = 2 * vp + k;
        rowOff[k] = task && r < rowsE && 4 * vq < colsE ? mirrorIdx(y0 - 4 + r, ny) * srcRow : -1;
    }
    float4 pre4[2];
    auto fetch = [&](int i) {
        const float* sl = src + u64(u32(mirrorIdx(z0 - 4 + i, nz))) * srcSlice;
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
            if (rowOff[k] >= 0) {
                const float* row = sl + rowOff[k];
                if (wide) {
                    v = *reinterpret_cast<const float4*>(row + xs);
                } else {
                    float t[4];
#pragma unroll
                    for (int e = 0; e < 4; ++e) t[e] = 4 * vq + e < colsE ? row[mirrorIdx(xs + e, nx)] : 0.0f;
                    v = make_float4(t[0], t[1], t[2], t[3]);
                }
            }
            pre4[k] = v;
        }
    };
    auto stage = [&]() {
        if (task) {
            float4* d = reinterpret_cast<float4*>(sIn + vp * kLvPairStride + 4 * vq);
            d[0] = make_float4(pre4[0].x, pre4[1].x, pre4[0].y, pre4[1].y);
            d[1] = make_float4(pre4[0].z, pre4[1].z, pre4[0].w, pre4[1].w);
        }
    };
    // X tasks: row pair xp, output columns 4 xg .. 4 xg + 3 (192 tasks);
    // warp w takes the row pairs 2w, 2w+1, and each quarter warp four
    // column groups of both (conflict-free 16-byte loads)
    const int xp = 2 * (tid >> 5) + ((tid >> 2) & 1), xg = (tid & 3) + 4 * ((tid & 31) >> 3);
    const bool xTask = tid < kLvPairs * 16 && 2 * xp < rowsE && 4 * xg < TXe;
    // Y/Z outputs: warp w rows 2w, 2w+1; lane l columns 2l, 2l+1
    const int w = tid >> 5, l = tid & 31;
    const bool outOk = 2 * w < TYe && 2 * l < TXe;
    const int hx = nx >> 1, hy = ny >> 1;
    const u32 plane = u32(hx) * u32(hy);
    const u32 inPlane = u32((y0 >> 1) + w) * u32(hx) + u32((x0 >> 1) + l);

    const int nSlices = ZCe + 8;
    int i0 = 0;
    float2 hiE = make_float2(0.0f, 0.0f), hiO = hiE;   // highpass Z chains awaiting their last tap
    // slice i = i0 + k (kc: k as a constant; i0 is a multiple of 8)
    auto slice = [&](auto kc) {
        constexpr int k = decltype(kc)::value;
        const int i = i0 + k;
        if (i >= nSlices) return;                           // CTA-uniform
        stage();
        __syncthreads();
        if (i + 1 < nSlices) fetch(i + 1);
        // X: two rows, four outputs (columns of both parities); window
        // element m is tap m - o of output o, taken in tap order as it loads
        if (xTask) {
            const float4* s4 = reinterpret_cast<const float4*>(sIn + xp * kLvPairStride + 4 * xg);
            float2 o[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) o[j] = make_float2(0.0f, 0.0f);
#pragma unroll
            for (int q = 0; q < 6; ++q) {
                const float4 v = s4[q];
                const float2 wm[2] = {make_float2(v.x, v.y), make_float2(v.z, v.w)};
#pragma unroll
                for (int h = 0; h < 2; ++h) {
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const int tap = 2 * q + h - j;
                        if (tap >= 0 && tap <= 8) {
                            const float c = kFwdTap[j & 1][tap];
                            o[j] = __ffma2_rn(make_float2(c, c), wm[h], o[j]);
                        }
                    }
                }
            }
            float4* d = reinterpret_cast<float4*>(sX + (2 * xp) * kLvXStride + 4 * xg);
            d[0] = make_float4(o[0].x, o[1].x, o[2].x, o[3].x);
            d[kLvXStride / 4] = make_float4(o[0].y, o[1].y, o[2].y, o[3].y);
        }
        __syncthreads();
        // Y: rows 2w (even taps) and 2w+1 (odd taps) of columns 2l, 2l+1
        float2 ne, no;
        {
            float2 yw[10];
#pragma unroll
            for (int q = 0; q < 10; ++q) yw[q] = *reinterpret_cast<const float2*>(sX + (2 * w + q) * kLvXStride + 2 * l);
            ne = fir9p<false, 0>(yw);
            no = fir9p<false, 1>(yw + 1);
        }
        // Z: output slice z = z0 + i - 8 once its nine input slices are in
        // (z0 and i0 are even, so z has the parity of k).  At an even k the
        // ring (slot (k + q) & 7 holds slice i - 8 + q) and slice i, in
        // registers, feed both chains in one read: the lowpass output z
        // (slices i-8 .. i) and the highpass output z + 1 (slices i-7 .. i+1)
        // up to its last tap, whose slice i + 1 arrives at the next (odd) k.
        if (i >= 8 && outOk) {
            float2 ve, vo;
            if constexpr ((k & 1) == 0) {
                ve = make_float2(0.0f, 0.0f);
                vo = make_float2(0.0f, 0.0f);
                hiE = make_float2(0.0f, 0.0f);
                hiO = make_float2(0.0f, 0.0f);
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    const float2 re = sZ[(k + q) & 7][0][tid], ro = sZ[(k + q) & 7][1][tid];
                    const float c = kFwdTap[0][q];
                    ve = __ffma2_rn(make_float2(c, c), re, ve);
                    vo = __ffma2_rn(make_float2(c, c), ro, vo);
                    if (q >= 1) {
                        const float h = kFwdTap[1][q - 1];
                        hiE = __ffma2_rn(make_float2(h, h), re, hiE);
                        hiO = __ffma2_rn(make_float2(h, h), ro, hiO);
                    }
                }
                constexpr float c8 = kFwdTap[0][8], h7 = kFwdTap[1][7];
                ve = __ffma2_rn(make_float2(c8, c8), ne, ve);
                vo = __ffma2_rn(make_float2(c8, c8), no, vo);
                hiE = __ffma2_rn(make_float2(h7, h7), ne, hiE);
                hiO = __ffma2_rn(make_float2(h7, h7), no, hiO);
            } else {
                constexpr float h8 = kFwdTap[1][8];
                ve = __ffma2_rn(make_float2(h8, h8), ne, hiE);
                vo = __ffma2_rn(make_float2(h8, h8), no, hiO);
            }
            const u64 li = u64(u32((z0 + i - 8) >> 1)) * plane + inPlane;
            constexpr int bz = (k & 1) << 2;
            // octants (x even, y even), (x odd, y even), (x even, y odd), (x odd, y odd)
            if (bz == 0) {
                if (lastLevel) reinterpret_cast<u16*>(lpBase)[li] = u16(symbolizeI(int(ve.x * invLP)));
                else reinterpret_cast<float*>(lpBase)[li] = ve.x;
            } else {
                symOut[u64(bz - 1) * bandStride + li] = u16(symbolizeI(int(ve.x * inv)));
            }
            symOut[u64(bz) * bandStride + li] = u16(symbolizeI(int(ve.y * inv)));
            symOut[u64(bz + 1) * bandStride + li] = u16(symbolizeI(int(vo.x * inv)));
            symOut[u64(bz + 2) * bandStride + li] = u16(symbolizeI(int(vo.y * inv)));
        }
        // the newest slice replaces the oldest, just used
        sZ[k][0][tid] = ne;
        sZ[k][1][tid] = no;
    };
    fetch(0);
    for (; i0 < nSlices; i0 += 8) {
        slice(SliceK<0>{});
        slice(SliceK<1>{});
        slice(SliceK<2>{});
        slice(SliceK<3>{});
        slice(SliceK<4>{});
        slice(SliceK<5>{});
        slice(SliceK<6>{});
        slice(SliceK<7>{});
    }
}

void launchBatchLevelFwd(const BLevelDesc* d, const u32* map, u32 ctas, const float* const* inTab, cudaStream_t st) {
    if (!ctas) return;
    k_bLevelFwd<<<ctas, 256, 0, st>>>(d, map, inTab);
    countLaunch();
}

void launchBatchRows(const BRowDesc* d, const u32* map, u32 ctas, bool inverse, const float* const* inTab,
                     float* const* outTab, cudaStream_t st) {
    if (!ctas) return;
    if (inverse) k_bRows<true><<<ctas, 256, 0, st>>>(d, map, inTab, outTab);
    else k_bRows<false><<<ctas, 256, 0, st>>>(d, map, inTab, outTab);
    countLaunch();
}

void launchBatchCols(const BColDesc* d, const u32* map, u32 ctas, bool inverse, bool fromSymbols, cudaStream_t st,
                     bool quantizeStore) {
    if (!ctas) return;
    const dim3 blk(32, 8);
    if (quantizeStore) k_bCols<false, false, true><<<ctas, blk, 0, st>>>(d, map);
    else if (fromSymbols) k_bCols<true, true><<<ctas, blk, 0, st>>>(d, map);
    else if (inverse) k_bCols<true, false><<<ctas, blk, 0, st>>>(d, map);
    else k_bCols<false, false><<<ctas, blk, 0, st>>>(d, map);
    countLaunch();
}

void launchBatchQuant(const BQuantDesc* d, const u32* map, u32 ctas, bool dequantize, cudaStream_t st) {
    if (!ctas) return;
    if (dequantize) k_bQuant<true><<<ctas, 256, 0, st>>>(d, map);
    else k_bQuant<false><<<ctas, 256, 0, st>>>(d, map);
    countLaunch();
}

}  // namespace ccb

using namespace ccb;

extern "C" {

int cc_dwt_float_forward(float* dst, float* buf2, float* buf1, const float* src, int sx, int sy, int sz, int ch,
                         int dstRow, int dstSlice, int srcRow, int srcSlice, void* stream) {
    return floatForward(dst, buf2, buf1, src, sx, sy, sz, ch, dstRow, dstSlice, srcRow, srcSlice,
                        static_cast<cudaStream_t>(stream), "dwtFloatForward");
}

int cc_dwt_float_forward_from_byte(float* dst, float* buf2, float* buf1, const uint8_t* src, int sx, int sy, int sz,
                                   int ch, int dstRow, int dstSlice, int srcRow, int srcSlice, void* stream) {
    return floatForward(dst, buf2, buf1, src, sx, sy, sz, ch, dstRow, dstSlice, srcRow, srcSlice,
                        static_cast<cudaStream_t>(stream), "dwtFloatForwardFromByte");
}

int cc_dwt_float_inverse(float* dst, float* buf2, float* buf1, const float* src, int sx, int sy, int sz, int ch,
                         int dstRow, int dstSlice, int srcRow, int srcSlice, void* stream) {
    return floatInverse(dst, buf2, buf1, src, sx, sy, sz, ch, dstRow, dstSlice, srcRow, srcSlice,
                        static_cast<cudaStream_t>(stream), "dwtFloatInverse");
}

int cc_dwt_float_inverse_to_byte(uint8_t* dst, float* buf2, float* buf1, const float* src, int sx, int sy, int sz,
                                 int ch, int dstRow, int dstSlice, int srcRow, int srcSlice, void* stream) {
    return floatInverse(dst, buf2, buf1, src, sx, sy, sz, ch, dstRow, dstSlice, srcRow, srcSlice,
                        static_cast<cudaStream_t>(stream), "dwtFloatInverseToByte");
}

int cc_dwt_float_inverse_from_symbols(float* dst, float* buf2, float* buf1, const float* lowpass,
                                      const void* const* highpass, int symBytes, float step, int sx, int sy, int sz,
                                      int ch, int dstRow, int dstSlice, int lpRow, int lpSlice, void* stream) {
    return floatInverseFromSymbols(dst, buf2, buf1, lowpass, highpass, symBytes, step, sx, sy, sz, ch, dstRow,
                                   dstSlice, lpRow, lpSlice, static_cast<cudaStream_t>(stream),
                                   "dwtFloatInverseFromSymbols");
}

int cc_dwt_float_inverse_from_symbols_to_byte(uint8_t* dst, float* buf2, float* buf1, const float* lowpass,
                                              const void* const* highpass, int symBytes, float step, int sx, int sy,
                                              int sz, int ch, int dstRow, int dstSlice, int lpRow, int lpSlice,
                                              void* stream) {
    return floatInverseFromSymbols(dst, buf2, buf1, lowpass, highpass, symBytes, step, sx, sy, sz, ch, dstRow,
                                   dstSlice, lpRow, lpSlice, static_cast<cudaStream_t>(stream),
                                   "dwtFloatInverseFromSymbolsToByte");
}

// dwtFloatForwardLowpassOnly (DWTFloat.cu:17-83, 535-551): the LL band of one
// 2D level; pitches default to size_x / 2 (destination) and size_x * channels
// (source).  The buffer is not used (the reference leaves its X-lowpass
// intermediate there).
int cc_dwt_float2d_forward_lowpass_only_from_byte(float* dst, float* buf, const uint8_t* src, int sx, int sy, int ch,
                                                  int dstRow, int srcRow, void* stream) {
    (void)buf;
    if (!checkSizes(sx, sy, 1, "dwtFloat2DForwardLowpassOnlyFromByte")) return CC_ERR_INVALID_ARGUMENT;
    if (ch < 1 || ch > 4) { setError("channel count must be 1..4"); return CC_ERR_INVALID_ARGUMENT; }
    if (dstRow <= 0) dstRow = sx / 2;
    if (srcRow <= 0) srcRow = sx * ch;
    const dim3 g(unsigned(ceilDiv(sx / 2, kLpTile)), unsigned(ceilDiv(sy / 2, kLpTile)));
    k_lowpass97<u8, float><<<g, 256, 0, static_cast<cudaStream_t>(stream)>>>(dst, src, sx, sy, ch, srcRow, 1, dstRow);
    countLaunch();
    CC_TRY_CUDA(cudaGetLastError(), "dwtFloat2DForwardLowpassOnlyFromByte");
    return CC_OK;
}

// dwtIntForwardLowpassOnly (DWTInt.cu:14-77): the LL band of one 2D level of
// the 5/3 lifting.  The reference transforms only whole blocks of 512 columns
// and 64 rows and leaves the rest of the band unwritten; here every LL sample
// is computed, equal to the reference's wherever it writes one.
int cc_dwt_int_forward_lowpass_only(int16_t* dst, int16_t* buf, const int16_t* src, int sx, int sy, int dstRow,
                                    int srcRow, void* stream) {
    (void)buf;
    if (!checkSizes(sx, sy, 1, "dwtIntForwardLowpassOnly")) return CC_ERR_INVALID_ARGUMENT;
    if (dstRow <= 0) dstRow = sx / 2;
    if (srcRow <= 0) srcRow = sx;
    const dim3 g(unsigned(ceilDiv(sx / 2, kLpTile)), unsigned(ceilDiv(sy / 2, kLpTile)));
    k_lowpass53<false><<<g, 256, 0, static_cast<cudaStream_t>(stream)>>>(dst, src, sx, sy, srcRow, dstRow, 0);
    countLaunch();
    CC_TRY_CUDA(cudaGetLastError(), "dwtIntForwardLowpassOnly");
    return CC_OK;
}

int cc_dwt_int_forward(int16_t* dst, int16_t* buf, const int16_t* src, int sx, int sy, int sz, int dstRow,
                       int dstSlice, int srcRow, int srcSlice, void* stream) {
    if (!checkSizes(sx, sy, sz, "dwtIntForward")) return CC_ERR_INVALID_ARGUMENT;
    if (dstRow <= 0) dstRow = sx;
    if (dstSlice <= 0) dstSlice = sy * dstRow;
    if (srcRow <= 0) srcRow = sx;
    if (srcSlice <= 0) srcSlice = sy * srcRow;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const bool do3D = sz > 1;
    i16* xDst = do3D ? dst : buf;                       // DWTInt.cu:111
    liftPass<false>(xDst, src, sx, sy, sz, 0, srcRow, srcSlice, dstRow, dstSlice, st);
    i16* yDst = do3D ? buf : dst;                       // DWTInt.cu:138
    liftPass<false>(yDst, xDst, sx, sy, sz, 1, dstRow, dstSlice, dstRow, dstSlice, st);
    if (do3D) liftPass<false>(dst, buf, sx, sy, sz, 2, dstRow, dstSlice, dstRow, dstSlice, st);
    CC_TRY_CUDA(cudaGetLastError(), "dwtIntForward");
    return CC_OK;
}

int cc_dwt_int_inverse(int16_t* dst, int16_t* buf, const int16_t* src, int sx, int sy, int sz, int dstRow,
                       int dstSlice, int srcRow, int srcSlice, void* stream) {
    if (!checkSizes(sx, sy, sz, "dwtIntInverse")) return CC_ERR_INVALID_ARGUMENT;
    if (dstRow <= 0) dstRow = sx;
    if (dstSlice <= 0) dstSlice = sy * dstRow;
    if (srcRow <= 0) srcRow = sx;
    if (srcSlice <= 0) srcSlice = sy * srcRow;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const bool do3D = sz > 1;
    const i16* ySrc = src;
    if (do3D) {
        liftPass<true>(dst, src, sx, sy, sz, 2, srcRow, srcSlice, srcRow, srcSlice, st);
        ySrc = dst;
    }
    liftPass<true>(buf, ySrc, sx, sy, sz, 1, srcRow, srcSlice, srcRow, srcSlice, st);
    liftPass<true>(dst, buf, sx, sy, sz, 0, srcRow, srcSlice, dstRow, dstSlice, st);
    CC_TRY_CUDA(cudaGetLastError(), "dwtIntInverse");
    return CC_OK;
}


// getLowpassImage (examples CompressImage.cpp:342-365): for the first
// `channels` of `channelCount` interleaved byte channels, the LL band of one
// 9/7 level converted back to bytes (floatToByte), into a byte image of
// size_x/2 x size_y/2 with the same interleaving.  One launch for all
// channels; no float intermediate.
int cc_get_lowpass_image(const uint8_t* src, int sx, int sy, int channelCount, int channels, uint8_t* dst,
                         void* stream) {
    if (!checkSizes(sx, sy, 1, "getLowpassImage")) return CC_ERR_INVALID_ARGUMENT;
    if (channelCount < 1 || channelCount > 4 || channels < 1 || channels > channelCount) {
        setError("getLowpassImage: channel counts must satisfy 1 <= channels <= channelCount <= 4");
        return CC_ERR_INVALID_ARGUMENT;
    }
    const dim3 g(unsigned(ceilDiv(sx / 2, kLpTile)), unsigned(ceilDiv(sy / 2, kLpTile)), unsigned(channels));
    k_lowpass97<u8, u8><<<g, 256, 0, static_cast<cudaStream_t>(stream)>>>(dst, src, sx, sy, channelCount,
                                                                           sx * channelCount, channelCount, sx / 2);
    countLaunch();
    CC_TRY_CUDA(cudaGetLastError(), "getLowpassImage");
    return CC_OK;
}

// getLowpassHeightfield (examples CompressHeightfield.cpp:218-235): the LL
// band of one 5/3 level with the lowpass shift added and the least
// significant bit removed (removeLSB without bits), dense size_x/2 x size_y/2.
int cc_get_lowpass_heightfield(const int16_t* src, int sx, int sy, int16_t* dst, int16_t shift, void* stream) {
    if (!checkSizes(sx, sy, 1, "getLowpassHeightfield")) return CC_ERR_INVALID_ARGUMENT;
    const dim3 g(unsigned(ceilDiv(sx / 2, kLpTile)), unsigned(ceilDiv(sy / 2, kLpTile)));
    k_lowpass53<true><<<g, 256, 0, static_cast<cudaStream_t>(stream)>>>(dst, src, sx, sy, sx, sx / 2, shift);
    countLaunch();
    CC_TRY_CUDA(cudaGetLastError(), "getLowpassHeightfield");
    return CC_OK;
}

// Forward float DWT with its intermediates in the library's fixed device
// scratch (no counterpart in the reference).  Same arguments and results as
// cc_dwt_float_forward without the two buffers; runs on the current device.
// The first call on a device resolves the scratch address there (set-up);
// make that first call before any stream capture.  All calls share one
// scratch per device and it keeps the last call's contents: calls that
// overlap on the GPU (other streams, other threads) race.  Nothing in it has
// to start at zero: each pass writes every element the next pass reads.
int cc_dwt_float_forward_static(float* dst, const float* src, int sx, int sy, int sz, int ch, int dstRow,
                                int dstSlice, int srcRow, int srcSlice, void* stream) {
    if (!checkSizes(sx, sy, sz, "dwtFloatForwardStatic")) return CC_ERR_INVALID_ARGUMENT;
    if (ch < 1 || ch > 4) { setError("channel count must be 1..4"); return CC_ERR_INVALID_ARGUMENT; }
    if (dstRow <= 0) dstRow = sx;
    if (dstSlice <= 0) dstSlice = sy * dstRow;
    if (srcRow <= 0) srcRow = sx * ch;
    if (srcSlice <= 0) srcSlice = sy * srcRow;
    if (dstRow < sx || (sz > 1 && dstSlice < sy * dstRow)) {
        setError("dwtFloatForwardStatic: destination pitches smaller than the volume");
        return CC_ERR_INVALID_ARGUMENT;
    }
    // extent of one intermediate volume (it uses the destination's pitches)
    const u64 extent = u64(sz - 1) * u64(dstSlice) + u64(sy - 1) * u64(dstRow) + u64(sx);
    if (extent > kStaticScratchFloats) {
        setError("dwtFloatForwardStatic: volume needs %llu scratch floats, the fixed scratch holds %llu",
                 (unsigned long long)extent, (unsigned long long)kStaticScratchFloats);
        return CC_ERR_CAPACITY;
    }
    int device = -1;
    CC_TRY_CUDA(cudaGetDevice(&device), "dwtFloatForwardStatic: cudaGetDevice");
    float* scratch = nullptr;
    const int rc = dwtScratchFor(device, &scratch);
    if (rc) return rc;
    float* buf1 = scratch;
    float* buf2 = scratch + kStaticScratchFloats;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const bool do3D = sz > 1;
    rowPass<float, float, false>(buf1, src, sx, sy, sz, ch, srcRow, srcSlice, 1, dstRow, dstSlice, st);
    float* yDst = do3D ? buf2 : dst;
    colPass<false>(yDst, pitchLoad(buf1, 1, dstRow, dstSlice), sx, sy, sz, 1, dstRow, dstSlice, st);
    if (do3D) colPass<false>(dst, pitchLoad(buf2, 2, dstRow, dstSlice), sx, sy, sz, 2, dstRow, dstSlice, st);
    CC_TRY_CUDA(cudaGetLastError(), "dwtFloatForwardStatic");
    return CC_OK;
}

}  // extern "C"
