// cc_common.cuh - shared types, error plumbing and warp/block primitives for
// the cudacompress_b200 library (sm_100a).
#pragma once

#include <cstdint>
#include <cstdio>
#include <cuda_runtime.h>

#include "../../include/cudacompress_b200.h"

#define CC_HD __host__ __device__ __forceinline__

namespace ccb {

typedef uint8_t u8;
typedef uint16_t u16;
typedef uint32_t u32;
typedef uint64_t u64;
typedef int16_t i16;
typedef int32_t i32;

// Device-side error flags (bit set, OR-ed by kernels, read back by the host).
enum DeviceError : u32 {
    DEV_ERR_SYMBOL_RANGE = 1u,
    DEV_ERR_CODEWORD_TOO_LONG = 2u,
    DEV_ERR_CORRUPT = 4u,
    DEV_ERR_TIMEOUT = 8u,
    DEV_ERR_TABLE_CAPACITY = 16u,
    DEV_ERR_OUTPUT_CAPACITY = 32u,
};

constexpr u32 kMaxCodewordBits = 32;      // EncodeCommon.h:24-25
constexpr u32 kZeroCountMax = 255;        // EncodeCommon.h:31
constexpr u32 kWarp = 32;

CC_HD u32 requiredBits(u32 v) { return v ? 32u - u32(__builtin_clz(v)) : 0u; }

CC_HD u64 ceilDiv(u64 a, u64 b) { return (a + b - 1) / b; }
CC_HD u64 alignUp(u64 a, u64 b) { return (a + b - 1) / b * b; }

#ifdef __CUDACC__
// Inclusive warp scan (sum).
__device__ __forceinline__ u32 warpInclusiveSum(u32 v) {
    const u32 lane = threadIdx.x & 31u;
#pragma unroll
    for (u32 o = 1; o < 32; o <<= 1) {
        u32 t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}
__device__ __forceinline__ u32 warpSum(u32 v) {
#pragma unroll
    for (u32 o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ u32 warpMax(u32 v) {
#pragma unroll
    for (u32 o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Exclusive scan of in[0, n) into out by one warp (in == out allowed), each
// lane taking eight consecutive elements per step; returns carry + the total.
__device__ __forceinline__ u32 warpExclusiveScan8(const u32* in, u32* out, u32 n, u32 carry) {
    const u32 lane = threadIdx.x & 31u;
    for (u32 base = 0; base < n; base += 256) {
        const u32 i0 = base + 8u * lane;
        u32 v[8], sum = 0;
#pragma unroll
        for (u32 k = 0; k < 8; ++k) {
            v[k] = i0 + k < n ? in[i0 + k] : 0u;
            sum += v[k];
        }
        const u32 incl = warpInclusiveSum(sum);
        u32 run = carry + incl - sum;
#pragma unroll
        for (u32 k = 0; k < 8; ++k) {
            if (i0 + k < n) out[i0 + k] = run;
            run += v[k];
        }
        carry += __shfl_sync(0xffffffffu, incl, 31);
    }
    return carry;
}

// Block-wide exclusive scan of one u32 per thread; returns the exclusive
// prefix and writes the block total to *total.  `scratch` holds >= 33 u32.
template <int kThreads>
__device__ __forceinline__ u32 blockExclusiveSum(u32 v, u32* scratch, u32* total) {
    static_assert(kThreads % 32 == 0 && kThreads <= 1024, "block size");
    const u32 lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    u32 inc = warpInclusiveSum(v);
    if (lane == 31) scratch[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        u32 w = lane < kThreads / 32 ? scratch[lane] : 0u;
        u32 wi = warpInclusiveSum(w);
        scratch[lane] = wi - w;
        if (lane == 31) scratch[32] = wi;
    }
    __syncthreads();
    u32 r = scratch[warp] + inc - v;
    if (total) *total = scratch[32];
    __syncthreads();
    return r;
}

// Block-wide exclusive scans of N values per thread at once (two barriers
// for all N): ex[k] = the exclusive prefix of v[k], tot[k] = its block
// total.  `scratch` holds >= 33 * N u32.
template <int kThreads, int N>
__device__ __forceinline__ void blockExclusiveSumN(const u32 (&v)[N], u32 (&ex)[N], u32 (&tot)[N], u32* scratch) {
    static_assert(kThreads % 32 == 0 && kThreads <= 1024, "block size");
    const u32 lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    u32 inc[N];
#pragma unroll
    for (int k = 0; k < N; ++k) inc[k] = warpInclusiveSum(v[k]);
    if (lane == 31) {
#pragma unroll
        for (int k = 0; k < N; ++k) scratch[33 * k + warp] = inc[k];
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < N; ++k) {
            const u32 w = lane < kThreads / 32 ? scratch[33 * k + lane] : 0u;
            const u32 wi = warpInclusiveSum(w);
            scratch[33 * k + lane] = wi - w;
            if (lane == 31) scratch[33 * k + 32] = wi;
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < N; ++k) {
        ex[k] = scratch[33 * k + warp] + inc[k] - v[k];
        tot[k] = scratch[33 * k + 32];
    }
    __syncthreads();
}

// Quantize.cuh:26-35: symbol = 2|v| for v >= 0, 2|v| - 1 for v < 0, and back.
__device__ __forceinline__ u32 symbolizeI(int v) { return 2u * u32(abs(v)) + u32(v >> 31); }
__device__ __forceinline__ int unsymbolizeI(u32 s) {
    int neg = int(s & 1u);
    return (1 - 2 * neg) * int((s + u32(neg)) >> 1);
}
__device__ __forceinline__ float signF(float v) { return v > 0.0f ? 1.0f : (v < 0.0f ? -1.0f : 0.0f); }
__device__ __forceinline__ float signI(int q) { return q > 0 ? 1.0f : (q < 0 ? -1.0f : 0.0f); }
// Quantize.cuh:75-131: type 0 deadzone (truncation; centre of the bin back),
// type 1 uniform (round half away from zero; bin value back).
__device__ __forceinline__ int quantizeV(float v, float inv, int type) {
    if (type == 0) return int(v * inv);
    return int(__fmaf_rn(v, inv, signF(v) * 0.5f));
}
__device__ __forceinline__ float unquantizeV(int q, float step, int type) {
    if (type == 0) return (float(q) + signI(q) * 0.5f) * step;
    return float(q) * step;
}

// Warp-aggregated increment of `bins[key]`: lanes with equal keys are merged
// with match_any so each distinct key issues one shared/global atomic.
__device__ __forceinline__ void aggregatedIncrement(u32* bins, u32 key, bool active) {
    const u32 mask = __ballot_sync(0xffffffffu, active);
    if (!active) return;
    const u32 peers = __match_any_sync(mask, key);
    if ((threadIdx.x & 31u) == u32(__ffs(peers) - 1)) atomicAdd(bins + key, u32(__popc(peers)));
}
#endif

}  // namespace ccb
