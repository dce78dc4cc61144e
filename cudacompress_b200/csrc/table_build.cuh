// table_build.cuh - the device side of the Huffman table construction: the
// same observable result as the reference's host builder (HuffmanTable.cu:
// 487-596, libstdc++ priority_queue + std::sort) with the work a block can
// share done by the block.
//
//  * tree: the priority-queue merge stays sequential (one thread), on a
//    shared-memory heap laid out 1-based so that the two children of a node
//    are one aligned 16-byte load;
//  * depths: one thread per leaf walks to the root;
//  * sort: std::sort's introsort is replayed exactly, but every partition
//    step runs on a warp: the left scan stops at the k-th element not less
//    than the pivot and the right scan at the k-th element not greater than
//    it, so the swap pairs, their count and the cut follow from two ordered
//    lists made with ballots; disjoint segments are partitioned by different
//    warps at the same time; segments left at <= 16 elements get the final
//    insertion sort independently (no element crosses a partition cut,
//    because every element left of a cut is not greater than any right of
//    it and the insertion only moves past strictly greater elements).
#pragma once

#include "huffman_build.cuh"

namespace ccb {
namespace tb {

// ---------------------------------------------------------------------------
// Tree (HuffmanTable.cu:507-529).  H[i + 1] holds heap element i, i.e. the
// heap is 1-based inside H; H must be 16-byte aligned and hold L + 2 entries.
// Elements: (probability << 32) | node id.  Writes parent[id] for every node
// except the root.
// ---------------------------------------------------------------------------
__device__ __forceinline__ u32 probOf(u64 v) { return u32(v >> 32); }

// libstdc++ __adjust_heap from the root with value v over `len` elements,
// then __push_heap; "less(a, b)" is b.prob < a.prob.
__device__ __forceinline__ void siftFromRoot(u64* H, int len, u64 v) {
    int hole = 0, child = 0;
    const int lim = (len - 1) / 2;
    while (child < lim) {
        child = 2 * (child + 1);                                     // right child (0-based)
        const ulonglong2 pr = *reinterpret_cast<const ulonglong2*>(H + child);   // elements child-1, child
        const bool takeLeft = probOf(pr.x) < probOf(pr.y);           // less(right, left)
        child -= takeLeft ? 1 : 0;
        H[hole + 1] = takeLeft ? pr.x : pr.y;
        hole = child;
    }
    if ((len & 1) == 0 && child == (len - 2) / 2) {
        child = 2 * (child + 1);
        H[hole + 1] = H[child];                                      // element child - 1
        hole = child - 1;
    }
    const u32 pv = probOf(v);
    while (hole > 0) {
        const int parent = (hole - 1) / 2;
        const u64 pe = H[parent + 1];
        if (!(pv < probOf(pe))) break;                               // less(a[parent], v)
        H[hole + 1] = pe;
        hole = parent;
    }
    H[hole + 1] = v;
}

__device__ __forceinline__ void pushLast(u64* H, int len, u64 v) {
    int hole = len - 1;
    const u32 pv = probOf(v);
    while (hole > 0) {
        const int parent = (hole - 1) / 2;
        const u64 pe = H[parent + 1];
        if (!(pv < probOf(pe))) break;
        H[hole + 1] = pe;
        hole = parent;
    }
    H[hole + 1] = v;
}

// One thread.  H[1..L] holds the leaves (prob << 32 | leaf index) in symbol
// order.
__device__ void buildTree(u64* H, u32* parent, int L) {
    hb::makeHeap(H + 1, L, hb::ProbInvLess());
    int len = L;
    u32 next = u32(L);
    while (len > 1) {
        const u64 a = H[1];
        siftFromRoot(H, len - 1, H[len]);
        --len;
        const u64 b = H[1];
        siftFromRoot(H, len - 1, H[len]);
        --len;
        parent[u32(a)] = next;
        parent[u32(b)] = next;
        const u64 node = (u64(probOf(a) + probOf(b)) << 32) | next;
        ++next;
        ++len;
        pushLast(H, len, node);
    }
}

// ---------------------------------------------------------------------------
// Sort (HuffmanTable.cu:538, libstdc++ std::sort) of keys (len << 27 | leaf).
// ---------------------------------------------------------------------------
struct Seg {
    int f, l, d;
};
constexpr int kSortThreshold = 16;
constexpr int kMaxSegs = 512;   // segments longer than 16 of up to 8192 keys

__device__ __forceinline__ u32 keyOf(u32 v) { return v >> 27; }

// Exact replay of __unguarded_partition(a + f + 1, a + l, a + f) by one warp.
// lList / rList: scratch positions for [f, l) (entries f .. l-1 are used).
__device__ int warpPartition(u32* a, int f, int l, u16* lList, u16* rList) {
    const u32 lane = threadIdx.x & 31u;
    const u32 ltMask = (1u << lane) - 1u;
    const u32 p = keyOf(a[f]);
    int nL = 0, nR = 0;
    for (int base = f + 1; base < l; base += 32) {
        const int j = base + int(lane);
        const bool pred = j < l && !(keyOf(a[j]) < p);
        const u32 m = __ballot_sync(0xffffffffu, pred);
        if (pred) lList[f + nL + __popc(m & ltMask)] = u16(j);
        nL += __popc(m);
    }
    for (int top = l - 1; top > f; top -= 32) {
        const int j = top - int(lane);
        const bool pred = j > f && !(p < keyOf(a[j]));
        const u32 m = __ballot_sync(0xffffffffu, pred);
        if (pred) rList[f + nR + __popc(m & ltMask)] = u16(j);
        nR += __popc(m);
    }
    __syncwarp();
    // K = number of leading k with lList[k] < rList[k] (monotone in k)
    const int kMax = min(nL, nR);
    int K = 0;
    for (int base = 0; base < kMax; base += 32) {
        const int k = base + int(lane);
        const bool ok = k < kMax && lList[f + k] < rList[f + k];
        const u32 m = __ballot_sync(0xffffffffu, ok);
        const int run = (m == 0xffffffffu) ? 32 : __ffs(~m) - 1;
        K += run;
        if (run < 32) break;
    }
    // swaps (disjoint positions)
    for (int k = int(lane); k < K; k += 32) {
        const int x = lList[f + k], y = rList[f + k];
        const u32 t = a[x];
        a[x] = a[y];
        a[y] = t;
    }
    int cut;
    if (K == 0) cut = lList[f];
    else cut = min(K < nL ? int(lList[f + K]) : 0x7fffffff, int(rList[f + K - 1]));
    __syncwarp();
    return cut;
}

// Block-cooperative introsort of a[0, n) (n <= 8192).  Scratch: lList, rList
// (n u16 each), mark (n bytes), two segment queues.  All threads call it.
template <int kThreads>
__device__ void blockIntrosort(u32* a, int n, u16* lList, u16* rList, u8* mark, Seg* qA, Seg* qB, int* counters) {
    constexpr int kWarps = kThreads / 32;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int i = threadIdx.x; i < n; i += kThreads) mark[i] = 0;
    if (threadIdx.x == 0) {
        counters[0] = 0;
        if (n > kSortThreshold) {
            qA[0] = Seg{0, n, 2 * hb::floorLog2(n)};
            counters[0] = 1;
        }
    }
    __syncthreads();
    if (n > 0 && threadIdx.x == 0 && n <= kSortThreshold) mark[0] = 1;
    Seg* cur = qA;
    Seg* nxt = qB;
    int nCur = counters[0];
    while (nCur > 0) {
        if (threadIdx.x == 0) counters[1] = 0;
        __syncthreads();
        for (int s = warp; s < nCur; s += kWarps) {
            const Seg g = cur[s];
            if (g.d == 0) {
                if (lane == 0) {
                    hb::makeHeap(a + g.f, g.l - g.f, hb::LenLess());
                    hb::sortHeap(a + g.f, g.l - g.f, hb::LenLess());
                    mark[g.f] = 2;   // sorted, no insertion pass
                }
                __syncwarp();
                continue;
            }
            if (lane == 0) hb::moveMedianToFirst(a, g.f, g.f + 1, g.f + (g.l - g.f) / 2, g.l - 1, hb::LenLess());
            __syncwarp();
            const int cut = warpPartition(a, g.f, g.l, lList, rList);
            if (lane == 0) {
                const Seg kids[2] = {Seg{g.f, cut, g.d - 1}, Seg{cut, g.l, g.d - 1}};
                for (int k = 0; k < 2; ++k) {
                    if (kids[k].l - kids[k].f > kSortThreshold) nxt[atomicAdd(&counters[1], 1)] = kids[k];
                    else if (kids[k].l > kids[k].f) mark[kids[k].f] = 1;
                }
            }
            __syncwarp();
        }
        __syncthreads();
        nCur = counters[1];
        Seg* t = cur;
        cur = nxt;
        nxt = t;
    }
    __syncthreads();
    // final insertion sort, one thread per segment of at most 16 keys
    for (int i = threadIdx.x; i < n; i += kThreads) {
        if (mark[i] != 1) continue;
        int e = i + 1;
        while (e < n && mark[e] == 0) ++e;
        for (int k = i + 1; k < e; ++k) {
            const u32 v = a[k];
            int j = k;
            while (j > i && keyOf(v) < keyOf(a[j - 1])) {
                a[j] = a[j - 1];
                --j;
            }
            a[j] = v;
        }
    }
    __syncthreads();
}

}  // namespace tb
}  // namespace ccb
