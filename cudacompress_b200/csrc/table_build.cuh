// table_build.cuh - the device side of the Huffman table construction: the
// same observable result as the reference's host builder (HuffmanTable.cu:
// 487-596, libstdc++ priority_queue + std::sort) with the work a block can
// share done by the block.
//
//  * tree: make_heap runs level by level over the block; the merge loop
//    stays sequential (one thread) on a shared-memory heap laid out 1-based
//    so that the two children of a node are one aligned 16-byte load, with
//    the grandchildren loaded speculatively beside them;
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
// Elements: (probability << 32) | node id; "less(a, b)" is b.prob < a.prob
// (the top is the smallest probability; ties are not broken by id, so the
// result depends on the exact libstdc++ heap moves, which are replayed).
// Writes parent[id] for every node except the root.
// ---------------------------------------------------------------------------
__device__ __forceinline__ u32 probOf(u64 v) { return u32(v >> 32); }

// make_heap (libstdc++ __make_heap): __adjust_heap of every parent from
// (len-2)/2 down to 0.  Parents at one depth have disjoint subtrees and all
// deeper parents come first in that order, so the parents of one depth are
// adjusted in parallel, deepest depth first, with the same result.  All
// threads of the block.
__device__ void blockMakeHeap(u64* H, int len) {
    if (len < 2) return;
    const int lastParent = (len - 2) / 2;
    for (int d = 31 - __clz(lastParent + 1); d >= 0; --d) {
        const int first = (1 << d) - 1, last = min(2 * first, lastParent);
        for (int p = first + int(threadIdx.x); p <= last; p += int(blockDim.x))
            hb::adjustHeap(H + 1, p, len, H[p + 1], hb::ProbInvLess());
        __syncthreads();
    }
}

__device__ __forceinline__ ulonglong2 ld2(const u64* H, int i) { return *reinterpret_cast<const ulonglong2*>(H + i); }

// pop_heap on H[1..n+1] (libstdc++ __pop_heap: the last element v goes
// through __adjust_heap(first, 0, n, v) and __push_heap); returns the top.
// One thread.  The sift-down resolves two levels per step: the children and
// both grandchild pairs are loaded together (capEven: the largest even index
// e with H[e + 1] inside the array clamps the speculative loads).  The
// push-up compares v with the last two values moved up, still in registers.
__device__ __forceinline__ u64 popTop(u64* H, int n, int capEven) {
    const u64 top = H[1];
    if (n <= 0) return top;
    const u64 v = H[n + 1];
    const u32 pv = probOf(v);
    const int lim = (n - 1) / 2;
    int hole = 0;
    u64 w1 = 0, w2 = 0;   // values moved into the hole's parent and grandparent
    while (hole < lim) {
        const int c = 2 * hole + 2;   // right child; the pair (c-1, c) is H[c], H[c+1]
        const ulonglong2 pr = ld2(H, c);
        const ulonglong2 gl = ld2(H, min(2 * c, capEven));
        const ulonglong2 gr = ld2(H, min(2 * c + 2, capEven));
        const bool left = probOf(pr.x) < probOf(pr.y);   // less(right, left)
        const u64 cv = left ? pr.x : pr.y;
        H[hole + 1] = cv;
        hole = left ? c - 1 : c;
        w2 = w1;
        w1 = cv;
        if (hole >= lim) break;
        const ulonglong2 q = left ? gl : gr;
        const bool left2 = probOf(q.x) < probOf(q.y);
        const u64 cv2 = left2 ? q.x : q.y;
        H[hole + 1] = cv2;
        hole = 2 * hole + (left2 ? 1 : 2);
        w2 = w1;
        w1 = cv2;
    }
    if ((n & 1) == 0 && hole == (n - 2) / 2) {
        const u64 cv = H[2 * hole + 2];
        H[hole + 1] = cv;
        hole = 2 * hole + 1;
        w2 = w1;
        w1 = cv;
    }
    if (hole > 0 && pv < probOf(w1)) {
        H[hole + 1] = w1;
        hole = (hole - 1) / 2;
        if (hole > 0 && pv < probOf(w2)) {
            H[hole + 1] = w2;
            hole = (hole - 1) / 2;
            while (hole > 0) {
                const int parent = (hole - 1) / 2;
                const u64 pe = H[parent + 1];
                if (!(pv < probOf(pe))) break;
                H[hole + 1] = pe;
                hole = parent;
            }
        }
    }
    H[hole + 1] = v;
    return top;
}

// push_heap of v as element len-1 (__push_heap); three ancestors per step are
// loaded together.
__device__ __forceinline__ void pushLast(u64* H, int len, u64 v) {
    int hole = len - 1;
    const u32 pv = probOf(v);
    while (hole > 0) {
        const int p1 = (hole - 1) / 2, p2 = p1 > 0 ? (p1 - 1) / 2 : 0, p3 = p2 > 0 ? (p2 - 1) / 2 : 0;
        const u64 e1 = H[p1 + 1], e2 = H[p2 + 1], e3 = H[p3 + 1];
        if (!(pv < probOf(e1))) break;
        H[hole + 1] = e1;
        hole = p1;
        if (hole == 0 || !(pv < probOf(e2))) break;
        H[hole + 1] = e2;
        hole = p2;
        if (hole == 0 || !(pv < probOf(e3))) break;
        H[hole + 1] = e3;
        hole = p3;
    }
    H[hole + 1] = v;
}

// The merge loop (HuffmanTable.cu:512-529) on a heap made by blockMakeHeap.
// One thread; H holds L + 2 entries.
__device__ void buildTree(u64* H, u32* parent, int L) {
    const int capEven = L & ~1;
    int len = L;
    u32 next = u32(L);
    while (len > 1) {
        const u64 a = popTop(H, len - 1, capEven);
        --len;
        const u64 b = popTop(H, len - 1, capEven);
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
        // counters[1] counts the next round's segments.  Its reset comes
        // after the barrier that ends the previous round's reads of it (the
        // third barrier below), and the barrier after the reset orders it
        // before this round's additions.
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
        __syncthreads();   // every thread has read the count before thread 0 resets it
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
