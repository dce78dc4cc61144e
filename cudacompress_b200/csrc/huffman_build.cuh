// huffman_build.cuh - Huffman table construction whose observable result is
// identical to the reference's host builder (HuffmanTable.cu:487-596).
//
// The reference builds the tree with std::priority_queue over node pointers
// ordered by probability only (HuffmanDesign.h:42-51), constructed from the
// leaf range in symbol order (HuffmanTable.cu:507), and orders the leaves by
// codeword length with the unstable std::sort (HuffmanTable.cu:538).  Ties are
// therefore resolved by the binary-heap sift order and by introsort's
// partitioning.  This file states those procedures explicitly (binary heap
// with hole-to-leaf sift-down followed by sift-up; introsort with
// median-of-three pivot, unguarded Hoare partition, 16-element cutoff,
// 2*floor(log2 n) depth limit falling back to heapsort, and a final insertion
// sort), so the same tie-breaks come out on the GPU and on the host.
//
// All routines are __host__ __device__ and run in one thread; the device
// kernel (codec.cu) wraps them with block-parallel leaf gathering, depth
// computation and serialization.
#pragma once

#include "cc_common.cuh"

namespace ccb {
namespace hb {

// ----- binary heap primitives (generic over element type and "less") -----
template <class T, class Less>
CC_HD void pushHole(T* a, int hole, int top, T v, Less less) {
    int parent = (hole - 1) / 2;
    while (hole > top && less(a[parent], v)) {
        a[hole] = a[parent];
        hole = parent;
        parent = (hole - 1) / 2;
    }
    a[hole] = v;
}

template <class T, class Less>
CC_HD void adjustHeap(T* a, int hole, int len, T v, Less less) {
    const int top = hole;
    int child = hole;
    while (child < (len - 1) / 2) {
        child = 2 * (child + 1);
        if (less(a[child], a[child - 1])) child--;
        a[hole] = a[child];
        hole = child;
    }
    if ((len & 1) == 0 && child == (len - 2) / 2) {
        child = 2 * (child + 1);
        a[hole] = a[child - 1];
        hole = child - 1;
    }
    pushHole(a, hole, top, v, less);
}

template <class T, class Less>
CC_HD void makeHeap(T* a, int len, Less less) {
    if (len < 2) return;
    int parent = (len - 2) / 2;
    while (true) {
        T v = a[parent];
        adjustHeap(a, parent, len, v, less);
        if (parent == 0) return;
        parent--;
    }
}

// Removes the top: moves it to a[len-1] and restores the heap on [0, len-1).
template <class T, class Less>
CC_HD void popHeap(T* a, int len, Less less) {
    if (len > 1) {
        T v = a[len - 1];
        a[len - 1] = a[0];
        adjustHeap(a, 0, len - 1, v, less);
    }
}

// a[len-1] is the new element.
template <class T, class Less>
CC_HD void pushHeap(T* a, int len, Less less) {
    T v = a[len - 1];
    pushHole(a, len - 1, 0, v, less);
}

template <class T, class Less>
CC_HD void sortHeap(T* a, int len, Less less) {
    while (len > 1) {
        len--;
        T v = a[len];
        a[len] = a[0];
        adjustHeap(a, 0, len, v, less);
    }
}

// ----- introsort -----
template <class T>
CC_HD void swapT(T& x, T& y) { T t = x; x = y; y = t; }

template <class T, class Less>
CC_HD void moveMedianToFirst(T* a, int result, int x, int y, int z, Less less) {
    if (less(a[x], a[y])) {
        if (less(a[y], a[z])) swapT(a[result], a[y]);
        else if (less(a[x], a[z])) swapT(a[result], a[z]);
        else swapT(a[result], a[x]);
    } else if (less(a[x], a[z])) {
        swapT(a[result], a[x]);
    } else if (less(a[y], a[z])) {
        swapT(a[result], a[z]);
    } else {
        swapT(a[result], a[y]);
    }
}

template <class T, class Less>
CC_HD int unguardedPartition(T* a, int lo, int hi, int pivot, Less less) {
    while (true) {
        while (less(a[lo], a[pivot])) ++lo;
        --hi;
        while (less(a[pivot], a[hi])) --hi;
        if (!(lo < hi)) return lo;
        swapT(a[lo], a[hi]);
        ++lo;
    }
}

template <class T, class Less>
CC_HD void unguardedLinearInsert(T* a, int last, Less less) {
    T v = a[last];
    int next = last - 1;
    while (less(v, a[next])) {
        a[last] = a[next];
        last = next;
        --next;
    }
    a[last] = v;
}

template <class T, class Less>
CC_HD void insertionSort(T* a, int first, int last, Less less) {
    if (first == last) return;
    for (int i = first + 1; i != last; ++i) {
        if (less(a[i], a[first])) {
            T v = a[i];
            for (int k = i; k > first; --k) a[k] = a[k - 1];
            a[first] = v;
        } else {
            unguardedLinearInsert(a, i, less);
        }
    }
}

CC_HD int floorLog2(int n) { return 31 - __builtin_clz(unsigned(n)); }

constexpr int kSortThreshold = 16;

// Partitioning phase of introsort on [first, last): leaves every segment of
// at most 16 elements unsorted (or heap-sorted when the depth limit runs out).
template <class T, class Less>
CC_HD void introsortLoop(T* a, int first, int last, int depthLimit, Less less) {
    struct Seg { int first, last, depth; };
    Seg stack[72];
    int sp = 0;
    stack[sp++] = Seg{first, last, depthLimit};
    while (sp > 0) {
        Seg s = stack[--sp];
        int f = s.first, l = s.last, d = s.depth;
        while (l - f > kSortThreshold) {
            if (d == 0) {
                makeHeap(a + f, l - f, less);
                sortHeap(a + f, l - f, less);
                break;
            }
            --d;
            int mid = f + (l - f) / 2;
            moveMedianToFirst(a, f, f + 1, mid, l - 1, less);
            int cut = unguardedPartition(a, f + 1, l, f, less);
            stack[sp++] = Seg{cut, l, d};
            l = cut;
        }
    }
}

template <class T, class Less>
CC_HD void finalInsertionSort(T* a, int n, Less less) {
    if (n > kSortThreshold) {
        insertionSort(a, 0, kSortThreshold, less);
        for (int i = kSortThreshold; i < n; ++i) unguardedLinearInsert(a, i, less);
    } else {
        insertionSort(a, 0, n, less);
    }
}

template <class T, class Less>
CC_HD void introsort(T* a, int n, Less less) {
    if (n == 0) return;
    introsortLoop(a, 0, n, 2 * floorLog2(n), less);
    finalInsertionSort(a, n, less);
}

// ----- Huffman tree -----
// Heap element: probability in the high 32 bits, node id in the low 32 bits.
// "less" follows HuffmanDesign.h:42-51: a < b  iff  b.prob < a.prob, so the
// heap top is the node with the smallest probability.
struct ProbInvLess {
    CC_HD bool operator()(u64 a, u64 b) const { return u32(b >> 32) < u32(a >> 32); }
};

// Sort element: codeword length in bits 27..31, leaf index in bits 0..26.
struct LenLess {
    CC_HD bool operator()(u32 a, u32 b) const { return (a >> 27) < (b >> 27); }
};
constexpr u32 kLeafMask = (1u << 27) - 1u;

// Runs the priority-queue merge of HuffmanTable.cu:507-529.  Input: heap[i] =
// (prob_i << 32) | i for the L leaves in symbol order.  Output: parent[id] for
// every node id in [0, 2L-1) except the root (2L-2, or 0 when L == 1).
CC_HD void buildTree(u64* heap, u32* parent, int L) {
    ProbInvLess less;
    makeHeap(heap, L, less);
    int len = L;
    u32 next = u32(L);
    while (len > 1) {
        u64 a = heap[0];
        popHeap(heap, len, less);
        --len;
        u64 b = heap[0];
        popHeap(heap, len, less);
        --len;
        u32 id = next++;
        parent[u32(a)] = id;
        parent[u32(b)] = id;
        u64 p = u64(u32(a >> 32) + u32(b >> 32));
        heap[len] = (p << 32) | id;
        ++len;
        pushHeap(heap, len, less);
    }
}

// Depth of every node from the parent links (HuffmanDesign.h:27-39 assigns
// length = tree depth).  Children always have smaller ids than their parent,
// so one pass from the root downwards suffices.
CC_HD void nodeDepths(const u32* parent, u8* depth, int L) {
    int nodes = 2 * L - 1;
    depth[nodes - 1] = 0;
    for (int id = nodes - 2; id >= 0; --id) {
        u32 d = u32(depth[parent[id]]) + 1u;
        depth[id] = u8(d > 255u ? 255u : d);   // saturate; lengths > 31 are rejected anyway
    }
}

}  // namespace hb
}  // namespace ccb
