"""The table builder's heap replay (table_build.cuh: blockMakeHeap, popTop,
pushLast) restated step for step in Python - make_heap one depth at a time
in any order inside a depth, the two-level sift-down with speculative
grandchild loads, the push-up against the values still in registers, the
push with three ancestors per step - and checked against a literal
restatement of libstdc++'s make_heap / pop_heap / push_heap (the reference's
std::priority_queue, HuffmanTable.cu:507-529) on tie-heavy inputs: the heap
contents after every operation and the resulting parent links must be
identical."""
import numpy as np

def prob(e):
    return e >> 32


def less(a, b):           # ProbInvLess: b.prob < a.prob
    return prob(b) < prob(a)


# ---------------------------------------------------------------- libstdc++
def push_hole(a, hole, top, v):
    parent = (hole - 1) // 2
    while hole > top and less(a[parent], v):
        a[hole] = a[parent]
        hole = parent
        parent = (hole - 1) // 2
    a[hole] = v


def adjust_heap(a, hole, n, v):
    top = hole
    child = hole
    while child < (n - 1) // 2:
        child = 2 * (child + 1)
        if less(a[child], a[child - 1]):
            child -= 1
        a[hole] = a[child]
        hole = child
    if (n & 1) == 0 and child == (n - 2) // 2:
        child = 2 * (child + 1)
        a[hole] = a[child - 1]
        hole = child - 1
    push_hole(a, hole, top, v)


def make_heap(a, n):
    if n < 2:
        return
    parent = (n - 2) // 2
    while True:
        adjust_heap(a, parent, n, a[parent])
        if parent == 0:
            return
        parent -= 1


def seq_pop(a, n):
    top = a[0]
    if n > 1:
        v = a[n - 1]
        a[n - 1] = a[0]
        adjust_heap(a, 0, n - 1, v)
    return top


def seq_push(a, n, v):
    a[n - 1] = v
    push_hole(a, n - 1, 0, v)


# ------------------------------------------------------- parallel restatement
def block_make_heap(a, n, rng):
    if n < 2:
        return
    last_parent = (n - 2) // 2
    for d in range((last_parent + 1).bit_length() - 1, -1, -1):
        first = (1 << d) - 1
        if first > last_parent:
            continue
        nodes = list(range(first, min(2 * first, last_parent) + 1))
        rng.shuffle(nodes)                       # order inside a depth must not matter
        for p in nodes:
            adjust_heap(a, p, n, a[p])


def pop_top(a, n):
    """popTop on the 0-based list a (heap of n + 1 elements)."""
    top = a[0]
    if n <= 0:
        return top
    v = a[n]
    lim = (n - 1) // 2
    hole = 0
    w1 = w2 = None
    while hole < lim:
        c = 2 * hole + 2                      # right child (0-based)
        left_e, right_e = a[c - 1], a[c]
        gl = (a[2 * c - 1], a[2 * c]) if 2 * c < len(a) else None          # children of c - 1
        gr = (a[2 * c + 1], a[2 * c + 2]) if 2 * c + 2 < len(a) else None  # children of c
        left = prob(left_e) < prob(right_e)
        cv = left_e if left else right_e
        a[hole] = cv
        hole = c - 1 if left else c
        w2, w1 = w1, cv
        if hole >= lim:
            break
        q = gl if left else gr
        left2 = prob(q[0]) < prob(q[1])
        cv2 = q[0] if left2 else q[1]
        a[hole] = cv2
        hole = 2 * hole + (1 if left2 else 2)
        w2, w1 = w1, cv2
    if n % 2 == 0 and hole == (n - 2) // 2:
        cv = a[2 * hole + 1]
        a[hole] = cv
        hole = 2 * hole + 1
        w2, w1 = w1, cv
    if hole > 0 and prob(v) < prob(w1):
        a[hole] = w1
        hole = (hole - 1) // 2
        if hole > 0 and prob(v) < prob(w2):
            a[hole] = w2
            hole = (hole - 1) // 2
            while hole > 0:
                parent = (hole - 1) // 2
                pe = a[parent]
                if not prob(v) < prob(pe):
                    break
                a[hole] = pe
                hole = parent
    a[hole] = v
    return top


def push_last(a, ln, v):
    hole = ln - 1
    while hole > 0:
        p1 = (hole - 1) // 2
        p2 = (p1 - 1) // 2 if p1 > 0 else 0
        p3 = (p2 - 1) // 2 if p2 > 0 else 0
        e1, e2, e3 = a[p1], a[p2], a[p3]
        if not prob(v) < prob(e1):
            break
        a[hole] = e1
        hole = p1
        if hole == 0 or not prob(v) < prob(e2):
            break
        a[hole] = e2
        hole = p2
        if hole == 0 or not prob(v) < prob(e3):
            break
        a[hole] = e3
        hole = p3
    a[hole] = v


# ---------------------------------------------------------------- the test
def build(keys, parallel, rng):
    a = list(keys) + [0, 0]
    n = len(keys)
    if parallel:
        block_make_heap(a, n, rng)
    else:
        make_heap(a, n)
    states = [a[:n]]
    parent = {}
    ln, nxt = n, n
    while ln > 1:
        x = pop_top(a, ln - 1) if parallel else seq_pop(a, ln)
        ln -= 1
        y = pop_top(a, ln - 1) if parallel else seq_pop(a, ln)
        ln -= 1
        parent[x & 0xffffffff] = nxt
        parent[y & 0xffffffff] = nxt
        node = ((prob(x) + prob(y)) << 32) | nxt
        nxt += 1
        ln += 1
        if parallel:
            push_last(a, ln, node)
        else:
            seq_push(a, ln, node)
        states.append(a[:ln])
    return states, parent


def test_parallel_heap_replay_matches_libstdcxx():
    rng = np.random.default_rng(2024)
    cases = 0
    for trial in range(160):
        n = int(rng.choice([1, 2, 3, 4, 5, 6, 7, 62, 63, 64, 65, 126, 127, 128, 129])) if trial < 40 \
            else int(rng.integers(1, 700))
        span = int(rng.choice([1, 2, 3, 8, 50, 1 << 20]))          # few distinct values: many ties
        probs = rng.integers(1, span + 1, size=n)
        if trial % 7 == 0:
            probs = np.sort(probs)[::-1] if trial % 2 else np.sort(probs)
        keys = [(int(p) << 32) | i for i, p in enumerate(probs)]
        s1, p1 = build(keys, False, rng)
        s2, p2 = build(keys, True, rng)
        assert s1 == s2, (trial, n, span)
        assert p1 == p2
        cases += 1
    assert cases == 160
    # larger heaps
    for n, span in ((4200, 3), (4500, 1 << 20)):
        probs = rng.integers(1, span + 1, size=n)
        keys = [(int(p) << 32) | i for i, p in enumerate(probs)]
        s1, p1 = build(keys, False, rng)
        s2, p2 = build(keys, True, rng)
        assert s1 == s2 and p1 == p2, n
