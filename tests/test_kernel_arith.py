"""Integer arithmetic the CUDA kernels take from float hardware, checked
exhaustively on the CPU with IEEE float32 (round to nearest, as the device's
__frcp_rn and fmul)."""
import numpy as np


def test_reciprocal_quotient_is_exact():
    """dwt.cu quotient(): floor(k / d) = trunc((k + 1/2) * rn(1/d)) for every
    0 <= k < 2^14 and 1 <= d <= 2^13 (the row pass uses k < 1024, d <= 1024)."""
    k = np.arange(1 << 14, dtype=np.int64)
    kf = k.astype(np.float32) + np.float32(0.5)
    for d in range(1, (1 << 13) + 1):
        r = np.float32(1.0) / np.float32(d)
        q = np.trunc(kf * r).astype(np.int64)
        assert np.array_equal(q, k // d), d


def test_branch_free_dequantizer_is_exact():
    """dwt.cu dequantSym(): (float(q) + sign(q) * 0.5) * step equals
    (float(m) * 0.5) * step, m = 0, s + 1 or -(s + 2) for a zero, even or odd
    symbol s, for every 16-bit symbol and steps across the float range."""
    s = np.arange(1 << 16, dtype=np.int64)
    neg = s & 1
    q = (1 - 2 * neg) * ((s + neg) >> 1)
    m = np.where(s == 0, 0, np.where(neg == 1, -(s + 2), s + 1))
    rng = np.random.default_rng(5)
    steps = np.concatenate([np.float32([1.0, 0.5, 1e-3, 3.7e-2, 1e-30, 1e30]),
                            (10.0 ** rng.uniform(-20, 20, 200)).astype(np.float32)])
    half = np.float32(0.5)
    qf = q.astype(np.float32) + np.sign(q).astype(np.float32) * half
    mf = m.astype(np.float32) * half
    assert np.array_equal(qf, mf)
    for st in steps:
        a = qf * np.float32(st)
        b = mf * np.float32(st)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), st
