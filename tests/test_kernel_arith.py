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
