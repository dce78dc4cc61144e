"""The product's table builder (huffman_build.cuh), compiled for the host into
the self-test library, must produce the same tables and serialized headers as
the oracle on histograms of every shape."""
import numpy as np
import pytest

from helpers import bind_build, load_oracle, load_selftest, random_histograms, run_build


def test_host_builder_matches_oracle():
    st = load_selftest()
    if st is None:
        pytest.skip("self-test library not built")
    fo = bind_build(load_oracle(), "orc_huffman_build")
    fs = bind_build(st, "ccst_huffman_build")
    for hist, smax in random_histograms(3000, seed=11, max_bins=5000):
        log2max = 14 if smax < (1 << 14) else 16
        a = run_build(fo, hist, smax, log2max)
        b = run_build(fs, hist, smax, log2max)
        if a[0] > 31:
            continue
        assert a[0] == b[0] and a[4] == b[4]
        assert np.array_equal(a[3], b[3])
        if hist.any():
            assert np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2])
