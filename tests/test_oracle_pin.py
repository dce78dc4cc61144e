"""Pins the CPU oracle against the reference's own code built from its
sources (oracle/ref/Makefile -> oracle/_ref/): Huffman table construction and
serialization must match byte for byte, and against the committed golden
vectors made from the reference build."""
import numpy as np
import pytest

from helpers import bind_build, load_oracle, load_ref_gpu_lib, random_histograms, run_build


@pytest.fixture(scope="module")
def oracle():
    return load_oracle()


def test_oracle_tables_match_reference_build(oracle):
    ref = load_ref_gpu_lib()
    if ref is None:
        pytest.skip("reference build (oracle/_ref) not present")
    fo = bind_build(oracle, "orc_huffman_build")
    fr = bind_build(ref, "ref_huffman_build")
    for hist, smax in random_histograms(1500, seed=7):
        log2max = 14 if smax < (1 << 14) else 16
        a = run_build(fo, hist, smax, log2max)
        b = run_build(fr, hist, smax, log2max)
        assert a[0] == b[0] and a[4] == b[4]
        assert np.array_equal(a[3], b[3])
        if hist.any():
            assert np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2])
