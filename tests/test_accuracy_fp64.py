"""The FP64 restatement of the float DWT behind the error report
(cudacompress_b200/accuracy.py) against the oracle's FP64 DWT
(orc_dwt_double_*: the reference's taps promoted to double, double FMA
chain), on the CPU."""
import numpy as np
import pytest

from helpers import Oracle

torch = pytest.importorskip("torch")

from cudacompress_b200 import accuracy  # noqa: E402


@pytest.mark.parametrize("shape", [(16, 24, 32), (8, 8, 8), (40, 56)])
@pytest.mark.parametrize("inverse", [False, True])
def test_fp64_dwt_matches_oracle(shape, inverse):
    rng = np.random.default_rng(11)
    a = rng.standard_normal(shape)
    want = Oracle().dwt_double(a, inverse=inverse)
    got = accuracy.dwt_fp64(torch.from_numpy(a), inverse=inverse).numpy()
    # the same products, summed in another order
    assert np.max(np.abs(got - want)) < 1e-13 * max(1.0, np.max(np.abs(want)))


def test_fp64_multilevel_round_trip():
    rng = np.random.default_rng(12)
    a = torch.from_numpy(rng.standard_normal((32, 32, 32)))
    coef = accuracy.multilevel_fp64(a, 3)
    back = accuracy.multilevel_fp64(coef, 3, inverse=True)
    # the taps are 7-digit float constants: near, not exact, reconstruction
    assert float((back - a).abs().max()) < 1e-4
    lvl1 = accuracy.dwt_fp64(a)
    assert torch.equal(coef[16:, :, :], lvl1[16:, :, :])   # level 0's z-high half is untouched later
