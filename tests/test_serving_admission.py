"""Host-side admission logic of the brick service (cudacompress_b200.serving),
on the CPU: a launch takes requests in arrival order while they fit the
slots and the HBM budget, and a budget that cannot hold the resident store
plus one request of the largest edge is rejected up front."""
import pytest

pytest.importorskip("torch")

from cudacompress_b200 import serving  # noqa: E402


def test_admit_in_order_within_slots_and_budget():
    b32, b64 = serving.request_bytes(32), serving.request_bytes(64)
    assert serving.admit([b32] * 10, 6, 10 * b64) == 6             # slots bind
    assert serving.admit([b32] * 10, 16, 3 * b32) == 3             # budget binds
    assert serving.admit([b64, b32, b32], 4, b64 + b32 - 1) == 1   # stops at the first misfit, never skips ahead
    assert serving.admit([b64], 4, b64 - 1) == 0
    assert serving.admit([], 4, b64) == 0


def test_budget_validation():
    serving.validate_budget(100, [32, 64], 100 + serving.request_bytes(64))
    with pytest.raises(ValueError):
        serving.validate_budget(100, [32, 64], 99 + serving.request_bytes(64))
    with pytest.raises(ValueError):
        serving.validate_budget(4 << 30, [128], 4 << 30)           # the store alone fills the budget


def test_fill_levels_are_powers_of_two_and_the_slot_count():
    assert serving.fill_levels(64) == [1, 2, 4, 8, 16, 32, 64]
    assert serving.fill_levels(12) == [1, 2, 4, 8, 12]
    assert serving.fill_levels(1) == [1]
    assert serving.fill_level(0, 16) == 0
    assert serving.fill_level(7, 16) == 4      # the rest waits for the lane's other codec
    assert serving.fill_level(16, 16) == 16
    assert serving.fill_level(11, 12) == 8
    assert serving.fill_level(12, 12) == 12
