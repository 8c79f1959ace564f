"""Host-side arithmetic of bench.py: the comparator weighting and the volume
pass's algorithmic bytes (no GPU)."""
import math

import pytest

import bench


def test_mix_rate_is_total_steps_over_total_time():
    # half the steps at 100/s and half at 300/s: 1 step takes (0.5/100 + 0.5/300) s
    assert math.isclose(bench._mix_rate({"a": 100.0, "b": 300.0}, {"a": 0.5, "b": 0.5}), 150.0)
    # one class only: its own rate
    assert math.isclose(bench._mix_rate({"a": 42.0, "b": 7.0}, {"a": 1.0}), 42.0)


def test_shares_normalise_step_counts():
    sh = bench._shares({"x": 3, "y": 1})
    assert sh == {"x": 0.75, "y": 0.25}
    d = bench._demand_shares([{"mesh": (64, 32, 16), "steps": 300},
                              {"mesh": (128, 64, 16), "steps": 100},
                              {"mesh": (64, 32, 16), "steps": 100}])
    assert d == {(64, 32, 16): 0.8, (128, 64, 16): 0.2}


@pytest.mark.parametrize("precision, per_mode, per_face", [("mixed", 8, 16), ("fp64", 32, 24)])
def test_volume_pass_bytes(precision, per_mode, per_face):
    # the 288-slot serving batch: 467,927,040 modes over 12,533,760 face columns
    modes, faces = 467927040, 12533760
    assert bench._volume_pass_bytes(modes, faces, precision) == per_mode * modes + per_face * faces
    if precision == "mixed":
        assert bench._volume_pass_bytes(modes, faces, precision) == 3943956480
