"""The process-wide tuning interface (CPU): round trip and validation."""
import pytest


def test_tuning_round_trip_and_validation():
    from nect_b200 import autotune

    before = autotune.get_tuning()
    try:
        assert before["forward_blocks_per_sm"] == 6 and before["backward_blocks_per_sm"] == 3
        assert before["staged_rounds"] == 4
        assert before["time_slice"] == 1 and before["encoding_store"] == 1
        autotune.set_tuning({"staged_rounds": 16, "run_threshold_3d": 0.5, "scatter_group_bytes": 8 << 20})
        now = autotune.get_tuning()
        assert now["staged_rounds"] == 16 and now["run_threshold_3d"] == 0.5 and now["scatter_group_bytes"] == 8 << 20
        for bad in ({"forward_blocks_per_sm": 0}, {"forward_blocks_per_sm": 7}, {"backward_blocks_per_sm": 4},
                    {"staged_rounds": 65}, {"scatter_group_bytes": 1000}, {"run_threshold_4d": -1.0}, {"encoding_store": 2}):
            with pytest.raises(RuntimeError):
                autotune.set_tuning(bad)
        assert autotune.get_tuning() == now   # a rejected setting changes nothing
    finally:
        autotune.set_tuning(before)
