"""The autotuner's choices and cache (no GPU): the crossover rule for
lane-per-component costing, the least-time pick, slice counting, and the
JSON cache keyed by GPU."""

import json

import pytest

import rivet_prores_b200 as P
from rivet_prores_b200 import autotune as A


def test_lane_threshold_is_the_smallest_size_from_which_lanes_keep_winning():
    # Warps win at 1 frame, lanes from 4 frames on: 3 x 16200 / 148 rounded up.
    pts = [(4050, 2.0, 1.0), (16200, 3.0, 3.5), (64800, 5.0, 9.0)]
    assert A.lane_threshold(pts, 148) == (3 * 16200 + 147) // 148
    # A win below a loss does not count: lanes must win at every larger size.
    pts = [(4050, 1.0, 2.0), (8100, 3.0, 2.0), (16200, 3.0, 4.0)]
    assert A.lane_threshold(pts, 148) == (3 * 16200 + 147) // 148
    assert A.lane_threshold([(4050, 1.0, 2.0), (8100, 1.0, 3.0)], 148) == 0
    never = A.lane_threshold([(4050, 3.0, 2.0), (8100, 5.0, 4.0)], 148)
    assert 3 * 8100 < never * 148
    with pytest.raises(ValueError):
        A.lane_threshold([], 148)


def test_best_takes_the_least_time_and_the_first_of_ties():
    assert A.best({(4, 0, 1): 2.0, (8, 0, 1): 1.5, (16, 0, 1): 1.5}) == (8, 0, 1)
    with pytest.raises(ValueError):
        A.best({})


def test_slices_follow_the_row_split():
    class F:
        width, height = 3840, 2160

    assert A.slices_in(F) == 135 * 30
    F.width, F.height = 1928, 1080  # 121 MBs: 15 slices of 8 and one of 1
    assert A.slices_in(F) == 68 * 16
    F.width = 1976  # 124 MBs: 15 x 8, then 4
    assert A.slices_in(F, 3) == 68 * 16
    assert A.slices_in(F, 1) == 68 * 62


def test_cache_round_trip(tmp_path, monkeypatch):
    path = tmp_path / "tune" / "tuning.json"
    monkeypatch.setenv(A.CACHE_ENV, str(path))
    assert A.load(key="GPU X|148 SMs") is None
    t = P.Tuning(cost_lane_items_per_sm=300, entropy_warps_per_block=4, entropy_blocks_per_sm=2,
                 entropy_components_per_lane=2, staging_depth=8)
    A.save(t, {"cost": [1]}, key="GPU X|148 SMs")
    A.save(P.Tuning(), {}, key="GPU Y|132 SMs")
    assert A.load(key="GPU X|148 SMs") == t
    assert A.load(key="GPU Y|132 SMs") == P.Tuning()
    data = json.loads(path.read_text())
    assert data["GPU X|148 SMs"]["evidence"] == {"cost": [1]}
    # A damaged cache is ignored, not raised.
    path.write_text("{not json")
    assert A.load(key="GPU X|148 SMs") is None
