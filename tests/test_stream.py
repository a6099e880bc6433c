"""Host-side checks of the round-trip pipeline that need no GPU: it refuses
work it cannot stream before touching the device."""

import pytest

import rivet_prores_b200 as P
from oracle import oracle as O
from rivet_prores_b200.stream import RoundTripPipeline, frames_per_second
from tests.util import to_frame


def test_round_trip_pipeline_refuses_mixed_sizes():
    frames = [to_frame(O.test_frame(64, 48, 2, 10, 12, 1)), to_frame(O.test_frame(80, 48, 2, 10, 12, 2))]
    with pytest.raises(ValueError):
        RoundTripPipeline(frames, P.Config(P.Profile.Hq), 2)


def test_round_trip_pipeline_refuses_an_empty_batch():
    with pytest.raises(ValueError):
        RoundTripPipeline([], P.Config(P.Profile.Hq), 2)


def test_frames_per_second():
    assert frames_per_second(32, 16.0) == pytest.approx(2000.0)
    assert frames_per_second(32, None) == 0.0
