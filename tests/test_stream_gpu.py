"""The host round trip (stream.RoundTripPipeline): frames in pinned host
memory, encoded and decoded part by part on their own streams, with the
next step's uploads queued across parts while earlier parts still decode.
Every step must leave the oracle's packets and decoded planes, whatever the
number of parts."""

import numpy as np
import pytest

from oracle import oracle as O
from rivet_prores_b200.stream import RoundTripPipeline
from tests.util import to_config, to_frame

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("depth", [1, 2, 3, 5])
def test_round_trip_pipeline_matches_the_oracle(depth):
    cfg = O.Config(3)
    cfg.log2_slice_mbs = 2
    pics = [O.test_frame(352, 288, 2, 10, 12, 500 + i) for i in range(5)]
    frames = [to_frame(p) for p in pics]
    pipe = RoundTripPipeline(frames, to_config(cfg), depth)
    try:
        for steps in (1, 3):
            start, end = pipe.run(steps)
            pipe.stream.synchronize()
            assert start.elapsed_time(end) > 0
            assert len(pipe.packets) == len(pics)
            for i, (pic, pk) in enumerate(zip(pics, pipe.packets)):
                k, msg, want = O.encode(cfg, pic)
                assert k == O.OK, msg
                assert bytes(pk) == want, f"frame {i}, {steps} steps"
                k, msg, back = O.decode(want)
                assert k == O.OK, msg
                assert np.array_equal(pipe.planes[i], np.asarray(back.data, dtype=np.uint16)), f"frame {i}"
        up, down = pipe.bytes_per_step()
        assert up == down == 2 * pipe.host.size + sum(len(p) for p in pipe.packets)
    finally:
        pipe.close()
