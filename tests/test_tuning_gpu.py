"""Launch shapes change no output: decoding and encoding a batch of mixed
frames under extreme tunings gives the bytes and samples of the default
shapes, which equal the oracle's."""

import numpy as np
import pytest

import rivet_prores_b200 as P
from oracle import oracle as O
from tests.util import to_config, to_frame

pytestmark = pytest.mark.gpu

SHAPES = [
    P.Tuning(),
    P.Tuning(cost_lane_items_per_sm=0, entropy_warps_per_block=1, entropy_blocks_per_sm=1,
             entropy_components_per_lane=4, staging_depth=1, decode_fused=0),
    P.Tuning(cost_lane_items_per_sm=1 << 30, entropy_warps_per_block=16, entropy_blocks_per_sm=0,
             entropy_components_per_lane=2, staging_depth=64, decode_fused=0),
    P.Tuning(cost_lane_items_per_sm=0, entropy_warps_per_block=3, entropy_blocks_per_sm=2,
             entropy_components_per_lane=1, staging_depth=3, decode_fused=0),
    # The fused decoder from one slice a CTA up to the most its shared memory takes.
    P.Tuning(decode_slot_positions=512),
    P.Tuning(decode_slot_positions=6144),
    P.Tuning(decode_slot_positions=65536),
    P.Tuning(decode_slot_positions=512, decode_slot_bytes=1),
    P.Tuning(decode_slot_positions=65536, decode_slot_bytes=1),
]


def _cases():
    cases = []
    kinds = [(352, 288, 2, 10, 3, 0), (200, 120, 3, 12, 4, 1), (720, 486, 2, 10, 3, 2), (97, 41, 3, 12, 5, 0),
             (1280, 720, 2, 10, 1, 0)]
    for i, (w, h, chroma, depth, profile, il) in enumerate(kinds):
        pic = O.test_frame(w, h, chroma, depth, 12, 40 + i)
        pic.interlace = il
        cfg = O.Config(profile)
        cfg.log2_slice_mbs = (3 - i) % 4
        cases.append((cfg, pic))
    return cases


def test_outputs_do_not_depend_on_the_tuning():
    ctx = P.context(0)
    saved = ctx.tuning
    cases = _cases()
    frames = [to_frame(p) for _, p in cases]
    configs = [to_config(c) for c, _ in cases]
    try:
        results = []
        for t in SHAPES:
            ctx.set_tuning(t)
            assert ctx.tuning == t
            packets = P.Encoder(configs[0]).encode_batch(frames, configs)
            decoded = P.Decoder.new().decode_batch(packets)
            results.append((packets, [d.data.copy() for d in decoded]))
        for packets, planes in results[1:]:
            assert packets == results[0][0]
            assert all(np.array_equal(a, b) for a, b in zip(planes, results[0][1]))
        for (cfg, pic), pk, planes in zip(cases, results[0][0], results[0][1]):
            k, msg, want = O.encode(cfg, pic)
            assert k == O.OK, msg
            assert pk == want
            k, msg, back = O.decode(want)
            assert k == O.OK, msg
            assert np.array_equal(planes, back.data)
    finally:
        ctx.set_tuning(saved)


def test_out_of_range_tunings_are_refused():
    ctx = P.context(0)
    saved = ctx.tuning
    for bad in [dict(entropy_warps_per_block=0), dict(entropy_warps_per_block=17), dict(entropy_components_per_lane=3),
                dict(staging_depth=0), dict(cost_lane_items_per_sm=-1), dict(entropy_blocks_per_sm=-1),
                dict(decode_fused=2), dict(decode_slot_positions=511), dict(decode_slot_positions=65537),
                dict(decode_slot_bytes=3)]:
        with pytest.raises(P.Error.Config):
            ctx.set_tuning(P.Tuning(**bad))
    assert ctx.tuning == saved


def test_quick_autotune_applies_a_valid_tuning(tmp_path, monkeypatch):
    from rivet_prores_b200 import autotune, workloads

    monkeypatch.setenv(autotune.CACHE_ENV, str(tmp_path / "tuning.json"))
    ctx = P.context(0)
    saved = ctx.tuning
    try:
        frames = [workloads.picture(1920, 1080, P.ChromaFormat.Yuv422, 10, 77 + i) for i in range(4)]
        t, ev = autotune.tune(quick=True, frames=frames, depths=[2, 4])
        assert ctx.tuning == t
        assert autotune.load() == t
        assert {"cost", "decode", "staging"} <= set(ev)
    finally:
        ctx.set_tuning(saved)
