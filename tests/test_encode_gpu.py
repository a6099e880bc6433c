"""GPU encode parity: the CUDA encoder's packets equal the oracle's byte for
byte (same rate control decisions, same bits), alone and batched."""

import random

import numpy as np
import pytest

import rivet_prores_b200 as P
from oracle import oracle as O
from tests.util import KIND, PREFIX, to_config, to_frame

pytestmark = pytest.mark.gpu


def _check_batch(cases):
    frames = [to_frame(p) for _, p in cases]
    configs = [to_config(c) for c, _ in cases]
    got = P.Encoder(configs[0]).encode_batch(frames, configs)
    for i, ((cfg, pic), g) in enumerate(zip(cases, got)):
        k, msg, want = O.encode(cfg, pic)
        if k != O.OK:
            assert isinstance(g, KIND[k]) and g.message == PREFIX[k] + msg, (i, g, msg)
            continue
        assert not isinstance(g, P.Error), (i, g)
        if g != want:
            n = min(len(g), len(want))
            diff = next((j for j in range(n) if g[j] != want[j]), n)
            raise AssertionError(f"case {i}: {len(g)} vs {len(want)} bytes, first difference at {diff}")
    return got


def test_readme_profiles_encode_bit_exact():
    """README.md:175-180: all six profiles at 1080p, the exact byte counts."""
    want = [187_677, 425_420, 613_107, 917_564, 1_376_337, 2_085_373]
    cases = []
    for profile in range(6):
        chroma, depth = (3, 12) if profile >= 4 else (2, 10)
        cases.append((O.Config(profile), O.test_frame(1920, 1080, chroma, depth, 24, 7)))
    got = _check_batch(cases)
    assert [len(g) for g in got] == want


def test_odd_sizes_field_orders_and_slice_widths():
    # tests/roundtrip.rs:140-187, both target regimes
    cases = []
    rng = random.Random(7)
    for (w, h) in [(1, 1), (2, 2), (17, 9), (31, 33), (48, 16), (100, 37), (129, 75), (250, 19)]:
        for chroma, profile in [(2, 3), (3, 4)]:
            for interlace in range(3):
                log2 = rng.randrange(4)
                p = O.test_frame(w, h, chroma, 12 if chroma == 3 else 10, 6, w * 131 + h)
                p.interlace = interlace
                target = (1 << 30) if rng.randrange(2) else None
                cases.append((O.Config(profile, log2_slice_mbs=log2, target_frame_bytes=target), p))
    _check_batch(cases)


def test_rate_control_regimes():
    """Targets that leave the coarsest quantiser too big, targets between, and
    targets loose enough for the finest; per-slice refinement included."""
    cases = []
    for target in [200, 2_000, 8_000, 20_000, 45_000, 90_000, 200_000, 10_000_000]:
        p = O.test_frame(320, 240, 2, 10, 30, target)
        cases.append((O.Config(0, target_frame_bytes=target), p))
        p = O.test_frame(256, 160, 3, 12, 20, target + 1)
        p.interlace = 2
        cases.append((O.Config(5, target_frame_bytes=target, log2_slice_mbs=1), p))
    _check_batch(cases)


def test_every_profile_at_720p_and_depths():
    cases = []
    for profile in range(6):
        chroma = 3 if profile >= 4 else 2
        for depth in [8, 10, 12, 16]:
            cases.append((O.Config(profile), O.test_frame(640, 360, chroma, depth, 12, profile * 10 + depth)))
    _check_batch(cases)


def test_alpha_lossless_and_matrices():
    cases = []
    rng = random.Random(99)
    for (depth, bits) in [(12, 2), (16, 2), (8, 1), (10, 2)]:
        for interlace in [0, 1, 2]:
            p = O.test_frame(97, 41, 3, depth, 4, 5)
            p.interlace = interlace
            mx = (1 << depth) - 1
            a = []
            for y in range(41):
                for x in range(97):
                    k = x // 20
                    a.append(0 if k == 0 else mx if k == 1 else (x * mx // 97) if k == 2 else
                             (rng.randrange(mx + 1) if y < 20 else mx // 2))
            p.alpha = np.array(a, np.uint16)
            cases.append((O.Config(4, alpha=bits), p))
    luma = bytes(4 + 2 * (u + v) for v in range(8) for u in range(8))
    chroma_m = bytes(6 + 3 * (u + v) for v in range(8) for u in range(8))
    for l, c in [(luma, chroma_m), (luma, None), (None, chroma_m), (bytes([2] * 64), bytes([2] * 64))]:
        cases.append((O.Config(3, luma_matrix=l, chroma_matrix=c), O.test_frame(320, 180, 2, 10, 8, 21)))
    # A vertical alpha ramp off the macroblock grid (tests/roundtrip.rs:332-357).
    for (w, h) in [(640, 360), (100, 40), (33, 17), (16, 8)]:
        p = O.test_frame(w, h, 3, 8, 2, w ^ h)
        p.alpha = np.array([y * 255 // (h - 1) for y in range(h) for _ in range(w)], np.uint16)
        p.interlace = 2
        cases.append((O.Config(5, alpha=1), p))
    _check_batch(cases)


def test_flat_and_extreme_pictures():
    cases = []
    for profile in range(6):
        chroma, depth = (3, 12) if profile >= 4 else (2, 10)
        p = O.test_frame(1920, 1080, chroma, depth, 0, 1)
        p.data[:] = 1 << (depth - 1)
        cases.append((O.Config(profile), p))
    p = O.test_frame(64, 32, 2, 10, 0, 1)
    planes = O.plane_layout(64, 32, 2)
    for off, w, h in planes:
        idx = np.arange(w * h)
        p.data[off:off + w * h] = np.where(((idx % w) // 3) % 2 == 0, 0, 1023)
    cases.append((O.Config(0), p))
    _check_batch(cases)


def test_config_errors_match_the_oracle():
    # tests/roundtrip.rs:467-515
    f422 = O.test_frame(32, 32, 2, 10, 0, 1)
    f444 = O.test_frame(32, 32, 3, 12, 0, 1)
    with_alpha = O.test_frame(32, 32, 2, 10, 0, 1)
    with_alpha.alpha = np.zeros(32 * 32, np.uint16)
    short_alpha = O.test_frame(32, 32, 3, 12, 0, 1)
    short_alpha.alpha = np.zeros(10, np.uint16)
    truncated = O.test_frame(32, 32, 2, 10, 0, 1)
    truncated.data = truncated.data[:100]
    alpha_off = O.test_frame(32, 32, 3, 12, 0, 1)
    alpha_off.alpha = np.full(32 * 32, 7, np.uint16)
    cases = [
        (O.Config(3), f444), (O.Config(4), f422), (O.Config(3), with_alpha), (O.Config(4), short_alpha),
        (O.Config(3, luma_matrix=bytes([1] * 64)), f422), (O.Config(3, log2_slice_mbs=4), f422),
        (O.Config(3), truncated), (O.Config(4, alpha=0), alpha_off), (O.Config(3), f422),
    ]
    # to_frame needs whole planes; the truncated frame goes in as given.
    frames = []
    for _, p in cases:
        f = P.Frame(p.width, p.height, p.bit_depth, P.ChromaFormat(p.chroma), P.Interlace(p.interlace),
                    P.Metadata(*p.metadata), np.array(p.data, np.uint16), None,
                    None if p.alpha is None else np.array(p.alpha, np.uint16))
        frames.append(f)
    configs = [to_config(c) for c, _ in cases]
    got = P.Encoder(configs[0]).encode_batch(frames, configs)
    for i, ((cfg, pic), g) in enumerate(zip(cases, got)):
        k, msg, want = O.encode(cfg, pic)
        if k != O.OK:
            assert isinstance(g, KIND[k]) and g.message == PREFIX[k] + msg, (i, g, msg)
        else:
            assert g == want, i


def test_round_trip_through_both_gpu_paths():
    cases = []
    for profile in [0, 3, 4, 5]:
        chroma, depth = (3, 12) if profile >= 4 else (2, 10)
        p = O.test_frame(720, 486, chroma, depth, 10, profile)
        p.interlace = 2
        cases.append((O.Config(profile), p))
    got = _check_batch(cases)
    dec = P.Decoder.new().decode_batch(got)
    for (cfg, pic), d, pkt in zip(cases, dec, got):
        k, msg, want = O.decode(pkt)
        assert np.array_equal(d.data, want.data)
