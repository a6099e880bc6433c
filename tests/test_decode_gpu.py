"""GPU decode parity: the CUDA decoder against the oracle and against the
reference's hand-built golden frames, bit for bit; errors by kind and text."""

import random

import numpy as np
import pytest

import rivet_prores_b200 as P
from oracle import oracle as O
from tests import handbuilt_frames as H
from tests.util import assert_decode_matches

pytestmark = pytest.mark.gpu


def test_hand_coded_macroblock():
    # tests/handbuilt.rs:230-280
    f = P.Decoder.new().decode(H.macroblock_frame())
    assert f.bit_depth == 10 and (f.width, f.height) == (16, 16)
    assert f.plane2d(0).tolist() == H.macroblock_expected_luma()
    assert (f.plane(1) == 512).all()
    assert (f.plane(2) == H.sample(-2.0)).all()


def test_field_pictures_are_woven():
    # tests/handbuilt.rs:285-327
    for mode, first_row, data in H.field_frames():
        f = P.Decoder.new().decode(data)
        assert f.interlace.value == mode
        y = f.plane2d(0)
        assert (y[first_row] == H.sample(4.0)).all()
        assert (y[1 - first_row] == H.sample(-4.0)).all()


def test_hand_coded_alpha():
    # tests/handbuilt.rs:332-361
    f = P.Decoder.with_bit_depth(8).decode(H.alpha_frame())
    a = f.alpha
    assert (a[:16] == 255).all() and (a[16:255] == 0).all() and a[255] == 10
    assert (f.data == 128).all()


def test_malformed_frames_fail_like_the_oracle():
    # tests/handbuilt.rs:363-424
    frames = H.malformed_frames()
    got = P.Decoder.new().decode_batch([d for _, d, _ in frames])
    for (name, data, _), r in zip(frames, got):
        assert_decode_matches(r, O.decode(data), name)


def _cases():
    """(config, picture) pairs over formats, sizes, field orders, slice
    widths, depths, alpha and matrices, encoded by the oracle."""
    out = []
    rng = random.Random(3)
    sizes = [(1, 1), (2, 2), (17, 9), (31, 33), (48, 16), (100, 37), (129, 75), (250, 19), (64, 64), (352, 288)]
    for (w, h) in sizes:
        for chroma, profile, depth in [(2, 3, 10), (3, 4, 12)]:
            interlace = rng.randrange(3)
            log2 = rng.randrange(4)
            p = O.test_frame(w, h, chroma, depth, 6, w * 131 + h)
            p.interlace = interlace
            out.append((O.Config(profile, log2_slice_mbs=log2, target_frame_bytes=1 << 30), p))
    # Alpha, both widths, off the macroblock grid (tests/roundtrip.rs:332-357).
    for (w, h), bits in [((100, 40), 1), ((33, 17), 2), ((97, 41), 2), ((24, 24), 1)]:
        p = O.test_frame(w, h, 3, 12, 4, 5)
        p.interlace = rng.randrange(3)
        p.alpha = np.array([(y * 4095 // max(h - 1, 1)) if x % 20 < 10 else (x * 37 + y) % 4096
                            for y in range(h) for x in range(w)], np.uint16)
        out.append((O.Config(4, alpha=bits), p))
    # Loaded matrices and a tight target.
    luma = bytes(4 + 2 * (u + v) for v in range(8) for u in range(8))
    chroma_m = bytes(6 + 3 * (u + v) for v in range(8) for u in range(8))
    p = O.test_frame(320, 180, 2, 10, 8, 21)
    out.append((O.Config(3, luma_matrix=luma, chroma_matrix=chroma_m), p))
    p = O.test_frame(320, 180, 2, 10, 30, 22)
    out.append((O.Config(0, target_frame_bytes=20000), p))
    return out


@pytest.fixture(scope="module")
def packets():
    res = []
    for cfg, pic in _cases():
        k, msg, pkt = O.encode(cfg, pic)
        assert k == 0, msg
        res.append(pkt)
    return res


def test_round_trip_frames_decode_bit_exact(packets):
    for depth in [0, 8, 10, 12, 16]:
        got = P.Decoder(bit_depth=depth or None).decode_batch(packets)
        for i, (pkt, r) in enumerate(zip(packets, got)):
            assert_decode_matches(r, O.decode(pkt, depth), f"case {i} depth {depth}")


def test_one_frame_alone_equals_in_a_batch(packets):
    batch = P.Decoder.new().decode_batch(packets)
    for pkt, b in zip(packets, batch):
        one = P.Decoder.new().decode(pkt)
        assert np.array_equal(one.data, b.data)


def test_readme_frames_decode_bit_exact():
    """The 1080p round-trip frames of README.md:175-180 (all six profiles)."""
    pkts, oracles = [], []
    for profile in range(6):
        chroma, depth = (3, 12) if profile >= 4 else (2, 10)
        f = O.test_frame(1920, 1080, chroma, depth, 24, 7)
        k, msg, pkt = O.encode(O.Config(profile), f)
        pkts.append(pkt)
        oracles.append(O.decode(pkt, depth))
    got = P.Decoder.new().decode_batch(pkts)
    for i, (r, o) in enumerate(zip(got, oracles)):
        assert_decode_matches(r, o, f"profile {i}")


def _mutations(seed_packets, n, rng):
    out = []
    for _ in range(n):
        d = bytearray(seed_packets[rng.randrange(len(seed_packets))])
        kind = rng.randrange(4)
        if kind == 0:
            for _ in range(rng.randint(1, 12)):
                d[rng.randrange(len(d))] = rng.randrange(256)
        elif kind == 1:
            for _ in range(rng.randint(1, 8)):
                bit = rng.randrange(len(d) * 8)
                d[bit // 8] ^= 0x80 >> (bit % 8)
        elif kind == 2:
            d = d[: rng.randrange(len(d))]
        else:
            at = rng.randrange(len(d))
            d = d[:at] + bytes(rng.randrange(256) for _ in range(rng.randint(0, 64))) + d[at:]
        out.append(bytes(d))
    return out


def test_damaged_frames_fail_like_the_oracle():
    """tests/fuzz.rs:46-97: changed bytes, flipped bits, cuts and splices; the
    GPU gives the oracle's error (kind and text) or the oracle's picture."""
    seeds = []
    f = O.test_frame(40, 24, 2, 10, 20, 1)
    seeds.append(O.encode(O.Config(2), f)[2])
    f = O.test_frame(33, 21, 3, 12, 20, 2)
    f.interlace = 1
    f.alpha = (np.arange(33 * 21) * 7 % 4096).astype(np.uint16)
    seeds.append(O.encode(O.Config(5, luma_matrix=bytes([5] * 64), chroma_matrix=bytes([9] * 64)), f)[2])
    f.interlace = 0
    seeds.append(O.encode(O.Config(4, alpha=1, log2_slice_mbs=0), f)[2])
    rng = random.Random(1234)
    cases = _mutations(seeds, 600, rng)
    got = P.Decoder.new().decode_batch(cases)
    for i, (d, r) in enumerate(zip(cases, got)):
        assert_decode_matches(r, O.decode(d), f"mutation {i}")


def test_extreme_coefficients_decode_like_the_oracle():
    """Slices whose levels and DCs reach the ends of the coded range (the
    reference's dsp extremes, src/dsp/mod.rs:458-489), built with the
    oracle's entropy coder into an otherwise valid 4:4:4 frame."""
    rng = random.Random(9)
    import struct

    frames = []
    for case in range(40):
        comps = []
        for _ in range(3):
            c = np.zeros(4 * 64, np.int32)
            for i in range(c.size):
                r = rng.randrange(20)
                if i < 4 or rng.randrange(3) == 0:
                    c[i] = (rng.randint(-(1 << 29), 1 << 29) if r == 0 else
                            rng.randint(-2048, 2047) if r < 5 else rng.randint(-8, 8))
            if case % 3 == 0:
                c[0] = (1 << 30) - 7
            data, _ = O.encode_coefficients(c, 4)
            comps.append(data)
        qi = rng.choice([1, 64, 128, 200, 224])
        s = bytearray([6 << 3, qi]) + struct.pack(">HH", len(comps[0]), len(comps[1]))
        s += comps[0] + comps[1] + comps[2]
        hdr = bytearray(H.frame_header(16, 16, 3, 0, 0, 1, 0))
        hdr[19] = 2  # a loaded luma matrix follows
        hdr[0:2] = struct.pack(">H", 20 + 64)
        hdr += bytes(rng.randint(2, 63) for _ in range(64))
        frames.append(H.frame(bytes(hdr), [H.picture(0, [bytes(s)])], 0, 0))
    for depth in [8, 12, 16]:
        got = P.Decoder(bit_depth=depth).decode_batch(frames)
        for i, (d, r) in enumerate(zip(frames, got)):
            assert_decode_matches(r, O.decode(d, depth), f"extreme {i} depth {depth}")
