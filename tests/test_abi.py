"""The C ABI without a GPU: the library loads, exports every declared entry
point, and its host-side logic (header parsing, the size guard, target
sizes) agrees with the oracle. No kernel runs here."""

import ctypes
import random

import numpy as np
import pytest

import rivet_prores_b200 as P
from rivet_prores_b200 import _abi
from tests import handbuilt_frames as H


def test_library_exports_every_declared_function():
    L = _abi.lib()
    names = _abi.declared_functions()
    assert len(names) >= 25
    for n in names:
        assert hasattr(L, n), n


def test_target_frame_bytes_matches_the_oracle(oracle):
    rng = random.Random(5)
    sizes = [(1920, 1080), (1280, 720), (3840, 2160), (4096, 2160), (720, 486), (1, 1), (16, 16), (65535, 65535)]
    sizes += [(rng.randint(1, 5000), rng.randint(1, 5000)) for _ in range(200)]
    for p in range(6):
        for w, h in sizes:
            assert P.Profile(p).target_frame_bytes(w, h) == oracle.target_frame_bytes(p, w, h), (p, w, h)
    assert P.Profile.Hq.target_frame_bytes(1920, 1080) == 917_583


def test_profiles_and_fourccs():
    # src/encode.rs:988-995
    for p in P.Profile.ALL:
        assert P.Profile.from_fourcc(p.fourcc()) is p
    assert P.Profile.Hq.fourcc() == b"apch"
    assert P.Profile.P4444Xq.chroma() is P.ChromaFormat.Yuv444


def test_frame_header_parse_of_the_hand_built_frame():
    # tests/handbuilt.rs:241-251
    data = H.macroblock_frame()
    h = P.FrameHeader.parse(data)
    assert h.header_size == 24
    assert h.frame_size == len(data) - 7
    assert h.encoder_identifier == b"hand"
    assert (h.width, h.height, h.chroma, h.interlace) == (16, 16, P.ChromaFormat.Yuv422, P.Interlace.Progressive)
    assert h.metadata.aspect_ratio == 1 and h.metadata.frame_rate() == (25, 1)
    assert h.alpha is P.AlphaType.None_


def test_field_heights_split_an_odd_frame_height():
    # src/header.rs:336-361, through a parsed interlaced header
    hdr = bytearray(H.frame_header(720, 487, 2, 1, 0, 0, 0))
    data = H.frame(bytes(hdr), [], 0, 0)
    h = P.FrameHeader.parse(data)
    assert (h.picture_height(0), h.picture_height(1)) == (244, 243)
    hdr = bytearray(H.frame_header(720, 487, 2, 2, 0, 0, 0))
    h = P.FrameHeader.parse(H.frame(bytes(hdr), [], 0, 0))
    assert (h.picture_height(0), h.picture_height(1)) == (243, 244)


def test_header_errors_match_the_oracle(oracle):
    """Header-level failures (no device work) name the same error as the
    oracle's decoder, for the reference's malformed cases and random bytes."""
    from tests.util import KIND, PREFIX

    cases = [d for _, d, _ in H.malformed_frames()]
    rng = random.Random(11)
    good = H.macroblock_frame()
    for _ in range(300):
        b = bytearray(good[:28 + rng.randint(0, 40)])
        for _ in range(rng.randint(1, 4)):
            b[rng.randrange(len(b))] = rng.randrange(256)
        cases.append(bytes(b))
    for _ in range(200):
        cases.append(bytes(rng.randrange(256) for _ in range(rng.randint(0, 60))))
    for d in cases:
        info = _abi.Frame_()
        code = _abi.lib().prores_probe(d, len(d), 0, ctypes.byref(info))
        k, msg, _ = oracle.decode(d)
        if code != 0:
            # The probe covers the frame header and the size guard: when it
            # fails, the oracle fails the same way.
            assert code == k and _abi.last_error() == PREFIX[k] + msg, (d.hex(), _abi.last_error(), msg)


def test_probe_gives_the_layout():
    data = H.alpha_frame()
    info = _abi.Frame_()
    assert _abi.lib().prores_probe(data, len(data), 8, ctypes.byref(info)) == 0
    assert (info.width, info.height, info.bit_depth, info.chroma) == (16, 16, 8, 3)
    assert info.data_len == 3 * 256 and info.alpha_len == 256
    assert _abi.lib().prores_probe(data, len(data), 7, ctypes.byref(info)) == _abi.CONFIG


def test_decoder_settings_are_checked():
    # tests/roundtrip.rs:462-463
    with pytest.raises(P.Error.Config):
        P.Decoder.with_bit_depth(7)
    with pytest.raises(P.Error.Config):
        P.Decoder.with_bit_depth(17)
    assert P.Decoder.with_bit_depth(16).bit_depth == 16


def test_frame_layout_rounds_chroma_width_up():
    # src/frame.rs:361-368
    f = P.Frame.new(15, 3, P.ChromaFormat.Yuv422, 10)
    assert f.planes[1].width == 8
    assert f.planes[2].offset == 45 + 24
    assert f.data.size == 45 + 48
    with pytest.raises(P.Error.Config):
        P.Frame.new(0, 1, P.ChromaFormat.Yuv422, 10)
    with pytest.raises(P.Error.Config):
        P.Frame.new(65536, 1, P.ChromaFormat.Yuv422, 10)
    with pytest.raises(P.Error.Config):
        P.Frame.new(1, 1, P.ChromaFormat.Yuv422, 7)


def test_le_bytes_and_frame_rates():
    f = P.Frame.new(5, 3, P.ChromaFormat.Yuv422, 16)
    f.data[:] = (np.arange(f.data.size) * 40503) & 0xFFFF
    want = b"".join(int(s).to_bytes(2, "little") for s in f.data)
    assert f.to_le_bytes() == want
    for c in range(1, 12):
        n, d = P.Metadata(frame_rate_code=c).frame_rate()
        assert P.Metadata.frame_rate_code_for(n, d) == c
    assert P.Metadata.frame_rate_code_for(48, 2) == 2
    assert P.Metadata.frame_rate_code_for(48, 1) == 0
