"""The benchmark configurations as parity cases, at their stated sizes: every
GPU packet of each batch equals the oracle's, and every picture the GPU
decodes from those packets equals the oracle's decode.

  config 0  1 x 1280x720 4:2:2 10-bit 422 HQ, round trip
  config 1  64 x 1920x1080 4:2:2 10-bit 422 HQ, decoded in one batched call
  config 2  16 x 3840x2160 4:4:4 12-bit 4444 XQ with 16-bit alpha, top field
            first, loaded matrices; encode and decode batched
  config 3  96 mixed frames (720x486i HQ, 720p LT, 1080p Proxy/422/HQ, UHD
            HQ, 4096x2160 4444 16-bit with 16-bit alpha), per-frame slice
            widths of 1, 2, 4 or 8 macroblocks; encode and decode batched
"""

import numpy as np
import pytest

import rivet_prores_b200 as P
from oracle import oracle as O
from rivet_prores_b200 import workloads
from tests.util import assert_decode_matches

pytestmark = pytest.mark.gpu


def _oracle_pic(f: P.Frame) -> "O.Picture":
    return O.Picture(f.width, f.height, f.bit_depth, f.chroma.value, f.interlace.value,
                     (f.metadata.aspect_ratio, f.metadata.frame_rate_code, f.metadata.color_primaries,
                      f.metadata.transfer_characteristic, f.metadata.matrix_coefficients),
                     f.data, f.alpha)


def _oracle_cfg(c: P.Config) -> "O.Config":
    return O.Config(c.profile.value, c.log2_slice_mbs, c.alpha.value, c.luma_matrix, c.chroma_matrix,
                    c.target_frame_bytes, c.encoder_identifier)


def _check(batch, depth=0):
    """One batched encode of the whole batch and one batched decode of its
    packets, each frame compared with the oracle."""
    frames = [f for f, _ in batch]
    configs = [c for _, c in batch]
    got = P.Encoder(configs[0]).encode_batch(frames, configs)
    for i, (f, c, g) in enumerate(zip(frames, configs, got)):
        k, msg, want = O.encode(_oracle_cfg(c), _oracle_pic(f))
        assert k == 0, msg
        assert g == want, f"frame {i} ({f.width}x{f.height} {c.profile.name}): {len(g)} vs {len(want)} bytes"
    dec = P.Decoder(bit_depth=depth or None).decode_batch(got)
    for i, (pkt, d) in enumerate(zip(got, dec)):
        assert_decode_matches(d, O.decode(pkt, depth), f"frame {i}")
    return got


def test_config0_720p_422hq_round_trip():
    f = workloads.picture(1280, 720, P.ChromaFormat.Yuv422, 10, 0)
    pkt = _check([(f, P.Config(P.Profile.Hq))])[0]
    assert len(pkt) <= P.Profile.Hq.target_frame_bytes(1280, 720)


def test_config1_64_1080p_hq_batched_decode():
    batch = workloads.hd_422_hq(64)
    assert len({bytes(f.data[:4096]) for f, _ in batch}) == 64  # distinct pictures
    _check(batch, depth=10)


def test_config2_16_uhd_4444xq_alpha_fields_matrices():
    batch = workloads.uhd_4444xq_alpha(16)
    f0, c0 = batch[0]
    assert (f0.width, f0.height, f0.bit_depth, f0.interlace) == (3840, 2160, 12, P.Interlace.TopFieldFirst)
    assert f0.alpha is not None and int(f0.alpha.max()) > 255 and c0.luma_matrix is not None
    _check(batch)


def test_config3_96_heterogeneous_frames():
    batch = workloads.mixed_batch(96)
    assert len(batch) == 96
    assert {c.log2_slice_mbs for _, c in batch} == {0, 1, 2, 3}
    assert any(f.alpha is not None for f, _ in batch)
    _check(batch)


def test_config3_batched_equals_alone():
    """The mixed batch's outputs do not depend on the batch: a few frames
    coded alone give the same packets and pictures as in the batch."""
    batch = workloads.mixed_batch(14, config=31)
    frames = [f for f, _ in batch]
    configs = [c for _, c in batch]
    together = P.Encoder(configs[0]).encode_batch(frames, configs)
    for i in (0, 5, 6, 13):
        assert P.Encoder(configs[i]).encode(frames[i]) == together[i]
        a = P.Decoder.new().decode(together[i])
        b = P.Decoder.new().decode_batch(together)[i]
        assert np.array_equal(a.data, b.data)
