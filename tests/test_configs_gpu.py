"""The benchmark configurations as parity cases (smaller batches): every GPU
packet equals the oracle's, every GPU picture the oracle's decode."""

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


def _check(frames, configs, depth=0):
    got = P.Encoder(configs[0]).encode_batch(frames, configs)
    for i, (f, c, g) in enumerate(zip(frames, configs, got)):
        k, msg, want = O.encode(_oracle_cfg(c), _oracle_pic(f))
        assert k == 0, msg
        assert g == want, f"frame {i}: {len(g)} vs {len(want)} bytes"
    dec = P.Decoder(bit_depth=depth or None).decode_batch(got)
    for i, (pkt, d) in enumerate(zip(got, dec)):
        assert_decode_matches(d, O.decode(pkt, depth), f"frame {i}")
    return got


def test_config0_720p_422hq_round_trip():
    f = workloads.picture(1280, 720, P.ChromaFormat.Yuv422, 10, 0)
    pkt = _check([f], [P.Config(P.Profile.Hq)])[0]
    assert len(pkt) <= P.Profile.Hq.target_frame_bytes(1280, 720)


def test_config1_1080p_hq_batched_decode():
    frames = [workloads.picture(1920, 1080, P.ChromaFormat.Yuv422, 10, 1000 + i) for i in range(4)]
    _check(frames, [P.Config(P.Profile.Hq)] * 4, depth=10)


def test_config2_uhd_4444xq_alpha_fields_matrices():
    frames, configs = [], []
    for i in range(2):
        f = workloads.picture(3840, 2160, P.ChromaFormat.Yuv444, 12, 2000 + i, alpha=True,
                              interlace=P.Interlace.TopFieldFirst)
        # 16-bit alpha: the generator's 0..65535 ellipses at 12-bit input scale.
        frames.append(f)
        configs.append(P.Config(P.Profile.P4444Xq, alpha=P.AlphaType.Bits16,
                                luma_matrix=workloads.matrix(2000 + i), chroma_matrix=workloads.matrix(2100 + i)))
    _check(frames, configs)


def test_config3_heterogeneous_batch():
    pool = workloads.mixed_pool()
    frames = [f for f, _ in pool]
    configs = [c for _, c in pool]
    _check(frames, configs)
