"""Frames found and decoded where they lie in device memory: the device
scan gives the host scan's spans, and decode_device writes into device
buffers exactly what the host path decodes (planes, alpha, metadata, and
the crate's error for a damaged frame)."""

import numpy as np
import pytest

import rivet_prores_b200 as P
from tests.test_scan import crate_frames, mov_like, planted

pytestmark = pytest.mark.gpu


def _to_device(data: bytes):
    import torch

    if not data:
        return torch.empty(0, dtype=torch.uint8, device="cuda")
    return torch.frombuffer(bytearray(data), dtype=torch.uint8).cuda()


def test_device_scan_equals_the_host_scan():
    for seed in range(40):
        data = planted(seed, 5000)
        assert P.scan_frames_device(_to_device(data)) == crate_frames(data), seed
    data, _ = mov_like(1)
    assert P.scan_frames_device(_to_device(data)) == P.scan_frames(data)
    assert P.scan_frames_device(_to_device(b"")) == []


def test_decode_in_device_memory_equals_the_host_decode():
    import torch

    data, spans = mov_like(3)
    # A damaged copy of the first frame at the end: the crate's error comes back.
    off, n = spans[0]
    bad = bytearray(data[off:off + n])
    bad[n // 2:] = b"\xff" * (n - n // 2)
    data = data + bytes(bad)
    spans = P.scan_frames(data)
    d = _to_device(data)
    dec = P.Decoder.new()
    alloc = lambda k: torch.empty(k, dtype=torch.int16, device="cuda")  # noqa: E731
    for rep in range(2):
        got = dec.decode_device(d, spans, alloc)
        want = dec.decode_batch([data[o:o + k] for o, k in spans])
        assert len(got) == len(want)
        for g, w in zip(got, want):
            if isinstance(w, P.Error):
                assert isinstance(g, type(w)) and g.message == w.message
                continue
            assert not isinstance(g, P.Error), g
            assert (g.width, g.height, g.bit_depth, g.chroma, g.interlace) == (w.width, w.height, w.bit_depth,
                                                                              w.chroma, w.interlace)
            assert np.array_equal(g.data.cpu().numpy().view(np.uint16), w.data)
            if w.alpha is not None:
                assert np.array_equal(g.alpha.cpu().numpy().view(np.uint16), w.alpha)


def test_spans_outside_the_buffer_are_refused():
    d = _to_device(b"\0" * 100)
    with pytest.raises(P.Error.Config):
        P.Decoder.new().decode_device(d, [(90, 20)], lambda k: None)


def test_encode_from_device_memory_equals_the_host_encode():
    """A transcoder's path on the GPU: frames decoded into device memory
    are encoded from there, and the packets equal the host path's."""
    import torch

    data, spans = mov_like(4)
    d = _to_device(data)
    alloc = lambda k: torch.empty(k, dtype=torch.int16, device="cuda")  # noqa: E731
    dev_frames = P.Decoder.new().decode_device(d, spans, alloc)
    host_frames = P.Decoder.new().decode_batch([data[o:o + k] for o, k in spans])
    configs = [P.Config(P.Profile.P4444 if f.chroma == P.ChromaFormat.Yuv444 else P.Profile.Hq, log2_slice_mbs=i % 4)
               for i, f in enumerate(host_frames)]
    enc = P.Encoder(configs[0])
    for rep in range(2):
        got = enc.encode_device(dev_frames, configs)
        want = enc.encode_batch(host_frames, configs)
        assert got == want
