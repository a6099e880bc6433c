"""One batch over several devices (prores_*_batch_multi): frames split by
macroblock count, each share one batched call on a host thread of its own,
results and per-frame errors gathered in input order. With one GPU at hand
the parts are two contexts' calls on the same device (nothing in them waits
on another part), which exercises the split, the threads and the gather."""

import numpy as np
import pytest

import rivet_prores_b200 as P
from oracle import oracle as O
from tests.util import KIND, PREFIX, assert_decode_matches, to_config, to_frame

pytestmark = pytest.mark.gpu


def _devices():
    import torch

    n = torch.cuda.device_count()
    return [0, 1, 0] if n >= 2 else [0, 0]


def _batch():
    pics = [O.test_frame(w, h, c, d, 12, s) for s, (w, h, c, d) in enumerate(
        [(1920, 1080, 2, 10), (352, 288, 2, 10), (720, 486, 3, 12), (64, 48, 2, 10), (1280, 720, 2, 10),
         (176, 144, 3, 12)])]
    cfgs = [O.Config(3), O.Config(2), O.Config(5), O.Config(3, 1), O.Config(1), O.Config(4, 0)]
    return pics, cfgs


def test_encode_and_decode_over_devices_equal_the_oracle():
    pics, cfgs = _batch()
    frames = [to_frame(p) for p in pics]
    configs = [to_config(c) for c in cfgs]
    got = P.Encoder(configs[0]).encode_batch(frames, configs, devices=_devices())
    wants = []
    for i, (p, c) in enumerate(zip(pics, cfgs)):
        k, msg, want = O.encode(c, p)
        assert k == 0, msg
        assert got[i] == want, f"frame {i}"
        wants.append(want)
    # Decode, with a damaged frame in the middle: its error comes back in its
    # place, with the oracle's message.
    bad = bytearray(wants[1])
    bad[len(bad) // 2:] = bytes(len(bad) - len(bad) // 2)
    packets = wants[:1] + [bytes(bad)] + wants[1:]
    res = P.Decoder.new().decode_batch(packets, devices=_devices())
    for i, (pkt, r) in enumerate(zip(packets, res)):
        assert_decode_matches(r, O.decode(pkt), f"frame {i}")
    # Same as the one-device call, frame for frame.
    one = P.Decoder.new().decode_batch(packets)
    for a, b in zip(res, one):
        if isinstance(b, P.Error):
            assert a == b
        else:
            assert np.array_equal(a.data, b.data)


def test_header_errors_over_devices():
    pics, cfgs = _batch()
    k, msg, good = O.encode(cfgs[1], pics[1])
    packets = [b"", good, b"\x00" * 40, good]
    res = P.Decoder.new().decode_batch(packets, devices=_devices())
    for i, (pkt, r) in enumerate(zip(packets, res)):
        kind, msg, _ = O.decode(pkt)
        if kind != O.OK:
            assert isinstance(r, KIND[kind]) and r.message == PREFIX[kind] + msg, (i, r)
        else:
            assert not isinstance(r, P.Error), (i, r)
