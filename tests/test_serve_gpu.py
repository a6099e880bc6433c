"""Serving on the GPU: requests of both kinds and mixed sizes, submitted
while others run, each come back exactly as they do alone."""

import concurrent.futures as cf

import numpy as np
import pytest

import rivet_prores_b200 as P
from oracle import oracle as O
from rivet_prores_b200.serve import Server

pytestmark = pytest.mark.gpu


def test_each_result_is_the_same_alone_and_in_the_mix():
    frames, configs, packets = [], [], []
    sizes = [(64, 48, 2, 3), (176, 144, 2, 0), (320, 240, 3, 4), (97, 41, 3, 5), (720, 486, 2, 3), (33, 17, 2, 1)]
    for i, (w, h, chroma, profile) in enumerate(sizes):
        p = O.test_frame(w, h, chroma, 12 if chroma == 3 else 10, 10, 100 + i)
        p.interlace = i % 3
        f = P.Frame.new(w, h, P.ChromaFormat(chroma), p.bit_depth)
        f.data[:] = p.data
        f.interlace = P.Interlace(p.interlace)
        cfg = P.Config(P.Profile(profile), log2_slice_mbs=i % 4)
        frames.append(f)
        configs.append(cfg)
        packets.append(P.Encoder(cfg).encode(f))
    alone_dec = [P.Decoder.new().decode(pk) for pk in packets]
    alone_enc = [P.Encoder(c).encode(f) for f, c in zip(frames, configs)]
    srv = Server(memory_budget=256 << 20, max_batch=8, workers=3)
    futs = []
    for rep in range(10):
        for i in range(len(sizes)):
            if (rep + i) % 3:
                futs.append(("d", i, srv.submit_decode(packets[i])))
            else:
                futs.append(("e", i, srv.submit_encode(frames[i], configs[i])))
    for kind, i, f in futs:
        r = f.result(timeout=120)
        if kind == "d":
            assert np.array_equal(r.data, alone_dec[i].data)
        else:
            assert r == alone_enc[i]
    srv.close()
    st = srv.stats()
    assert st["requests"] == len(futs) and st["mean_batch"] >= 1.0
