"""The oracle's AVX2 dsp kernels against its scalar ones (the crate's own
SIMD dispatch is defined to give the scalar results, src/dsp/mod.rs:1-20):
the same samples, coefficients, quantised values and masks bit for bit,
on random blocks with edge values, and the same packets and pictures
through whole encodes and decodes."""

import numpy as np
import pytest

from oracle import oracle as O


@pytest.fixture
def both():
    """Runs f with the scalar forms, then the AVX2 forms (left on)."""
    def run(f):
        O.set_simd(False)
        try:
            a = f()
        finally:
            O.set_simd(True)
        return a, f()
    return run


def test_idct_put(both):
    rng = np.random.default_rng(1)
    for trial in range(3000):
        depth = int(rng.integers(8, 17))
        kind = trial % 4
        if kind == 0:
            coef = rng.integers(-8, 9, 64)
        elif kind == 1:
            coef = rng.integers(-(1 << 15), 1 << 15, 64)
        elif kind == 2:
            coef = rng.integers(-(1 << 31), (1 << 31) - 1, 64, dtype=np.int64)
        else:
            coef = np.where(rng.random(64) < 0.85, 0, rng.integers(-300, 301, 64))
            coef[8 * rng.integers(0, 8):][:8] = 0  # all-zero rows
        scale = (rng.integers(1, 64, 64) * rng.integers(1, 1025)).astype(np.float32) / np.float32(8.0)
        a, b = both(lambda: O.idct_put(coef.astype(np.int32), scale, depth))
        assert np.array_equal(a, b), (trial, depth)


def test_fdct_load(both):
    rng = np.random.default_rng(2)
    for trial in range(3000):
        bits = int(rng.integers(8, 17))
        pix = rng.integers(0, 1 << bits, 64).astype(np.uint16)
        if trial % 5 == 0:
            pix[:] = pix[0]  # flat blocks
        scale = np.float32(512.0) / np.float32(1 << bits)
        a, b = both(lambda: O.fdct_load(pix, float(scale)))
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), trial


@pytest.mark.parametrize("n", [8, 16, 32, 4, 2, 1])
def test_quantise(both, n):
    rng = np.random.default_rng(3 + n)
    for trial in range(200):
        f = (rng.standard_normal(64 * n) * rng.choice([1.0, 30.0, 1000.0, 1e9])).astype(np.float32)
        f[rng.random(64 * n) < 0.1] = np.float32(-0.0)
        f[rng.random(64 * n) < 0.02] = np.float32(3e38)
        f[rng.random(64 * n) < 0.02] = np.float32(-3e38)
        inv = (np.float32(8.0) / rng.integers(1, 64 * 1024, 64).astype(np.float32)).astype(np.float32)
        for r in (0.42, 0.5, 0.0):
            (qa, ma), (qb, mb) = both(lambda: O.quantise(f, n, inv, r))
            assert np.array_equal(qa, qb) and np.array_equal(ma, mb), (n, trial, r)


@pytest.mark.parametrize("w,h,chroma,depth,profile,log2,interlace", [
    (1280, 720, 2, 10, 3, 3, 0),   # 422 HQ, the baseline's small case
    (720, 486, 2, 10, 3, 1, 1),    # interlaced, 2-macroblock slices
    (352, 288, 3, 12, 4, 0, 0),    # 4444, 1-macroblock slices (components of 4 blocks)
    (704, 480, 2, 10, 0, 2, 0),    # Proxy
])
def test_codec_frames(both, w, h, chroma, depth, profile, log2, interlace):
    pic = O.test_frame(w, h, chroma, depth, 24, 7)
    pic.interlace = interlace
    cfg = O.Config(profile, log2_slice_mbs=log2)

    def run():
        k, msg, pkt = O.encode(cfg, pic)
        assert k == O.OK, msg
        k, msg, dec = O.decode(pkt)
        assert k == O.OK, msg
        return pkt, dec.data

    (pa, da), (pb, db) = both(run)
    assert pa == pb
    assert np.array_equal(da, db)
