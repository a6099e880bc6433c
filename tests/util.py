"""Helpers shared by the parity tests: conversions between the oracle's
pictures and the package's frames, and the comparisons."""

from __future__ import annotations

import numpy as np

import rivet_prores_b200 as P
from oracle import oracle as O

KIND = {O.INVALID: P.Error.Invalid, O.UNSUPPORTED: P.Error.Unsupported, O.CONFIG: P.Error.Config}
PREFIX = {O.INVALID: "invalid ProRes data: ", O.UNSUPPORTED: "unsupported ProRes feature: ",
          O.CONFIG: "invalid ProRes configuration: "}


def to_frame(p: "O.Picture") -> P.Frame:
    chroma = P.ChromaFormat(p.chroma)
    f = P.Frame.new(p.width, p.height, chroma, p.bit_depth)
    f.data = np.array(p.data, dtype=np.uint16)
    f.interlace = P.Interlace(p.interlace)
    f.metadata = P.Metadata(*p.metadata)
    f.alpha = None if p.alpha is None else np.array(p.alpha, dtype=np.uint16)
    return f


def to_config(c: "O.Config") -> P.Config:
    return P.Config(P.Profile(c.profile), c.log2_slice_mbs, P.AlphaType(c.alpha), c.luma_matrix, c.chroma_matrix,
                    c.target_frame_bytes, c.encoder_identifier, c.threads)


def assert_decode_matches(result, oracle_result, what=""):
    """GPU decode result (Frame or Error) equals the oracle's (kind, message,
    planes, alpha, metadata)."""
    k, msg, pic = oracle_result
    if k != O.OK:
        assert isinstance(result, P.Error), f"{what}: oracle {msg!r}, GPU decoded"
        assert isinstance(result, KIND[k]), f"{what}: {type(result).__name__} vs {msg!r}"
        assert result.message == PREFIX[k] + msg, f"{what}: {result.message!r} vs {msg!r}"
        return
    assert not isinstance(result, P.Error), f"{what}: GPU error {result}"
    assert (result.width, result.height, result.bit_depth) == (pic.width, pic.height, pic.bit_depth), what
    assert result.chroma.value == pic.chroma and result.interlace.value == pic.interlace, what
    assert (result.metadata.aspect_ratio, result.metadata.frame_rate_code, result.metadata.color_primaries,
            result.metadata.transfer_characteristic, result.metadata.matrix_coefficients) == tuple(pic.metadata)
    if not np.array_equal(result.data, pic.data):
        bad = np.nonzero(result.data != pic.data)[0]
        raise AssertionError(f"{what}: {bad.size} samples differ, first at {bad[0]}: "
                             f"{result.data[bad[0]]} vs {pic.data[bad[0]]}")
    assert (result.alpha is None) == (pic.alpha is None), what
    if pic.alpha is not None:
        assert np.array_equal(result.alpha, pic.alpha), f"{what}: alpha differs"


def psnr(a: np.ndarray, b: np.ndarray, depth: int) -> float:
    mse = np.mean((a.astype(np.float64) - b.astype(np.float64)) ** 2)
    peak = (1 << depth) - 1
    return float("inf") if mse == 0 else 10 * np.log10(peak * peak / mse)
