"""Frames assembled byte by byte and bit by bit from RDD 36's syntax, the way
the reference's tests/handbuilt.rs builds them (:116-196), and the samples
they decode to, computed independently of any codec.

These are the only bit-level golden decode vectors the reference holds; the
oracle and the CUDA decoder are both checked against them.
"""

from __future__ import annotations

import math
import struct


def bits(s: str) -> bytes:
    """Bytes from '0'/'1' characters (spaces ignored), zero-padded to a byte
    (tests/handbuilt.rs:116-125)."""
    b = [int(c) for c in s if c != " "]
    out = bytearray()
    for i in range(0, len(b), 8):
        chunk = b[i:i + 8]
        v = 0
        for j, bit in enumerate(chunk):
            v |= bit << (7 - j)
        out.append(v)
    return bytes(out)


def frame_header(w, h, chroma, interlace, alpha, version, extra) -> bytes:
    """tests/handbuilt.rs:130-153: square pixels, 25 fps, BT.709 codes."""
    v = bytearray(struct.pack(">H", 20 + extra))
    v.append(0)
    v.append(version)
    v += b"hand"
    v += struct.pack(">HH", w, h)
    v.append((chroma << 6) | (interlace << 2))
    v.append((1 << 4) | 3)
    v += bytes([1, 1, 1])
    v.append(alpha)
    v += bytes([0, 0])
    v += bytes([0xAA] * extra)
    return bytes(v)


def slice_(qindex, y, cb, cr, extra) -> bytes:
    """tests/handbuilt.rs:156-165 (no alpha: Cr size implied)."""
    v = bytearray([((6 + extra) << 3) & 0xFF, qindex])
    v += struct.pack(">HH", len(y), len(cb))
    v += bytes([0x55] * extra)
    v += y + cb + cr
    return bytes(v)


def picture(log2_slice_mbs, slices) -> bytes:
    """tests/handbuilt.rs:168-181."""
    size = 8 + 2 * len(slices) + sum(len(s) for s in slices)
    v = bytearray([8 << 3])
    v += struct.pack(">IH", size, len(slices))
    v.append(log2_slice_mbs << 4)
    for s in slices:
        v += struct.pack(">H", len(s))
    for s in slices:
        v += s
    return bytes(v)


def frame(header, pictures, stuffing, trailing) -> bytes:
    """tests/handbuilt.rs:185-196."""
    size = 8 + len(header) + sum(len(p) for p in pictures) + stuffing
    v = bytearray(struct.pack(">I", size))
    v += b"icpf" + header
    for p in pictures:
        v += p
    v += bytes(stuffing)
    v += bytes([0xFF] * trailing)
    return bytes(v)


def one_macroblock():
    """tests/handbuilt.rs:198-223: Y' DCs 0, 64, -64, 128 and one AC +100;
    Cb DCs 0, 0; Cr DCs -32, -32 with a trailing zero byte."""
    y = bits("100000 000010001000 00000100000111 00000110000111 010 0000000 1100011 0")
    cb = bits("100000 1000")
    cr = bits("01011111 1000") + b"\x00"
    return y, cb, cr


def sample(v: float) -> int:
    """10-bit s = round(2v + 512) (tests/handbuilt.rs:226-228), half away from zero."""
    x = 2.0 * v + 512.0
    return int(math.floor(x + 0.5)) if x >= 0 else -int(math.floor(-x + 0.5))


def macroblock_frame() -> bytes:
    y, cb, cr = one_macroblock()
    s = slice_(1, y, cb, cr, 1)
    return frame(frame_header(16, 16, 2, 0, 0, 0, 4), [picture(0, [s])], 5, 7)


def macroblock_expected_luma():
    """The 16x16 Y' samples §7 gives for macroblock_frame() (handbuilt.rs:258-275)."""
    out = []
    for row in range(16):
        r = []
        for col in range(16):
            key = (col // 8, row // 8)
            if key == (0, 0):
                want = sample(0.0)
            elif key == (1, 0):
                x = float(col - 8)
                ac = 50.0 / (4.0 * math.sqrt(2.0)) * math.cos((2.0 * x + 1.0) * math.pi / 16.0)
                want = sample(4.0 + ac)
            elif key == (0, 1):
                want = sample(-4.0)
            else:
                want = sample(8.0)
            r.append(want)
        out.append(r)
    return out


def field_frames():
    """tests/handbuilt.rs:285-327: two one-row field pictures of a 16x2 frame;
    returns [(frame bytes, first_row)] for interlace modes 1 and 2."""
    y_hi = bits("0010100000 1000 1 1")
    y_lo = bits("0010011111 1000 1 1")
    flat = bits("100000 1000")
    out = []
    for mode, first_row in [(1, 0), (2, 1)]:
        first = picture(0, [slice_(1, y_hi, flat, flat, 0)])
        second = picture(0, [slice_(1, y_lo, flat, flat, 0)])
        out.append((mode, first_row, frame(frame_header(16, 2, 2, mode, 0, 0, 0), [first, second], 0, 0)))
    return out


def alpha_frame() -> bytes:
    """tests/handbuilt.rs:332-361: 16x16 4:4:4, 8-bit alpha by hand."""
    flat4 = bits("100000 1000 1 1")
    alpha = bits("1 00000000 01111  1 00000001 00000 00011101110  1 00001010 1")
    s = bytearray([8 << 3, 1])
    for _ in range(3):
        s += struct.pack(">H", len(flat4))
    for _ in range(3):
        s += flat4
    s += alpha
    return frame(frame_header(16, 16, 3, 0, 1, 1, 0), [picture(3, [bytes(s)])], 0, 0)


def malformed_frames():
    """tests/handbuilt.rs:363-424: (name, bytes, expected kind) with kinds
    'Invalid' / 'Unsupported'; the good frame decodes."""
    y, cb, cr = one_macroblock()
    good = frame(frame_header(16, 16, 2, 0, 0, 0, 0), [picture(0, [slice_(1, y, cb, cr, 0)])], 0, 0)
    cases = [("good", good, None), ("short", good[:20], "Invalid"), ("frame_size past data", good[:-1], "Invalid")]

    def edit(i, v):
        b = bytearray(good)
        b[i] = v
        return bytes(b)

    cases += [
        ("not icpf", edit(4, ord("x")), "Invalid"),
        ("chroma 1", edit(8 + 12, 1 << 6), "Invalid"),
        ("interlace 3", edit(8 + 12, (2 << 6) | (3 << 2)), "Invalid"),
        ("alpha 3", edit(8 + 17, 3), "Invalid"),
        ("version 2", edit(8 + 3, 2), "Unsupported"),
        ("qindex 0", edit(8 + 20 + 8 + 2 + 1, 0), "Invalid"),
        ("slice past picture", edit(8 + 20 + 8, 0xFF), "Invalid"),
        ("picture past frame", edit(8 + 20 + 4, 0xFF), "Invalid"),
    ]
    yrun = bits("100000 1000 1 1 00000000 100101101 1 0")
    cases.append(("run past end", frame(frame_header(16, 16, 2, 0, 0, 0, 0),
                                        [picture(0, [slice_(1, yrun, cb, cr, 0)])], 0, 0), "Invalid"))
    ycut = bits("0000000000")
    cases.append(("cut mid-codeword", frame(frame_header(16, 16, 2, 0, 0, 0, 0),
                                            [picture(0, [slice_(1, ycut, cb, cr, 0)])], 0, 0), "Invalid"))
    return cases
