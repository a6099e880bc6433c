"""Finding frames in a MOV without parsing the container: the library's scan
against a restatement of the crate's own helper (tests/sample.rs:20-38,
examples/prores_bench.rs:103-121), on planted and random cases."""

import numpy as np

import rivet_prores_b200 as P
from oracle import oracle as O


def crate_frames(data: bytes):
    """tests/sample.rs:22-38, line by line."""
    out = []
    i = 4
    while i + 4 <= len(data):
        if data[i:i + 4] == b"icpf":
            size = int.from_bytes(data[i - 4:i], "big")
            if size >= 28 and i - 4 + size <= len(data):
                out.append((i - 4, size))
                i += size - 4
                continue
        i += 1
    return out


def planted(seed: int, n: int = 4000) -> bytes:
    """Random bytes with 'icpf' planted often: valid and invalid sizes,
    overlapping candidates, candidates inside frames and at the ends."""
    rng = np.random.Generator(np.random.PCG64(seed))
    b = bytearray(rng.integers(0, 256, n, dtype=np.uint8).tobytes())
    for _ in range(int(rng.integers(1, 40))):
        i = int(rng.integers(0, n))
        size = int(rng.choice([0, 7, 27, 28, 29, int(rng.integers(28, 400)), n, n + 5, 1 << 31]))
        chunk = size.to_bytes(4, "big") + b"icpf"
        b[i:i + 8] = chunk[: max(0, min(8, n - i))]
    return bytes(b[:n])


def mov_like(seed: int):
    """Junk, then frames (encoded by the oracle) with junk between them;
    returns the buffer and the frames' spans."""
    rng = np.random.Generator(np.random.PCG64(seed))
    pieces, spans, pos = [], [], 0
    kinds = [(64, 48, 2, 10, 3, 0), (97, 41, 3, 12, 4, 1), (128, 64, 2, 10, 2, 2), (33, 17, 3, 12, 5, 0)]
    for k, (w, h, chroma, depth, profile, il) in enumerate(kinds):
        junk = rng.integers(0, 256, int(rng.integers(0, 300)), dtype=np.uint8).tobytes()
        pic = O.test_frame(w, h, chroma, depth, 10, 50 + seed * 10 + k)
        pic.interlace = il
        code, msg, pkt = O.encode(O.Config(profile), pic)
        assert code == O.OK, msg
        pieces += [junk, pkt]
        spans.append((pos + len(junk), len(pkt)))
        pos += len(junk) + len(pkt)
    tail = rng.integers(0, 256, 37, dtype=np.uint8).tobytes()
    return b"".join(pieces) + tail, spans


def test_scan_matches_the_crate_walk_on_planted_bytes():
    for seed in range(300):
        data = planted(seed, int(np.random.Generator(np.random.PCG64(seed)).integers(0, 3000)))
        assert P.scan_frames(data) == crate_frames(data), seed


def test_scan_finds_the_frames_of_a_mov_like_buffer():
    for seed in range(5):
        data, spans = mov_like(seed)
        got = P.scan_frames(data)
        assert got == crate_frames(data)
        # Every frame is found (junk may hold a stray 'icpf' of its own).
        assert all(s in got for s in spans)


def test_scan_of_short_and_empty_buffers():
    for data in [b"", b"icpf", b"\0\0\0\x1cicpf", b"\0\0\0\x08icpf" + b"\0" * 30, b"\0\0\0\x1cicpf" + b"\0" * 20]:
        assert P.scan_frames(data) == crate_frames(data)
