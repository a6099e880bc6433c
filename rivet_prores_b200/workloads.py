"""Seeded synthetic pictures for the benchmark configurations.

No public dataset is involved: each plane is generated at its own
resolution as 512 + a sum of 8 random 2-D cosines (frequencies U(0, 0.05)
cycles/px on each axis, amplitudes U(0, 150), phases U(0, 2 pi)) + 16
axis-aligned rectangles set to a constant level U(64, 940) at positions and
sizes uniform over the plane + Gaussian noise of sigma 12, clamped to 64-940
(luma) or 64-960 (chroma) at 10-bit scale; 12- and 16-bit inputs are the
10-bit picture shifted left by 2 and 6. The generator is numpy's PCG64 with
seed = 1000 * config + frame index, and per-plane sub-seeds 0, 1, 2 (and 3
for alpha: soft-edged ellipses over a 0 / max background plus sigma-200
noise, clamped).
"""

from __future__ import annotations

import os
from concurrent.futures import ThreadPoolExecutor
from typing import Callable, List, Optional, Sequence

import numpy as np

from . import AlphaType, ChromaFormat, Config, Frame, Interlace, Profile


def generate(makers: Sequence[Callable[[], object]]) -> list:
    """Runs the picture makers on host threads (numpy's array work releases
    the GIL), in order."""
    if len(makers) <= 1:
        return [m() for m in makers]
    with ThreadPoolExecutor(max_workers=min(len(makers), os.cpu_count() or 4)) as ex:
        return list(ex.map(lambda m: m(), makers))


def _plane(h: int, w: int, rng: np.random.Generator, hi: float) -> np.ndarray:
    y = np.arange(h, dtype=np.float64)
    x = np.arange(w, dtype=np.float64)
    v = np.full((h, w), 512.0)
    for _ in range(8):
        fx, fy = rng.uniform(0.0, 0.05, 2)
        amp = rng.uniform(0.0, 150.0)
        phase = rng.uniform(0.0, 2 * np.pi)
        # cos(a + b) = cos a cos b - sin a sin b: two outer products.
        ax = 2 * np.pi * fx * x + phase
        by = 2 * np.pi * fy * y
        v += amp * (np.outer(np.cos(by), np.cos(ax)) - np.outer(np.sin(by), np.sin(ax)))
    for _ in range(16):
        x0, x1 = np.sort(rng.integers(0, w + 1, 2))
        y0, y1 = np.sort(rng.integers(0, h + 1, 2))
        v[y0:y1, x0:x1] = rng.uniform(64.0, 940.0)
    v += rng.normal(0.0, 12.0, (h, w))
    return np.clip(np.rint(v), 64.0, hi)


def _alpha(h: int, w: int, rng: np.random.Generator) -> np.ndarray:
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    a = np.zeros((h, w))
    for _ in range(4):
        cx, cy = rng.uniform(0, w), rng.uniform(0, h)
        rx, ry = rng.uniform(0.1, 0.4) * w, rng.uniform(0.1, 0.4) * h
        d = np.sqrt(((xx - cx) / rx) ** 2 + ((yy - cy) / ry) ** 2)
        a = np.maximum(a, np.clip((1.0 - d) * 8.0, 0.0, 1.0))
    a = a * 65535.0 + rng.normal(0.0, 200.0, (h, w))
    return np.clip(np.rint(a), 0, 65535)


def picture(width: int, height: int, chroma: ChromaFormat, bit_depth: int, seed: int,
            alpha: bool = False, interlace: Interlace = Interlace.Progressive) -> Frame:
    f = Frame.new(width, height, chroma, bit_depth)
    f.interlace = interlace
    for i in range(3):
        p = f.planes[i]
        rng = np.random.Generator(np.random.PCG64([seed, i]))
        v = _plane(p.height, p.width, rng, 940.0 if i == 0 else 960.0)
        v = v * float(1 << (bit_depth - 10)) if bit_depth >= 10 else np.rint(v / float(1 << (10 - bit_depth)))
        f.data[p.offset:p.offset + p.len()] = v.astype(np.uint16).ravel()
    if alpha:
        rng = np.random.Generator(np.random.PCG64([seed, 3]))
        a = _alpha(height, width, rng)
        f.alpha = (a.astype(np.uint32) >> (16 - bit_depth)).astype(np.uint16).ravel()
    return f


def matrix(seed: int) -> bytes:
    """A loaded quantisation matrix: 64 weights U(4, 63)."""
    rng = np.random.Generator(np.random.PCG64([seed, 7]))
    return bytes(int(v) for v in rng.integers(4, 64, 64))


def uhd_422_hq(n: int, config: int = 1, unique: Optional[int] = None) -> List[Frame]:
    """n 3840x2160 4:2:2 10-bit frames (the 422 HQ headline workload); with
    `unique`, that many distinct pictures repeated."""
    u = n if unique is None else max(1, min(unique, n))
    base = generate([lambda i=i: picture(3840, 2160, ChromaFormat.Yuv422, 10, 1000 * config + i)
                     for i in range(u)])
    return [base[i % u] for i in range(n)]


def uhd_422_hq_at(indices: Sequence[int], config: int = 1) -> List[Frame]:
    """Frames `indices` of the headline batch (3840x2160 4:2:2 10-bit, the
    seed of frame i is 1000 * config + i): one rank's share of a batch
    split over ranks."""
    return generate([lambda i=i: picture(3840, 2160, ChromaFormat.Yuv422, 10, 1000 * config + i)
                     for i in indices])


def hd_422_hq(n: int = 64, config: int = 1):
    """Batched 1080p decode: n 1920x1080 4:2:2 10-bit frames with per-frame
    seeds, to be coded as 422 HQ at the profile's target. [(frame, config)]"""
    frames = generate([lambda i=i: picture(1920, 1080, ChromaFormat.Yuv422, 10, 1000 * config + i)
                       for i in range(n)])
    return [(f, Config(Profile.Hq)) for f in frames]


def uhd_4444xq_alpha(n: int = 16, config: int = 2):
    """n 3840x2160 4:4:4 12-bit frames with a 16-bit alpha plane, interlaced
    top field first, each with its own loaded luma and chroma matrices
    (entries U(4, 63)), coded as 4444 XQ. [(frame, config)]"""
    frames = generate([lambda i=i: picture(3840, 2160, ChromaFormat.Yuv444, 12, 1000 * config + i, alpha=True,
                                           interlace=Interlace.TopFieldFirst) for i in range(n)])
    return [(f, Config(Profile.P4444Xq, alpha=AlphaType.Bits16, luma_matrix=matrix(1000 * config + i),
                       chroma_matrix=matrix(1000 * config + 100 + i))) for i, f in enumerate(frames)]


MIXED_KINDS = [
    (720, 486, ChromaFormat.Yuv422, 10, Profile.Hq, Interlace.BottomFieldFirst, False),
    (1280, 720, ChromaFormat.Yuv422, 10, Profile.Lt, Interlace.Progressive, False),
    (1920, 1080, ChromaFormat.Yuv422, 10, Profile.Proxy, Interlace.Progressive, False),
    (1920, 1080, ChromaFormat.Yuv422, 10, Profile.Standard, Interlace.Progressive, False),
    (1920, 1080, ChromaFormat.Yuv422, 10, Profile.Hq, Interlace.Progressive, False),
    (3840, 2160, ChromaFormat.Yuv422, 10, Profile.Hq, Interlace.Progressive, False),
    (4096, 2160, ChromaFormat.Yuv444, 16, Profile.P4444, Interlace.Progressive, True),
]


def mixed_batch(n: int = 96, config: int = 3):
    """The heterogeneous batch: n frames cycling through the mix's kinds
    (720x486 interlaced 422 HQ, 1280x720 LT, 1920x1080 Proxy / 422 / HQ,
    3840x2160 HQ, 4096x2160 4444 from 16-bit input with a 16-bit alpha
    plane), per-frame seeds, each with a slice width drawn from {1, 2, 4, 8}
    macroblocks. [(frame, config)]"""
    rng = np.random.Generator(np.random.PCG64([1000 * config, 98]))
    kinds = [MIXED_KINDS[i % len(MIXED_KINDS)] for i in range(n)]
    log2s = [int(v) for v in rng.integers(0, 4, n)]
    frames = generate([lambda i=i, k=k: picture(k[0], k[1], k[2], k[3], 1000 * config + i, alpha=k[6],
                                                interlace=k[5]) for i, k in enumerate(kinds)])
    return [(f, Config(k[4], log2_slice_mbs=l, alpha=AlphaType.Bits16 if k[6] else AlphaType.None_))
            for f, k, l in zip(frames, kinds, log2s)]


def hq_config() -> Config:
    return Config(Profile.Hq)


def mixed_pool(seed_base: int = 3000):
    """One frame of each kind in the heterogeneous mix: 720x486 interlaced 422
    HQ, 1280x720 LT, 1920x1080 Proxy / 422 / HQ, 3840x2160 HQ and 4096x2160
    4444 from 16-bit input; slice widths drawn from {1, 2, 4, 8} macroblocks.
    Returns [(frame, config)]."""
    rng = np.random.Generator(np.random.PCG64([seed_base, 99]))
    kinds = [
        (720, 486, ChromaFormat.Yuv422, 10, Profile.Hq, Interlace.BottomFieldFirst),
        (1280, 720, ChromaFormat.Yuv422, 10, Profile.Lt, Interlace.Progressive),
        (1920, 1080, ChromaFormat.Yuv422, 10, Profile.Proxy, Interlace.Progressive),
        (1920, 1080, ChromaFormat.Yuv422, 10, Profile.Standard, Interlace.Progressive),
        (1920, 1080, ChromaFormat.Yuv422, 10, Profile.Hq, Interlace.Progressive),
        (3840, 2160, ChromaFormat.Yuv422, 10, Profile.Hq, Interlace.Progressive),
        (4096, 2160, ChromaFormat.Yuv444, 16, Profile.P4444, Interlace.Progressive),
    ]
    out = []
    for i, (w, h, chroma, depth, profile, interlace) in enumerate(kinds):
        f = picture(w, h, chroma, depth, seed_base + i, interlace=interlace)
        out.append((f, Config(profile, log2_slice_mbs=int(rng.integers(0, 4)))))
    return out
