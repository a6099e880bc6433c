"""Autotuner for the launch shapes of libprores_b200.

The shapes are the fields of `Tuning` (prores_tuning in the C ABI):

* `cost_lane_items_per_sm`: the batch size (slice components per SM) from
  which rate-control costing runs a lane per slice component rather than a
  warp per component. Lanes need many components to fill the GPU; warps
  finish a small batch sooner.
* `decode_fused`, `decode_slot_positions`: whether the per-slice decode
  runs as one kernel, and how many coefficient positions (so how many
  slices) one of its CTAs holds in shared memory at once.
* `entropy_warps_per_block`, `entropy_blocks_per_sm`,
  `entropy_components_per_lane`: for the two-kernel decode, the persistent
  entropy decoder's warps per CTA, resident CTAs per SM and slice
  components per lane per grab of the shared work counter.
* `staging_depth`: the parts a batch of host frames is split into when it is
  streamed through resident jobs (`stream.RoundTripPipeline`): copies of one
  part overlap the kernels of another.

None of them changes a decoded sample or an encoded byte, so the tuner only
times: each candidate on this GPU, on seeded synthetic UHD 422 HQ frames.
The choice is cached as JSON keyed by GPU name and SM count, at
$RIVET_PRORES_TUNE_CACHE or ~/.cache/rivet_prores_b200/tuning.json; a new
context of that GPU takes it.
"""

from __future__ import annotations

import json
import os
from dataclasses import asdict
from typing import Callable, Dict, List, Optional, Sequence, Tuple

CACHE_ENV = "RIVET_PRORES_TUNE_CACHE"


def cache_path() -> str:
    p = os.environ.get(CACHE_ENV)
    if p:
        return p
    return os.path.join(os.path.expanduser("~"), ".cache", "rivet_prores_b200", "tuning.json")


def gpu_key(device: int = 0) -> Optional[str]:
    """The cache key of `device`: its name and SM count."""
    try:
        import torch

        p = torch.cuda.get_device_properties(device)
        return f"{p.name}|{p.multi_processor_count} SMs"
    except Exception:
        return None


def _read(path: str) -> dict:
    try:
        with open(path) as f:
            data = json.load(f)
        return data if isinstance(data, dict) else {}
    except (OSError, ValueError):
        return {}


def load(device: int = 0, key: Optional[str] = None):
    """The cached Tuning of this GPU, or None."""
    from . import Tuning

    key = key or gpu_key(device)
    if key is None:
        return None
    entry = _read(cache_path()).get(key)
    if not isinstance(entry, dict) or not isinstance(entry.get("tuning"), dict):
        return None
    fields = Tuning.__dataclass_fields__
    try:
        return Tuning(**{k: int(v) for k, v in entry["tuning"].items() if k in fields})
    except (TypeError, ValueError):
        return None


def save(tuning, evidence: dict, device: int = 0, key: Optional[str] = None) -> str:
    """Stores `tuning` (and the timings it was chosen from) for this GPU."""
    key = key or gpu_key(device)
    if key is None:
        raise RuntimeError("no GPU to key the tuning by")
    path = cache_path()
    data = _read(path)
    data[key] = {"tuning": asdict(tuning), "evidence": evidence}
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
    os.replace(tmp, path)
    return path


# ------------------------------------------------------------- choices


def lane_threshold(points: Sequence[Tuple[int, float, float]], sm_count: int) -> int:
    """`cost_lane_items_per_sm` from timings (slices, lane ms, warp ms) of
    several batch sizes: the smallest measured size from which lanes win at
    every larger size, as slice components per SM (0: lanes always won;
    above every measured size: warps always won)."""
    pts = sorted(points)
    if not pts:
        raise ValueError("no timings")
    start = None
    for i in range(len(pts) - 1, -1, -1):
        if pts[i][1] <= pts[i][2]:
            start = i
        else:
            break
    if start is None:
        return (3 * pts[-1][0]) // sm_count + 1
    if start == 0:
        return 0
    return (3 * pts[start][0] + sm_count - 1) // sm_count


def best(timings: Dict):
    """The candidate with the least time (ties: the first listed)."""
    items = list(timings.items())
    if not items:
        raise ValueError("no timings")
    return min(items, key=lambda kv: kv[1])[0]


def slices_in(frame, log2_slice_mbs: int = 3) -> int:
    """Slices of a progressive frame: each macroblock row splits into slices
    of 2^log2 macroblocks, the rest into smaller powers of two
    (src/header.rs:308-320)."""
    mb_w = (frame.width + 15) // 16
    mb_h = (frame.height + 15) // 16
    q, r = divmod(mb_w, 1 << log2_slice_mbs)
    return mb_h * (q + bin(r).count("1"))


# ------------------------------------------------------------- timing


def _time(launch: Callable, stream, reps: int) -> float:
    import torch

    launch()
    stream.synchronize()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(reps):
        launch()
    b.record(stream)
    stream.synchronize()
    return a.elapsed_time(b) / reps


def tune(device: int = 0, quick: bool = False, store: bool = True, frames: Optional[List] = None,
         stage_frames: Optional[List] = None, depths: Optional[Sequence[int]] = None,
         log: Optional[Callable[[str], None]] = None):
    """Times the candidate shapes on this GPU and applies the fastest to the
    device's context; returns (Tuning, evidence). `frames` (UHD 422 10-bit
    by default) feed the costing and decoder searches, `stage_frames` (the
    same by default) the staging-depth search over `depths`."""
    import torch

    from . import Config, DecodeJob, EncodeJob, Profile, context, workloads
    from .stream import RoundTripPipeline, time_round_trip

    say = log or (lambda s: None)
    ctx = context(device)
    tuning = ctx.tuning
    sms = torch.cuda.get_device_properties(device).multi_processor_count
    cfg = Config(Profile.Hq)
    n_big = 8 if quick else 16
    frames = frames or workloads.uhd_422_hq(n_big, config=9, unique=4)
    stream = torch.cuda.Stream(device)
    reps = 3 if quick else 5
    evidence: dict = {}

    # Costing: lanes against warps by batch size.
    sizes = [1, 4, n_big] if quick else [1, 2, 4, 8, 16]
    points = []
    for n in sizes:
        job = EncodeJob(frames[:n], cfg, device=device)
        t = {}
        for mode, items in (("lane", 0), ("warp", 1 << 30)):
            ctx.set_tuning(type(tuning)(**{**asdict(tuning), "cost_lane_items_per_sm": items}))
            t[mode] = _time(lambda: job.launch(stream), stream, reps)
        slices = n * slices_in(frames[0])
        points.append((slices, t["lane"], t["warp"]))
        say(f"encode {n} frames: lane {t['lane']:.3f} ms, warp {t['warp']:.3f} ms")
        job.close()
    tuning = type(tuning)(**{**asdict(tuning), "cost_lane_items_per_sm": lane_threshold(points, sms)})
    evidence["cost"] = [{"slices": s, "lane_ms": round(a, 4), "warp_ms": round(b, 4)} for s, a, b in points]

    # Entropy decoder shapes.
    enc = EncodeJob(frames, cfg, device=device)
    enc.launch(stream)
    packets = [bytes(p) for p in enc.fetch(stream, copy=False)]
    enc.close()
    dec = DecodeJob(packets, device=device)
    shapes = {}
    # The fused decoder by slice group size ...
    for nbytes in (1, 2):
        for pos in ([16384, 32768, 65536] if quick else [8192, 16384, 24576, 32768, 49152, 65536]):
            ctx.set_tuning(type(tuning)(**{**asdict(tuning), "decode_fused": 1, "decode_slot_positions": pos,
                                           "decode_slot_bytes": nbytes}))
            shapes[(1, pos, nbytes, 0, 0, 0)] = _time(lambda: dec.launch(stream), stream, reps)
    # ... against the two-kernel form's shapes.
    warps = [8] if quick else [4, 8, 16]
    blocks = [0] if quick else [0, 1, 2, 3]
    per_lane = [1] if quick else [1, 2, 4]
    for w in warps:
        for b in blocks:
            for k in per_lane:
                cand = type(tuning)(**{**asdict(tuning), "decode_fused": 0, "entropy_warps_per_block": w,
                                       "entropy_blocks_per_sm": b, "entropy_components_per_lane": k})
                ctx.set_tuning(cand)
                shapes[(0, tuning.decode_slot_positions, tuning.decode_slot_bytes, w, b, k)] = _time(
                    lambda: dec.launch(stream), stream, reps)
    dec.close()
    fused, pos, nbytes, w, b, k = best(shapes)
    chosen = {"decode_fused": fused, "decode_slot_positions": pos, "decode_slot_bytes": nbytes}
    if not fused:
        chosen.update(entropy_warps_per_block=w, entropy_blocks_per_sm=b, entropy_components_per_lane=k)
    tuning = type(tuning)(**{**asdict(tuning), **chosen})
    evidence["decode"] = [{"fused": a, "slot_positions": p, "slot_bytes": q, "warps_per_block": c,
                           "blocks_per_sm": d, "components_per_lane": e, "ms": round(v, 4)}
                          for (a, p, q, c, d, e), v in shapes.items()]
    say(f"decode: {chosen} ({shapes[(fused, pos, nbytes, w, b, k)]:.3f} ms)")

    # Staging depth of the host round trip.
    ctx.set_tuning(tuning)
    stage_frames = stage_frames or frames
    timed = {}
    # The quick search leaves out depth 2, which no full search on a B200
    # has chosen (the copies of two parts do not cover each other's
    # kernels), and times 3 steps a depth rather than 2, whose noise once
    # chose depth 2 all the same.
    for d in depths or ([3, 4, 6, 8] if quick else [2, 3, 4, 6, 8, 16]):
        if d > len(stage_frames):
            continue
        pipe = RoundTripPipeline(stage_frames, cfg, d, device=device)
        timed[d] = time_round_trip(pipe, steps=3, warmup=1)
        pipe.close()
        say(f"round trip, depth {d}: {timed[d]:.2f} ms for {len(stage_frames)} frames")
    if timed:
        tuning = type(tuning)(**{**asdict(tuning), "staging_depth": best(timed)})
    evidence["staging"] = [{"depth": d, "ms": round(v, 3), "frames": len(stage_frames)} for d, v in timed.items()]

    ctx.set_tuning(tuning)
    if store:
        save(tuning, evidence, device)
    return tuning, evidence


if __name__ == "__main__":
    import sys

    t, ev = tune(quick="--quick" in sys.argv, log=print)
    print(json.dumps({"tuning": asdict(t), "evidence": ev, "cache": cache_path()}))
