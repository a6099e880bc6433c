"""ProRes UHD 422 HQ throughput on B200.

One step = encode a batch of B 3840x2160 4:2:2 10-bit frames as 422 HQ
(apch, target 3 643 238 B each) and decode the B packets back to planes,
each direction one batched, CUDA-graph-captured launch on device-resident
buffers. `value` is frames/s through both directions (B distinct pictures
per step); decode-only and encode-only rates, the plain one-frame-per-launch
forms, the end-to-end rate through the C ABI with host buffers (`e2e`), the
other benchmark configurations (`configs`), serving under a Poisson request
stream (`serve`) and the CPU codec on the host's cores (`cpu_baseline`) are
reported beside it. Inputs are seeded synthetic pictures
(rivet_prores_b200/workloads.py); every step's inputs (B x 33 MB of planes)
are larger than L2.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--batch B] [--impl b200|reference]

Under torchrun each rank codes its share of a global batch of B x N frames,
split by macroblock count as the library's multi-device calls split it
(weak scaling, no collective on the data path); times are the max over
ranks. `--impl reference` times the reference codec's CPU path (the
oracle's restatement of it, with its slice-parallel thread pool on every
host core) on the same workload.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "ProRes UHD HQ frames/s on 1 B200, bit-exact; batched vs plain; serve p50/p99"
W, H = 3840, 2160
SAMPLES = W * H * 2  # u16 samples of a 4:2:2 frame: Y' plus two half-width chroma planes
TARGET = 3_643_238  # Profile::target_frame_bytes(HQ, 3840, 2160)

# Each kernel's own algorithmic bytes per frame and launch, for a frame of
# `s` u16 samples coded into a packet of `p` bytes (the encoder's
# coefficients are f32 in the slice's scanned order, plus one f32 maximum
# per 32 of them; the decoder reads the packet once and writes the planes).
KERNEL_BYTES = {
    "k_fdct": (lambda s, p: 2 * s + 4 * s + s // 8, "planes in (2 B a sample), f32 coefficients and chunk maxima out"),
    "k_cost": (lambda s, p: 4 * s + s // 8, "f32 coefficients and chunk maxima a probe reads when it skips no chunk"),
    "k_pack": (lambda s, p: 4 * s + s // 8 + p, "f32 coefficients and chunk maxima in, packet out"),
    "k_decode": (lambda s, p: p + 2 * s, "packet in, u16 planes out"),
    "k_entropy": (lambda s, p: p, "packet in (coefficient lists are an intermediate)"),
    "k_idct": (lambda s, p: 2 * s, "u16 planes out (coefficient lists are an intermediate)"),
}
# What the CPU codec timed beside the GPU is, and what the crate itself
# publishes for the same work on other hardware.
CPU_CODE = ("the oracle's restatement of the crate's CPU path, with its slice-parallel pool and AVX2 forms of the dsp "
            "kernels (IDCT, FDCT, quantise), which give the scalar forms' results bit for bit as the crate's own SIMD "
            "levels do; entropy coding and rate control scalar, as in the crate; compiled -O3 -march=x86-64-v3 "
            "-ffp-contract=off")
PUBLISHED_CRATE = ("the crate's README: 1920x1080 422 HQ at 296 encode / 907 decode frames/s on 32 threads of a Ryzen 9 "
                   "9950X, about 74 / 227 at UHD (4x the samples), about 56 round trips/s; other hardware")
# Figures from ncu captures of these kernels, not measured by this run: the
# capture's DRAM bytes (read + write) per frame and launch, and issue-slot use.
CAPTURED = {
    "k_cost": {"dram_bytes_per_frame": 70.96e6, "issue_active_pct": "41.5",
               "thread_instructions_per_coefficient": 26.7,
               "capture": "ncu --set full on an 8-frame UHD 422 HQ encode, its fifth k_cost launch (a dense probe, "
                          "which reads every coefficient: the heaviest of the nine)"},
}
# What limits each kernel, from the ncu captures summarised under profiles/.
# The roofline's "bound" is the roof the kernel is measured against (HBM
# bandwidth: the work is byte and integer work, no tensor-core math); none of
# these kernels reaches it, and "limiter" names what holds it back instead.
LIMITER = {
    "k_cost": "latency: 41.5 % of issue slots active, a quarter to two fifths of the warp slots busy",
    "k_cost_window": "latency, as k_cost; it costs a list of slices that changes with the pictures (level 0 "
                     "copies from a probe at the same quantiser where there is one), so it has no fixed byte basis",
    "k_fdct": "instruction issue (83 % of issue slots active)",
    "k_pack": "latency: half of each warp's lanes active",
    "k_entropy": "latency: a warp waits for its longest component",
    "k_idct": "instruction issue (about 108 instructions per sample)",
    "k_decode": "latency: too few components in flight per SM for the entropy step",
}


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--batch", type=int, default=64)
    ap.add_argument("--unique", type=int, default=0, help="distinct pictures in a batch (0: all of them)")
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--e2e-chunks", type=int, default=0,
                    help="parts the end-to-end batch is split over (0: the tuned staging depth)")
    ap.add_argument("--no-tune", action="store_true", help="keep the cached or default launch shapes")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-configs", action="store_true", help="skip the other benchmark configurations")
    ap.add_argument("--no-check", action="store_true", help="skip the bit-exactness checks against the oracle")
    ap.add_argument("--serve-seconds", type=float, default=60.0, help="0 skips the serving run")
    ap.add_argument("--serve-rate", type=float, default=2000.0, help="mean requests/s (Poisson)")
    return ap.parse_args()


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """Samples nvidia-smi every 200 ms while the timed region runs."""

    Q = ("index,uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid: str):
        self.uuid = uuid
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        self.file.flush()
        self.file.seek(0)
        rows = [r.split(", ") for r in self.file.read().strip().splitlines() if r.strip()]
        os.unlink(self.file.name)
        mine = [r for r in rows if len(r) >= 10 and (not self.uuid or self.uuid in r[1])] or \
               [r for r in rows if len(r) >= 10]
        if not mine:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(r[2]) for r in mine if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in mine for i in range(4) if r[6 + i].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": float(mine[0][3]),
                "reasons": reasons, "samples": len(mine),
                "power_w_max": max(float(r[4]) for r in mine if r[4].replace(".", "").isdigit())}


# ---------------------------------------------------------------- CPU codec

def _oracle_pic(f):
    from oracle import oracle as O

    return O.Picture(f.width, f.height, f.bit_depth, f.chroma.value, f.interlace.value,
                     (f.metadata.aspect_ratio, f.metadata.frame_rate_code, f.metadata.color_primaries,
                      f.metadata.transfer_characteristic, f.metadata.matrix_coefficients), f.data, f.alpha)


def _oracle_cfg(c):
    from oracle import oracle as O

    return O.Config(c.profile.value, c.log2_slice_mbs, c.alpha.value, c.luma_matrix, c.chroma_matrix,
                    c.target_frame_bytes, c.encoder_identifier)


def _best(fn, reps):
    best = None
    for _ in range(reps):
        t = time.perf_counter()
        fn()
        dt = time.perf_counter() - t
        best = dt if best is None else min(best, dt)
    return best


def cpu_codec_rates(frames, cfg, threads: int, reps: int = 5):
    """The oracle's CPU codec (the crate's slice-parallel path, restated) on
    `threads` host threads (0: all): encode and decode timed separately,
    best of `reps`, with the pictures and packets prepared outside the
    timed region. Returns (encode fps, decode fps)."""
    from dataclasses import replace

    from oracle import oracle as O

    pics = [_oracle_pic(f) for f in frames]
    c = replace(_oracle_cfg(cfg), threads=threads)
    packets = []
    for p in pics:
        k, msg, pkt = O.encode(c, p)
        assert k == 0, msg
        packets.append(pkt)

    def enc():
        for p in pics:
            assert O.encode(c, p)[0] == 0

    def dec():
        for pkt in packets:
            assert O.decode(pkt, 0, threads)[0] == 0

    return len(pics) / _best(enc, reps), len(pics) / _best(dec, reps)


def cpu_baseline(frames, cfg):
    """Encode and decode rates of the CPU codec at every host thread and at
    one, beside the crate's own published rates for comparison."""
    import rivet_prores_b200 as P

    cores = os.cpu_count()
    n_all = min(4, len(frames))
    enc_all, dec_all = cpu_codec_rates(frames[:n_all], cfg, 0, reps=5)
    enc_1, dec_1 = cpu_codec_rates(frames[:1], cfg, 1, reps=5)
    rt = 1.0 / (1.0 / enc_all + 1.0 / dec_all)
    return {"value": round(rt, 3), "unit": "frames/s", "cores": cores, "kind": "port",
            "encode_fps": round(enc_all, 3), "decode_fps": round(dec_all, 3),
            "encode_fps_1_thread": round(enc_1, 3), "decode_fps_1_thread": round(dec_1, 3),
            "sample": f"UHD 422 HQ frames: encode and decode timed separately, best of 5, pictures prepared "
                      f"outside the timed region; {n_all} frames on all {cores} host threads, 1 frame on 1 thread; "
                      f"`value` is the round trip (1 / (1/encode + 1/decode)) on all threads",
            "code": CPU_CODE, "published_crate": PUBLISHED_CRATE}


def headline_config(batch, unique, world):
    """The headline workload, the same for both arms: a step encodes `batch`
    UHD 422 HQ frames (`unique` distinct pictures) on each of `world` ranks
    and decodes their packets."""
    return {"workload": "uhd_422hq_transcode", "frames_per_step": batch, "distinct_pictures": unique,
            "width": W, "height": H, "chroma": "4:2:2", "bit_depth": 10, "profile": "HQ (apch)",
            "target_frame_bytes": TARGET, "step": "encode the frames, then decode their packets",
            "l2": "inputs larger than L2 (B x 33 MB of planes per step)",
            "parallelism": f"{world} rank(s), frames split by macroblock count, no collective"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O
    from rivet_prores_b200 import workloads

    n = 2
    frames = workloads.uhd_422_hq(n, config=1, unique=n)
    cfg = O.Config(3)
    pics = [_oracle_pic(f) for f in frames]

    def step():
        for p in pics:
            k, msg, pkt = O.encode(cfg, p)
            assert k == 0, msg
            k, msg, _ = O.decode(pkt)
            assert k == 0, msg

    for _ in range(args.warmup):
        step()
    t = time.perf_counter()
    for _ in range(args.steps):
        step()
    dt = time.perf_counter() - t
    fps = n * args.steps / dt
    cores = os.cpu_count()
    sample = (f"the workload's first {n} UHD 422 HQ frames each step (encode + decode each), oracle codec on "
              f"{cores} threads")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(fps, 3), "unit": "frames/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1000 * dt / args.steps, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded PCG64 cosines + rectangles + noise)",
        "config": headline_config(args.batch, args.unique or args.batch, int(os.environ.get("WORLD_SIZE", "1"))),
        "form": f"each step a bounded sample of the workload: {n} of its frames encoded and decoded on the host "
                f"cores, one after the other",
        "cpu_baseline": {"value": round(fps, 3), "unit": "frames/s", "cores": cores, "kind": "port",
                         "sample": sample, "code": CPU_CODE, "published_crate": PUBLISHED_CRATE},
        "e2e": {"value": round(fps, 3), "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


# ---------------------------------------------------------------- GPU

def time_jobs(enc, dec, stream, steps, warmup):
    """Device times (ms, summed over `steps`) of the encode and the decode
    job, each one CUDA-graph launch a step, with CUDA events on the
    launching stream."""
    import torch

    for _ in range(warmup):
        enc.launch(stream, graph=True)
        dec.launch(stream, graph=True)
    stream.synchronize()
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(steps)]
    with torch.cuda.stream(stream):
        for k in range(steps):
            ev[k][0].record(stream)
            enc.launch(stream, graph=True)
            ev[k][1].record(stream)
            dec.launch(stream, graph=True)
            ev[k][2].record(stream)
    stream.synchronize()
    t_enc = sum(ev[k][0].elapsed_time(ev[k][1]) for k in range(steps))
    t_dec = sum(ev[k][1].elapsed_time(ev[k][2]) for k in range(steps))
    return t_enc, t_dec, ev[0][0].elapsed_time(ev[-1][2])


def check_exact(frames, configs, packets, planes):
    """Every packet equals the oracle's encode of its frame, and every
    decoded picture the oracle's decode of its packet."""
    import numpy as np

    from oracle import oracle as O

    bad = []
    for i, (f, c) in enumerate(zip(frames, configs)):
        k, msg, want = O.encode(_oracle_cfg(c), _oracle_pic(f))
        if k != 0 or bytes(packets[i]) != want:
            bad.append(f"packet {i}")
            continue
        k, msg, pic = O.decode(want)
        d = planes[i]
        if k != 0 or not np.array_equal(d.data, pic.data) or (pic.alpha is not None and
                                                            not np.array_equal(d.alpha, pic.alpha)):
            bad.append(f"picture {i}")
    return not bad, bad[:5]


def run_config(name, batch, stream, steps, warmup, check, local):
    """One benchmark configuration: its frames encoded in one graph-captured
    launch and their packets decoded in another, each timed over `steps`
    launches; throughput, algorithmic HBM GB/s and bit-exactness."""
    import rivet_prores_b200 as P

    frames = [f for f, _ in batch]
    configs = [c for _, c in batch]
    enc = P.EncodeJob(frames, configs, device=local)
    enc.launch(stream)
    packets = enc.fetch(stream)
    assert all(isinstance(p, bytes) for p in packets), packets[:1]
    dec = P.DecodeJob(packets, device=local)
    dec.launch(stream)
    planes = dec.fetch(stream)
    t_enc, t_dec, _ = time_jobs(enc, dec, stream, steps, warmup)
    n = len(frames)
    samples = sum(int(f.data.size) + (0 if f.alpha is None else int(f.alpha.size)) for f in frames)
    pkt_bytes = sum(len(p) for p in packets)
    out = {"frames": n, "encode_fps": round(n * steps / (t_enc / 1000.0), 2),
           "decode_fps": round(n * steps / (t_dec / 1000.0), 2),
           "encode_ms": round(t_enc / steps, 4), "decode_ms": round(t_dec / steps, 4),
           "algorithmic_bytes": 2 * samples + pkt_bytes,
           "decode_hbm_gbs": round((2 * samples + pkt_bytes) / (t_dec / steps / 1000.0) / 1e9, 2),
           "encode_hbm_gbs": round((2 * samples + pkt_bytes) / (t_enc / steps / 1000.0) / 1e9, 2),
           "form": "one CUDA-graph launch per direction over the whole batch, resident buffers"}
    if check:
        out["bit_exact"], bad = check_exact(frames, configs, packets, planes)
        if bad:
            out["mismatches"] = bad
    enc.close()
    dec.close()
    # Where the time goes: one profiled launch of each direction.
    os.environ["PRORES_PROFILE_KERNELS"] = "1"
    penc = P.EncodeJob(frames, configs, device=local)
    pdec = P.DecodeJob(packets, device=local)
    os.environ.pop("PRORES_PROFILE_KERNELS")
    for key, job in (("encode_kernels_ms", penc), ("decode_kernels_ms", pdec)):
        job.launch(stream)
        stream.synchronize()
        ms = {}
        for kname, t in job.kernel_times():
            if kname.startswith("k_"):
                ms[kname] = round(ms.get(kname, 0.0) + t, 4)
        out[key] = dict(sorted(ms.items(), key=lambda x: -x[1]))
        job.close()
    return name, out


def run_b200(args):
    import numpy as np
    import torch

    import rivet_prores_b200 as P
    from rivet_prores_b200 import workloads
    from rivet_prores_b200.sharding import max_over_ranks, shard_by_macroblocks

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    B = args.batch
    # This rank's share of a global batch of B x world frames, split as the
    # library's multi-device calls split one (all frames are UHD, so the
    # shares are equal).
    mine = shard_by_macroblocks([(W, H)] * (B * world), world)[rank]
    unique = args.unique or B
    distinct = workloads.uhd_422_hq_at(mine[:unique])
    frames = [distinct[k % len(distinct)] for k in range(B)]
    cfg = P.Config(P.Profile.Hq)
    stream = torch.cuda.Stream()

    # Launch shapes: tuned on this GPU before anything is timed (none of them
    # changes an output).
    tuning_note = "cached or default"
    if not args.no_tune:
        from rivet_prores_b200 import autotune

        autotune.tune(device=local, quick=True, store=False, frames=frames, stage_frames=frames)
        tuning_note = "tuned in this run (rivet_prores_b200.autotune, quick search)"
    from dataclasses import asdict

    tuning = asdict(P.context(local).tuning)

    # Resident jobs: the encoder's packets of this batch feed the decoder.
    enc = P.EncodeJob(frames, cfg, device=local)
    enc.launch(stream)
    packets = enc.fetch(stream)
    assert all(isinstance(p, bytes) for p in packets), packets[:1]
    dec = P.DecodeJob(packets, device=local)
    dec.launch(stream)
    first_planes = dec.fetch(stream)
    pkt_bytes = sum(len(p) for p in packets)

    for _ in range(args.warmup):
        enc.launch(stream, graph=True)
        dec.launch(stream, graph=True)
    stream.synchronize()
    uuid = str(getattr(torch.cuda.get_device_properties(local), "uuid", ""))
    clocks = Clocks(uuid)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    time.sleep(0.4)
    t_enc, t_dec, total = time_jobs(enc, dec, stream, args.steps, 0)
    torch.cuda.synchronize()
    clock_info = clocks.stop()
    total, t_enc, t_dec = max_over_ranks([total, t_enc, t_dec], dist, "cuda")
    frames_done = B * args.steps * world
    value = frames_done / (total / 1000.0)
    dec_fps = frames_done / (t_dec / 1000.0)
    enc_fps = frames_done / (t_enc / 1000.0)
    ms_per_step = total / args.steps

    # Per-kernel device times: a separate, profiled launch of each job (the
    # kernels bracketed by events on the launching stream).
    os.environ["PRORES_PROFILE_KERNELS"] = "1"
    penc = P.EncodeJob(frames, cfg, device=local)
    pdec = P.DecodeJob(packets, device=local)
    kernel_ms, counts = {}, {}
    for job in (penc, pdec):
        job.launch(stream)
        stream.synchronize()
        job.launch(stream)
        stream.synchronize()
        for name, ms in job.kernel_times():
            if name.startswith("k_"):
                kernel_ms[name] = kernel_ms.get(name, 0.0) + ms
                counts[name] = counts.get(name, 0) + 1
    os.environ.pop("PRORES_PROFILE_KERNELS")
    penc.close()
    pdec.close()
    launches_per_step = sum(counts.values())
    peak, peak_kind = load_peaks()
    p_frame = pkt_bytes / B
    kernels = {}
    for name, ms in sorted(kernel_ms.items(), key=lambda x: -x[1]):
        entry = {"ms_per_step": round(ms, 4), "launches": counts[name], "limiter": LIMITER.get(name)}
        if name in KERNEL_BYTES:
            fn, basis = KERNEL_BYTES[name]
            per_launch = fn(SAMPLES, p_frame) * B
            gbs = per_launch / (ms / counts[name] / 1000.0) / 1e9
            entry.update({"algorithmic_bytes_per_launch": int(per_launch), "basis": basis,
                          "achieved_gbs": round(gbs, 2), "frac": round(gbs / peak, 4)})
        kernels[name] = entry
    dominant = max(kernel_ms, key=kernel_ms.get)
    dom = kernels[dominant]
    step_bytes = 2 * (p_frame + 2 * SAMPLES) * B
    step_gbs = step_bytes / (ms_per_step / 1000.0) / 1e9
    cap = CAPTURED.get(dominant)
    roofline = {
        "kernel": dominant, "bound": "hbm", "limiter": LIMITER.get(dominant),
        "achieved": dom.get("achieved_gbs"), "peak": peak, "unit": "GB/s",
        "frac": dom.get("frac"), "peak_source": f"{peak_kind} (HBM copy bandwidth)",
        "algorithmic_bytes_per_launch": dom.get("algorithmic_bytes_per_launch"), "basis": dom.get("basis"),
        "launch_ms": round(kernel_ms[dominant] / counts[dominant], 4), "launches_per_step": counts[dominant],
        "arithmetic": "achieved = algorithmic_bytes_per_launch / launch_ms; frac = achieved / peak",
        "traffic": round(cap["dram_bytes_per_frame"] * B) if cap else None,
        "traffic_source": (cap["capture"] + ", scaled to this launch's frames; not measured by this run")
        if cap else "no capture of this kernel",
        "issue_active_pct": cap["issue_active_pct"] if cap else None,
        "thread_instructions_per_coefficient": cap.get("thread_instructions_per_coefficient") if cap else None,
        "step": {"bytes": int(step_bytes), "basis": "packet + u16 planes, each direction, every frame",
                 "ms": round(ms_per_step, 4), "achieved_gbs": round(step_gbs, 2),
                 "frac": round(step_gbs / peak, 4)},
    }

    # Plain: one frame per launch, no graph, each frame waited for.
    plain_n = min(B, 8)
    penc1 = [P.EncodeJob([frames[i]], cfg, device=local) for i in range(plain_n)]
    pdec1 = [P.DecodeJob([packets[i]], device=local) for i in range(plain_n)]
    for j in penc1 + pdec1:
        j.launch(stream)
    stream.synchronize()
    pe = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    pe[0].record(stream)
    for j in penc1:
        j.launch(stream)
        stream.synchronize()
    pe[1].record(stream)
    for j in pdec1:
        j.launch(stream)
        stream.synchronize()
    pe[2].record(stream)
    stream.synchronize()
    plain_enc_fps = plain_n / (pe[0].elapsed_time(pe[1]) / 1000.0)
    plain_dec_fps = plain_n / (pe[1].elapsed_time(pe[2]) / 1000.0)
    plain_fps = plain_n / (pe[0].elapsed_time(pe[2]) / 1000.0)
    for j in penc1 + pdec1:
        j.close()

    # End to end through the C ABI with host buffers (stream.RoundTripPipeline):
    # each step copies the frames in from pinned memory, encodes, reads the
    # packets back, copies them in, decodes and reads the planes back, the
    # batch split into parts on their own streams and host threads.
    e2e = None
    if not args.no_e2e:
        from rivet_prores_b200.stream import RoundTripPipeline, time_round_trip

        depth = args.e2e_chunks or P.context(local).tuning.staging_depth
        pipe = RoundTripPipeline(frames, cfg, depth, device=local)
        e2e_steps = max(2, args.steps // 2)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        t = time_round_trip(pipe, e2e_steps, warmup=2) * e2e_steps
        h2d, d2h = pipe.bytes_per_step()
        t = max_over_ranks([t], dist, "cuda")[0]
        sec = t / 1000.0
        e2e = {"value": round(B * e2e_steps * world / sec, 3), "unit": "frames/s",
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h), "steps": e2e_steps,
               "pcie_gbs_each_way": {"h2d": round(h2d * e2e_steps / sec / 1e9, 2),
                                     "d2h": round(d2h * e2e_steps / sec / 1e9, 2)},
               "path": f"stream.RoundTripPipeline: prores_{{encode,decode}}_job_{{upload,launch,fetch}}, pinned host "
                       f"buffers, {len(pipe.parts)} parts on their own streams"}
        assert [bytes(p) for p in pipe.packets] == packets
        assert np.array_equal(pipe.planes[0], first_planes[0].data)
        pipe.close()

    # Bit-exactness on the GPU: every frame of the first step, packet and
    # picture, against the oracle.
    exact, mismatches = None, []
    if rank == 0 and not args.no_check:
        exact, mismatches = check_exact(frames[:unique], [cfg] * unique, packets, first_planes)
        if not exact:
            print(json.dumps({"error": "GPU output differs from the oracle", "where": mismatches}), file=sys.stderr)

    configs = None
    if rank == 0 and world == 1 and not args.no_configs:
        configs = {}
        for name, make in [("config1_1080p_hq_x64", lambda: workloads.hd_422_hq(64)),
                           ("config2_uhd_4444xq_alpha_x16", lambda: workloads.uhd_4444xq_alpha(16)),
                           ("config3_mixed_x96", lambda: workloads.mixed_batch(96))]:
            key, res = run_config(name, make(), stream, steps=5, warmup=3, check=not args.no_check, local=local)
            configs[key] = res

    cpu = None
    if rank == 0 and not args.no_cpu:
        cpu = cpu_baseline(frames, cfg)

    serve = None
    if rank == 0 and world == 1 and args.serve_seconds > 0:
        serve = run_serving(args, local)

    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": "frames/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded PCG64 cosines + rectangles + noise, rivet_prores_b200/workloads.py)",
        "config": headline_config(B, unique, world),
        "form": "one CUDA-graph launch per direction a step over resident buffers",
        "tuning": tuning, "tuning_source": tuning_note,
        "bit_exact": exact, "bit_exact_scope": f"all {unique} packets and pictures of the first step vs the oracle",
        "decode_fps": round(dec_fps, 3), "encode_fps": round(enc_fps, 3),
        "plain": {"value": round(plain_fps, 3), "decode_fps": round(plain_dec_fps, 3),
                  "encode_fps": round(plain_enc_fps, 3), "frames": plain_n,
                  "form": "one frame per launch, no graph, waited for"},
        "e2e": e2e,
        "gpu_launches": launches_per_step * args.steps,
        "kernels_ms_per_step": {k: v["ms_per_step"] for k, v in kernels.items()},
        "kernels": kernels,
        "roofline": roofline,
        "configs": configs,
        "cpu_baseline": cpu,
        "serve": serve,
        "clocks": clock_info,
    }
    print(json.dumps(line))


def run_serving(args, device):
    """Poisson requests (70 % decode, 30 % encode) over the heterogeneous
    mix, served with continuous batching under an 8 GiB device budget: at
    the offered rate for the full run (with p50/p99 per 10 s window, to show
    whether the queue is stationary), at half the rate, and the offered
    load served one request per launch."""
    import numpy as np

    import rivet_prores_b200 as P
    from rivet_prores_b200 import serve as S
    from rivet_prores_b200 import workloads

    pool = workloads.mixed_pool()
    packets = [P.Encoder(c, device=device).encode(f) for f, c in pool]
    # Requests arrive in page-locked receive buffers.
    receive = S.PinnedPool()
    pool = [(S.pinned_frame(f, receive), c) for f, c in pool]
    packets = [S.pinned_bytes(p, receive) for p in packets]

    def maker(seed):
        rng = np.random.Generator(np.random.PCG64(seed))

        def make(i):
            k = int(rng.integers(len(pool)))
            if rng.random() < 0.7:
                return ("decode", packets[k])
            return ("encode", pool[k][0], pool[k][1])
        return make

    out = {"mix": "720x486i HQ, 720p LT, 1080p Proxy/422/HQ, UHD HQ, 4096x2160 4444 (16-bit in); 70/30 decode/encode",
           "budget_bytes": 8 << 30,
           "host_buffers": "requests (packets, frames) in page-locked receive buffers; decoded planes into "
                           "pooled page-locked buffers"}
    window = 10.0
    # (name, workers, batch cap, seconds, offered rate, warm-up rate): a batched
    # server warms up at the offered rate, so that its workspaces and output
    # pools have grown to the batches that rate makes before anything is
    # measured (as a server in service would have); the plain form, which
    # cannot keep up with that rate, at a rate it can.
    for name, workers, max_batch, seconds, rate, warm in [
            ("batched", 4, 16, args.serve_seconds, args.serve_rate, args.serve_rate),
            ("batched_half_load", 4, 16, max(1.0, min(20.0, args.serve_seconds / 2)), args.serve_rate / 2,
             args.serve_rate),
            ("plain", 1, 1, max(1.0, min(10.0, args.serve_seconds / 6)), args.serve_rate, 200.0)]:
        # One backend (and its pool of page-locked output buffers) for the
        # warm-up and the measured run.
        backend = S.GpuBackend(device)
        srv = S.Server(backend, memory_budget=8 << 30, max_batch=max_batch, workers=workers, device=device)
        S.poisson_run(srv, maker(1), rate=warm, seconds=2.0 if warm > 200.0 else 0.3)  # not measured
        srv.close()
        srv = S.Server(backend, memory_budget=8 << 30, max_batch=max_batch, workers=workers, device=device)
        st = S.poisson_run(srv, maker(2), rate=rate, seconds=seconds, window=window)
        srv.close()
        out[name] = st
    return out


def main():
    args = parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
