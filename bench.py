"""ProRes UHD 422 HQ throughput on B200.

One step = encode a batch of B 3840x2160 4:2:2 10-bit frames as 422 HQ
(apch, target 3 643 238 B each) and decode the B packets back to planes,
each direction one batched, CUDA-graph-captured launch on device-resident
buffers. `value` is frames/s through both directions (B per step);
decode-only and encode-only rates, the plain one-frame-per-launch forms,
and the end-to-end rate through the C ABI with host buffers (`e2e`) are
reported beside it. Inputs are seeded synthetic pictures
(rivet_prores_b200/workloads.py); every step's inputs (B x 33 MB of planes)
are larger than L2.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--batch B] [--impl b200|reference]

Under torchrun each rank codes its own batch (weak scaling, no collective
on the data path); times are the max over ranks. `--impl reference` times
the reference codec's CPU path (the oracle's restatement of it, with its
slice-parallel thread pool on every host core) on the same workload.
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
# Algorithmic bytes per frame and direction: the packet (3 643 238 B at the
# 422 HQ target) plus the 16.59 M u16 samples of the planes.
ALGO_BYTES_PER_FRAME = 3_643_238 + 2 * (W * H * 2)
# DRAM bytes (read + write) per frame and launch, and issue-slot use, from
# one ncu capture of 14 UHD 422 HQ frames (profiles/kernels_uhd_422hq_b14.md;
# traffic grows with the frames a launch covers). k_cost is the mean of its
# nine probe launches.
PROFILED = {
    "k_cost": {"dram_bytes_per_frame": 51.29e6, "issue_active_pct": "39-54"},
    "k_idct": {"dram_bytes_per_frame": 51.28e6, "issue_active_pct": "80"},
    "k_fdct": {"dram_bytes_per_frame": 97.77e6, "issue_active_pct": "83"},
    "k_entropy": {"dram_bytes_per_frame": 40.13e6, "issue_active_pct": "57"},
    "k_pack": {"dram_bytes_per_frame": 78.75e6, "issue_active_pct": "61"},
}


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--batch", type=int, default=32)
    ap.add_argument("--unique", type=int, default=4, help="distinct synthetic pictures in a batch")
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--e2e-chunks", type=int, default=0,
                    help="parts the end-to-end batch is split over (0: the tuned staging depth)")
    ap.add_argument("--no-tune", action="store_true", help="keep the cached or default launch shapes")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--serve-seconds", type=float, default=8.0, help="0 skips the serving run")
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


def cpu_baseline(frames, cfg_oracle, reps=3):
    """The oracle's slice-parallel CPU codec on every host core: best of
    `reps` runs over the sample, encode then decode of each frame."""
    from oracle import oracle as O

    pics = [O.Picture(f.width, f.height, f.bit_depth, f.chroma.value, f.interlace.value, (0, 0, 2, 2, 2),
                      f.data, None) for f in frames]
    best = None
    for _ in range(reps):
        t = time.perf_counter()
        for p in pics:
            k, msg, pkt = O.encode(cfg_oracle, p)
            assert k == 0, msg
            k, msg, d = O.decode(pkt)
            assert k == 0, msg
        dt = time.perf_counter() - t
        best = dt if best is None else min(best, dt)
    return len(pics) / best, os.cpu_count()


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O
    from rivet_prores_b200 import workloads

    n = 2
    frames = workloads.uhd_422_hq(n, config=1, unique=n)
    cfg = O.Config(3)
    pics = [O.Picture(f.width, f.height, f.bit_depth, 2, 0, (0, 0, 2, 2, 2), f.data, None) for f in frames]

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
    sample = f"{n} UHD 422 HQ frames per step (encode + decode each), oracle codec on {cores} threads"
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(fps, 3), "unit": "frames/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1000 * dt / args.steps, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded PCG64 cosines + rectangles + noise)",
        "config": {"workload": "uhd_422hq_transcode", "frames_per_step": n, "width": W, "height": H,
                   "chroma": "4:2:2", "bit_depth": 10, "profile": "HQ (apch)",
                   "step": "encode each frame, then decode its packet"},
        "cpu_baseline": {"value": round(fps, 3), "unit": "frames/s", "cores": cores, "kind": "port",
                         "sample": sample},
        "e2e": {"value": round(fps, 3), "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def run_b200(args):
    import numpy as np
    import torch

    import rivet_prores_b200 as P
    from rivet_prores_b200 import workloads
    from rivet_prores_b200.sharding import max_over_ranks

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
    frames = workloads.uhd_422_hq(B, config=1 + rank, unique=args.unique)
    cfg = P.Config(P.Profile.Hq)
    stream = torch.cuda.Stream()

    # Launch shapes: tuned on this GPU before anything is timed (none of them
    # changes an output).
    tuning_note = "cached or default"
    if not args.no_tune:
        from rivet_prores_b200 import autotune

        autotune.tune(device=local, quick=True, store=False, frames=frames, stage_frames=frames,
                      depths=[2, 3, 4, 6, 8])
        tuning_note = "tuned in this run (rivet_prores_b200.autotune, quick search)"
    from dataclasses import asdict

    tuning = asdict(P.context(local).tuning)

    # Resident jobs: the encoder's packets of this batch feed the decoder.
    enc = P.EncodeJob(frames, cfg, device=local)
    enc.launch(stream)
    packets = enc.fetch(stream)
    assert all(isinstance(p, bytes) for p in packets), packets[:1]
    dec = P.DecodeJob(packets, device=local)

    # Bit-exactness on the GPU: the first frame's packet and picture equal
    # the oracle's.
    exact = None
    if rank == 0:
        from oracle import oracle as O

        f0 = frames[0]
        k, msg, want = O.encode(O.Config(3), O.Picture(W, H, 10, 2, 0, (0, 0, 2, 2, 2), f0.data, None))
        dec.launch(stream)
        got = dec.fetch(stream)[0]
        k2, msg2, pic = O.decode(want)
        exact = bool(k == 0 and packets[0] == want and np.array_equal(got.data, pic.data))
        if not exact:
            print(json.dumps({"error": "GPU output differs from the oracle"}), file=sys.stderr)

    def step():
        enc.launch(stream, graph=True)
        dec.launch(stream, graph=True)

    for _ in range(args.warmup):
        step()
    stream.synchronize()

    uuid = str(getattr(torch.cuda.get_device_properties(local), "uuid", ""))
    clocks = Clocks(uuid)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    time.sleep(0.4)
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    with torch.cuda.stream(stream):
        for k in range(args.steps):
            ev[k][0].record(stream)
            enc.launch(stream, graph=True)
            ev[k][1].record(stream)
            dec.launch(stream, graph=True)
            ev[k][2].record(stream)
    stream.synchronize()
    torch.cuda.synchronize()
    clock_info = clocks.stop()
    t_enc = sum(ev[k][0].elapsed_time(ev[k][1]) for k in range(args.steps))
    t_dec = sum(ev[k][1].elapsed_time(ev[k][2]) for k in range(args.steps))
    total = ev[0][0].elapsed_time(ev[-1][2])
    total, t_enc, t_dec = max_over_ranks([total, t_enc, t_dec], dist, "cuda")
    frames_done = B * args.steps * world
    value = frames_done / (total / 1000.0)
    dec_fps = frames_done / (t_dec / 1000.0)
    enc_fps = frames_done / (t_enc / 1000.0)

    # Per-kernel device times (a separate, profiled launch of each job: the
    # kernels bracketed by events on the launching stream).
    os.environ["PRORES_PROFILE_KERNELS"] = "1"
    penc = P.EncodeJob(frames, cfg, device=local)
    pdec = P.DecodeJob(packets, device=local)
    kernel_ms = {}
    counts = {}
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
    dominant = max(kernel_ms, key=kernel_ms.get)
    dom_avg = kernel_ms[dominant] / counts[dominant]
    peak, peak_kind = load_peaks()
    achieved = ALGO_BYTES_PER_FRAME * B / (dom_avg / 1000.0) / 1e9

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
        e2e = {"value": round(B * e2e_steps * world / (t / 1000.0), 3), "unit": "frames/s",
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h), "steps": e2e_steps,
               "path": f"stream.RoundTripPipeline: prores_{{encode,decode}}_job_{{upload,launch,fetch}}, pinned host "
                       f"buffers, {len(pipe.parts)} parts on their own streams"}
        assert [bytes(p) for p in pipe.packets] == packets
        assert np.array_equal(pipe.planes[0], dec.fetch(stream)[0].data)
        pipe.close()

    cpu = None
    if rank == 0 and not args.no_cpu:
        from oracle import oracle as O

        n_cpu = min(8, args.unique)
        fps, cores = cpu_baseline(frames[:n_cpu], O.Config(3))
        cpu = {"value": round(fps, 3), "unit": "frames/s", "cores": cores, "kind": "port",
               "sample": f"{n_cpu} UHD 422 HQ frames, encode + decode each, best of 3, oracle codec on "
                         f"{cores} threads"}

    serve = None
    if rank == 0 and args.serve_seconds > 0:
        serve = run_serving(args, local)

    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": "frames/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(total / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded PCG64 cosines + rectangles + noise, rivet_prores_b200/workloads.py)",
        "config": {"workload": "uhd_422hq_transcode", "frames_per_step": B, "width": W, "height": H,
                   "chroma": "4:2:2", "bit_depth": 10, "profile": "HQ (apch)", "target_frame_bytes": 3_643_238,
                   "step": "encode B frames, then decode their packets; one graph launch each, resident buffers",
                   "l2": "inputs larger than L2 (B x 33 MB of planes per step)",
                   "parallelism": f"{world} rank(s), frames sharded by rank, no collective",
                   "tuning": tuning, "tuning_source": tuning_note},
        "bit_exact": exact,
        "decode_fps": round(dec_fps, 3), "encode_fps": round(enc_fps, 3),
        "plain": {"value": round(plain_fps, 3), "decode_fps": round(plain_dec_fps, 3),
                  "encode_fps": round(plain_enc_fps, 3), "frames": plain_n,
                  "form": "one frame per launch, no graph, waited for"},
        "e2e": e2e,
        "gpu_launches": launches_per_step * args.steps,
        "kernels_ms_per_step": {k: round(v, 4) for k, v in sorted(kernel_ms.items(), key=lambda x: -x[1])},
        "roofline": {"kernel": dominant, "bound": "hbm", "achieved": round(achieved, 2), "peak": peak,
                     "unit": "GB/s", "frac": round(achieved / peak, 4),
                     "traffic": (round(PROFILED[dominant]["dram_bytes_per_frame"] * B) if dominant in PROFILED
                                 else None),
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per launch, 14 frames, "
                                       "scaled to the launch's frames (profiles/kernels_uhd_422hq_b14.md)",
                     "issue_active_pct": PROFILED.get(dominant, {}).get("issue_active_pct"),
                     "peak_source": peak_kind,
                     "algorithmic_bytes": f"{ALGO_BYTES_PER_FRAME} B per frame (packet + u16 planes) x {B}"},
        "cpu_baseline": cpu,
        "serve": serve,
        "clocks": clock_info,
    }
    print(json.dumps(line))


def run_serving(args, device):
    """Poisson requests (70 % decode, 30 % encode) over the heterogeneous
    mix, served with continuous batching under an 8 GiB device budget, at
    the offered rate (near what the server can take: throughput) and at half
    of it (latency with headroom); then the full offered load served one
    request per launch."""
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
    # Batches of at most 16: large enough to fill the device, small enough
    # that a request does not wait behind a long batch.
    for name, workers, max_batch, seconds, rate in [
            ("batched", 4, 16, args.serve_seconds, args.serve_rate),
            ("batched_half_load", 4, 16, max(1.0, args.serve_seconds / 2), args.serve_rate / 2),
            ("plain", 1, 1, max(1.0, args.serve_seconds / 4), args.serve_rate)]:
        # One backend (and its pool of page-locked output buffers) for the
        # warm-up and the measured run.
        backend = S.GpuBackend(device)
        srv = S.Server(backend, memory_budget=8 << 30, max_batch=max_batch, workers=workers, device=device)
        S.poisson_run(srv, maker(1), rate=200.0, seconds=0.3)  # workspaces allocated, not measured
        srv.close()
        srv = S.Server(backend, memory_budget=8 << 30, max_batch=max_batch, workers=workers, device=device)
        st = S.poisson_run(srv, maker(2), rate=rate, seconds=seconds)
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
