"""Host buffers streamed through resident jobs.

`RoundTripPipeline` is the encode-then-decode path a caller of the crate's
API takes for a batch of host frames (`Encoder::encode` to host packets,
`Decoder::decode` of those packets back to host planes, src/encode.rs:223-287
and src/decode.rs:61-104), with the batch split into `depth` parts that move
on their own streams and host threads. One part's copies then overlap
another's kernels, and both copy directions run at once. Frames and results
stay in pinned host memory, so every copy is a DMA at full PCIe rate.
"""

from __future__ import annotations

import concurrent.futures as cf
import threading
from typing import List, Optional, Sequence

import numpy as np


class RoundTripPipeline:
    """Encodes `frames` (all of one size and format) with `config` and
    decodes the packets back, `depth` parts in flight.

    `run(steps)` streams the batch through `steps` times: every part copies
    its frames in from pinned memory, runs both directions and copies its
    planes out, then starts over, each part at its own pace. A part's next
    frames go up on its own upload stream as soon as its encode has read the
    last ones, so they overlap its decode and download; uploads of all
    parts queue in one order (each waits for the one issued before it), so
    the copy engine finishes one part's frames at a time and the parts fall
    into step behind one another instead of all uploading, then all
    encoding, then all downloading at once. The last packets (views into
    pinned staging, valid until the next run) and decoded planes
    (`self.planes`, one pinned row per frame) stay. It returns (start, end)
    CUDA events on `self.stream` that bracket the run on the device."""

    def __init__(self, frames: Sequence, config, depth: int, device: int = 0):
        import torch

        from . import DecodeJob, EncodeJob, Frame

        self.torch = torch
        self.device = device
        n = len(frames)
        if n == 0:
            raise ValueError("no frames")
        samples = frames[0].data.size
        if any(f.data.size != samples for f in frames):
            raise ValueError("frames of one size only")
        self.host = torch.empty((n, samples), dtype=torch.uint16, pin_memory=True).numpy()
        self.planes = torch.empty((n, samples), dtype=torch.uint16, pin_memory=True).numpy()
        depth = max(1, min(int(depth), n))
        self.bounds = [(c * n // depth, (c + 1) * n // depth) for c in range(depth)]
        self.parts = []
        for lo, hi in self.bounds:
            hframes = []
            for i in range(lo, hi):
                f = frames[i]
                self.host[i] = f.data
                hframes.append(Frame(f.width, f.height, f.bit_depth, f.chroma, f.interlace, f.metadata, self.host[i],
                                     f.planes, None))
            enc = EncodeJob(hframes, config, device=device)
            enc.launch()
            packets = enc.fetch(copy=False)
            for p in packets:
                if not isinstance(p, memoryview):
                    raise p
            dec = DecodeJob([bytes(p) for p in packets], device=device)
            self.parts.append({"enc": enc, "dec": dec, "frames": hframes, "stream": torch.cuda.Stream(device),
                               "up": torch.cuda.Stream(device),
                               "arrays": [(self.planes[i], None) for i in range(lo, hi)]})
        self.stream = torch.cuda.Stream(device)
        self.pool = cf.ThreadPoolExecutor(max_workers=depth)
        self.packets: List[memoryview] = []
        self._order = threading.Lock()
        self._last_upload = None

    def _upload(self, part):
        """Queues the part's frames behind the last upload of any part."""
        up = part["up"]
        with self._order:
            if self._last_upload is not None:
                up.wait_event(self._last_upload)
            part["enc"].upload(part["frames"], up)
            done = self.torch.cuda.Event()
            done.record(up)
            self._last_upload = done
        part["uploaded"] = done

    def _part(self, part, steps: int):
        st, up = part["stream"], part["up"]
        pk = []
        self._upload(part)
        for k in range(steps):
            st.wait_event(part["uploaded"])
            part["enc"].launch(st, graph=True)
            if k + 1 < steps:
                # The next frames may overwrite the input once this encode
                # has run.
                read = self.torch.cuda.Event()
                read.record(st)
                up.wait_event(read)
                self._upload(part)
            pk = part["enc"].fetch(st, copy=False)
            part["dec"].upload([np.frombuffer(p, dtype=np.uint8) for p in pk], st)
            part["dec"].launch(st, graph=True)
            part["dec"].fetch(st, part["arrays"])
        part["end"].record(st)
        return pk

    def run(self, steps: int = 1):
        torch = self.torch
        start = torch.cuda.Event(enable_timing=True)
        start.record(self.stream)
        self._last_upload = None
        for part in self.parts:
            part["stream"].wait_event(start)
            part["up"].wait_event(start)
            part["end"] = torch.cuda.Event(enable_timing=True)
        outs = list(self.pool.map(lambda p: self._part(p, steps), self.parts))
        for part in self.parts:
            self.stream.wait_event(part["end"])
        end = torch.cuda.Event(enable_timing=True)
        end.record(self.stream)
        self.packets = [p for o in outs for p in o]
        return start, end

    def bytes_per_step(self):
        """(host-to-device, device-to-host) bytes one step copies."""
        pk = sum(len(p) for p in self.packets)
        planes = 2 * self.host.size
        return planes + pk, pk + planes

    def close(self):
        self.pool.shutdown()
        for part in self.parts:
            part["enc"].close()
            part["dec"].close()
        self.parts = []


def time_round_trip(pipe: RoundTripPipeline, steps: int, warmup: int = 2) -> float:
    """Device milliseconds per step over `steps` streamed steps, after a
    run of `warmup`."""
    if warmup:
        pipe.run(warmup)
        pipe.stream.synchronize()
    start, end = pipe.run(steps)
    pipe.stream.synchronize()
    return start.elapsed_time(end) / steps


def frames_per_second(n_frames: int, ms_per_step: Optional[float]) -> float:
    return n_frames / (ms_per_step / 1000.0) if ms_per_step else 0.0
