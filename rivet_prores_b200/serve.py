"""Serving: continuous batching of decode and encode requests on one GPU.

Requests arrive at any time (`submit_decode`, `submit_encode`, each a
Future). Worker threads each take the oldest waiting request's kind and as
many further requests of that kind, oldest first, as the device-memory
budget admits. Each batch is one launch into the library (`decode_batch` /
`encode_batch`). Requests that arrive while other batches run are admitted
as workers and memory free up, and their batches run on the device
alongside the others: each call has its own workspace and stream, and the
library releases the GIL while it runs. Every result is the one the request
would get alone; the library's output never depends on the batch.

The memory estimate per frame covers what a batch keeps on the device:
for decode the bitstream, the coefficient lists (8 B a coefficient) and the
planes; for encode the planes in, the f32 coefficients and the packet
region.
"""

from __future__ import annotations

import collections
import ctypes
import threading
import time
from concurrent.futures import Future
from dataclasses import dataclass, field
from typing import Callable, Deque, Dict, List, Optional

import numpy as np


@dataclass
class Request:
    kind: str  # "decode" or "encode"
    payload: object  # bytes for decode, Frame for encode
    config: object = None  # encode Config
    bit_depth: Optional[int] = None
    cost: int = 0  # device bytes while in flight
    t_submit: float = 0.0
    t_done: float = 0.0
    future: Future = field(default_factory=Future)


def decode_cost(data: bytes) -> int:
    """Device bytes a decode of `data` holds: bitstream, lists, planes."""
    from . import _abi

    info = _abi.Frame_()
    a = np.frombuffer(data, dtype=np.uint8) if len(data) else np.zeros(1, np.uint8)
    if _abi.lib().prores_probe(a.ctypes.data_as(ctypes.c_char_p), len(data), 0, ctypes.byref(info)) != _abi.OK:
        return len(data) + 4096
    return len(data) + 10 * info.data_len + 2 * info.alpha_len + 4096


def encode_cost(frame, config) -> int:
    """Device bytes an encode of `frame` holds: planes in, f32 coefficients,
    the packet region."""
    n = int(frame.data.size)
    target = config.target_frame_bytes or config.profile.target_frame_bytes(frame.width, frame.height)
    alpha = 0 if frame.alpha is None else 4 * frame.alpha.size
    return 6 * n + int(target) + alpha + 4096


class _Lease:
    """Exposes one pooled block to numpy; the block goes back to its pool
    when the lease (the base of every array made from it) is collected."""

    def __init__(self, mv: memoryview):
        self.mv = mv

    def __buffer__(self, flags):
        return self.mv

    def __release_buffer__(self, view):
        pass


def _pinned_block(size: int) -> np.ndarray:
    import torch

    return torch.empty(size, dtype=torch.uint8, pin_memory=True).numpy()


class PinnedPool:
    """Reusable page-locked host buffers for decoded planes.

    Fresh host memory costs a page fault per 4 KB on first touch, which for
    decoded UHD planes takes longer than the decode; pooled page-locked
    blocks are already mapped, and the device writes them by DMA with no
    staging copy. A block returns to the pool when the last array viewing it
    is collected. Blocks come in 1 MiB steps; `limit` bounds the bytes kept
    idle."""

    def __init__(self, limit: int = 4 << 30, allocate: Optional[Callable[[int], np.ndarray]] = None):
        self.limit = limit
        self.idle = 0
        self.made = 0
        self.free = collections.defaultdict(list)
        self.lock = threading.Lock()
        self.allocate = allocate or _pinned_block

    def take(self, n: int, dtype=np.uint16) -> np.ndarray:
        import weakref

        nbytes = max(1, n * np.dtype(dtype).itemsize)
        size = (nbytes + (1 << 20) - 1) & ~((1 << 20) - 1)
        with self.lock:
            block = self.free[size].pop() if self.free[size] else None
            if block is not None:
                self.idle -= size
        if block is None:
            block = self.allocate(size)
            with self.lock:
                self.made += 1
        lease = _Lease(memoryview(block))
        weakref.finalize(lease, self._give, size, block)
        return np.frombuffer(lease, dtype=np.uint8, count=nbytes).view(dtype)[:n]

    def _give(self, size, block):
        with self.lock:
            if self.idle + size <= self.limit:
                self.free[size].append(block)
                self.idle += size


def pinned_bytes(data, pool: PinnedPool) -> np.ndarray:
    """A copy of `data` in page-locked pooled memory (a receive buffer)."""
    out = pool.take(len(data), np.uint8)
    out[:] = np.frombuffer(data, dtype=np.uint8)
    return out


def pinned_frame(frame, pool: PinnedPool):
    """A copy of `frame` whose planes (and alpha) lie in page-locked pooled
    memory, as a server's receive buffers would: the device then reads them
    by DMA, with no staging copy."""
    from . import Frame

    data = pool.take(frame.data.size)
    data[:] = frame.data
    alpha = None
    if frame.alpha is not None:
        alpha = pool.take(frame.alpha.size)
        alpha[:] = frame.alpha
    return Frame(frame.width, frame.height, frame.bit_depth, frame.chroma, frame.interlace, frame.metadata, data,
                 frame.planes, alpha)


class GpuBackend:
    """The library's batched calls; decoded planes land in a pool of
    page-locked host buffers."""

    def __init__(self, device: int = 0, pool: Optional[PinnedPool] = None):
        from . import Decoder, Encoder

        self.device = device
        self._Decoder = Decoder
        self._Encoder = Encoder
        self.pool = pool if pool is not None else PinnedPool()

    def decode(self, reqs: List[Request]):
        by_depth = collections.defaultdict(list)
        for i, r in enumerate(reqs):
            by_depth[r.bit_depth].append(i)
        out = [None] * len(reqs)
        for depth, idx in by_depth.items():
            res = self._Decoder(bit_depth=depth, device=self.device).decode_batch([reqs[i].payload for i in idx],
                                                                               alloc=self.pool.take)
            for i, r in zip(idx, res):
                out[i] = r
        return out

    def encode(self, reqs: List[Request]):
        frames = [r.payload for r in reqs]
        configs = [r.config for r in reqs]
        return self._Encoder(configs[0], device=self.device).encode_batch(frames, configs)


class Server:
    """Continuous batching over `backend` (GpuBackend by default).

    memory_budget: device bytes all in-flight batches may hold together.
    max_batch: frames per batch. workers: batches in flight at once.
    """

    def __init__(self, backend=None, memory_budget: int = 8 << 30, max_batch: int = 64, workers: int = 2,
                 device: int = 0):
        self.backend = backend if backend is not None else GpuBackend(device)
        self.budget = memory_budget
        self.max_batch = max_batch
        self.in_use = 0
        # One first-in-first-out queue per kind: taking a batch pops from the
        # front of one of them, whatever is waiting behind.
        self.queues: Dict[str, Deque[Request]] = {"decode": collections.deque(), "encode": collections.deque()}
        self.waiting = 0
        self.cv = threading.Condition()
        self.closed = False
        # (submitted, done) times of finished requests: the requests
        # themselves are let go, so that their results live only as long as
        # the callers keep them.
        self.done: List[tuple] = []
        self.batches: List[int] = []
        # (kind, frames, start, end) of every batch call into the library.
        self.calls: List[tuple] = []
        self.peak_in_use = 0
        self.peak_queue = 0
        self.threads = [threading.Thread(target=self._worker, daemon=True) for _ in range(workers)]
        for t in self.threads:
            t.start()

    # -------------------------------------------------------------- intake

    def submit_decode(self, data: bytes, bit_depth: Optional[int] = None, cost: Optional[int] = None) -> Future:
        """`data`: bytes, or an array (for example a page-locked receive
        buffer, which reaches the device by DMA) that stays unchanged until
        the future resolves; other buffers are copied."""
        if not isinstance(data, (bytes, np.ndarray)):
            data = bytes(data)
        r = Request("decode", data, None, bit_depth, decode_cost(data) if cost is None else cost)
        return self._submit(r)

    def submit_encode(self, frame, config, cost: Optional[int] = None) -> Future:
        r = Request("encode", frame, config, None, encode_cost(frame, config) if cost is None else cost)
        return self._submit(r)

    def _submit(self, r: Request) -> Future:
        r.t_submit = time.perf_counter()
        with self.cv:
            if self.closed:
                raise RuntimeError("server closed")
            self.queues[r.kind].append(r)
            self.waiting += 1
            self.peak_queue = max(self.peak_queue, self.waiting)
            self.cv.notify()
        return r.future

    # -------------------------------------------------------------- batching

    def _take(self) -> List[Request]:
        """Under the lock: the oldest request's kind, and further requests of
        that kind oldest first, while the budget admits them. A request larger
        than the whole budget runs alone once nothing else is in flight."""
        heads = [q for q in self.queues.values() if q]
        q = min(heads, key=lambda d: d[0].t_submit)
        batch, cost = [], 0
        free = self.budget - self.in_use
        while q and len(batch) < self.max_batch:
            r = q[0]
            if cost + r.cost > free and not (not batch and self.in_use == 0):
                break
            batch.append(q.popleft())
            cost += r.cost
        self.waiting -= len(batch)
        self.in_use += cost
        self.peak_in_use = max(self.peak_in_use, self.in_use)
        return batch

    def _worker(self):
        while True:
            with self.cv:
                while True:
                    if self.closed and not self.waiting:
                        return
                    if self.waiting:
                        batch = self._take()
                        if batch:
                            break
                    self.cv.wait(0.05)
            t_call = time.perf_counter()
            try:
                results = self.backend.decode(batch) if batch[0].kind == "decode" else self.backend.encode(batch)
                exc = None
            except Exception as e:  # a device failure fails the batch, not the server
                results, exc = None, e
            now = time.perf_counter()
            with self.cv:
                self.in_use -= sum(r.cost for r in batch)
                self.batches.append(len(batch))
                self.calls.append((batch[0].kind, len(batch), t_call, now))
                for r in batch:
                    r.t_done = now
                    self.done.append((r.t_submit, now))
                self.cv.notify_all()
            for i, r in enumerate(batch):
                if exc is not None:
                    r.future.set_exception(exc)
                else:
                    r.future.set_result(results[i])
            del batch, results

    def close(self):
        with self.cv:
            self.closed = True
            self.cv.notify_all()
        for t in self.threads:
            t.join()

    # -------------------------------------------------------------- metrics

    def stats(self, window: float = 0.0) -> dict:
        """Latency percentiles, throughput and batching; with `window`
        seconds, the same per window of submission time (whether the queue
        is stationary), and where a request's time went: waiting for a
        worker, or in the batch call that served it."""
        with self.cv:
            done = list(self.done)
            batches = list(self.batches)
            calls = list(self.calls)
        if not done:
            return {"requests": 0}
        lat = sorted((d - a) * 1000.0 for a, d in done)
        first = min(a for a, _ in done)
        last = max(d for _, d in done)
        out = {"requests": len(lat), "p50_ms": round(_pct(lat, 50), 3), "p99_ms": round(_pct(lat, 99), 3),
               "max_ms": round(lat[-1], 3), "frames_per_s": round(len(lat) / max(last - first, 1e-9), 2),
               "batches": len(batches), "mean_batch": round(float(np.mean(batches)), 2),
               "peak_device_bytes_admitted": self.peak_in_use, "peak_queue": self.peak_queue}
        for kind in ("decode", "encode"):
            mine = [c for c in calls if c[0] == kind]
            if mine:
                ms = sorted((e - b) * 1000.0 for _, _, b, e in mine)
                out[f"{kind}_calls"] = {"count": len(mine), "mean_frames": round(float(np.mean([n for _, n, _, _ in mine])), 2),
                                        "p50_ms": round(_pct(ms, 50), 3), "p99_ms": round(_pct(ms, 99), 3)}
        if window > 0:
            wins = []
            k = 0
            while first + k * window < max(a for a, _ in done) + 1e-9:
                lo, hi = first + k * window, first + (k + 1) * window
                w = sorted((d - a) * 1000.0 for a, d in done if lo <= a < hi)
                if w:
                    wins.append({"t0_s": round(k * window, 1), "requests": len(w), "p50_ms": round(_pct(w, 50), 3),
                                 "p99_ms": round(_pct(w, 99), 3),
                                 "completed_per_s": round(sum(1 for _, d in done if lo <= d < hi) / window, 1)})
                k += 1
            out["windows"] = wins
        return out


def _pct(sorted_ms, p):
    return sorted_ms[min(len(sorted_ms) - 1, int(round(p / 100.0 * (len(sorted_ms) - 1))))]


def poisson_run(server: Server, make_request: Callable[[int], tuple], rate: float, seconds: float,
                seed: int = 0, window: float = 0.0) -> dict:
    """Submits requests at Poisson times (mean `rate` per second) for
    `seconds`; make_request(i) gives ("decode", data) or ("encode", frame,
    config). Each result is dropped as it arrives, as a client that consumes
    it would; waits for all and returns the server's stats."""
    rng = np.random.Generator(np.random.PCG64(seed))
    lock = threading.Condition()
    state = {"submitted": 0, "finished": 0, "errors": 0}

    def finished(f: Future):
        failed = f.exception() is not None
        with lock:
            state["finished"] += 1
            state["errors"] += int(failed)
            lock.notify_all()

    t0 = time.perf_counter()
    t = 0.0
    i = 0
    while True:
        t += rng.exponential(1.0 / rate)
        if t > seconds:
            break
        delay = t0 + t - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        req = make_request(i)
        if req[0] == "decode":
            fut = server.submit_decode(req[1])
        else:
            fut = server.submit_encode(req[1], req[2])
        with lock:
            state["submitted"] += 1
        fut.add_done_callback(finished)
        del fut
        i += 1
    with lock:
        while state["finished"] < state["submitted"]:
            lock.wait(1.0)
    s = server.stats(window)
    s["offered_rate"] = rate
    s["seconds"] = seconds
    s["errors"] = state["errors"]
    return s
