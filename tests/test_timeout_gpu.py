"""Bounded waits. Every wait of the host for the device is bounded by the
context's limit; one that runs out raises Error.Timeout instead of hanging,
the work is left to finish, and the context and the job stay usable (the
crate's promise that every failure comes back as an error,
src/error.rs:3-5, pool.rs:138-143).

The stall is made on the host, not on the device: a host function (libc's
sleep, queued with cudaLaunchHostFunc) holds the stream for a second ahead
of the decode, so nothing ever waits on the GPU itself."""

import ctypes
import time

import numpy as np
import pytest

import rivet_prores_b200 as P
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _hold_stream(stream, seconds: int):
    """Queues libc sleep(seconds) on `stream` as a host function: the stream
    makes no progress for that long."""
    rt = ctypes.CDLL("libcudart.so.12")  # the runtime the library has loaded already
    libc = ctypes.CDLL("libc.so.6")
    rt.cudaLaunchHostFunc.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    rt.cudaLaunchHostFunc.restype = ctypes.c_int
    fn = ctypes.cast(libc.sleep, ctypes.c_void_p)
    assert rt.cudaLaunchHostFunc(ctypes.c_void_p(stream.cuda_stream), fn, ctypes.c_void_p(seconds)) == 0


def test_a_wait_that_runs_out_is_a_timeout_and_the_job_survives():
    import torch

    pic = O.test_frame(352, 288, 2, 10, 12, 7)
    k, msg, pkt = O.encode(O.Config(3), pic)
    assert k == 0, msg
    k, msg, want = O.decode(pkt)
    ctx = P.context(0)
    saved = ctx.timeout_ms
    job = P.DecodeJob([pkt])
    stream = torch.cuda.Stream()
    try:
        ctx.timeout_ms = 150
        _hold_stream(stream, 1)
        job.launch(stream)
        t = time.perf_counter()
        with pytest.raises(P.Error.Timeout):
            job.fetch(stream)
        assert time.perf_counter() - t < 0.9  # gave up at the limit, not when the stream freed
        stream.synchronize()
        # The same job, fetched again once the stream has moved on.
        got = job.fetch(stream)[0]
        assert np.array_equal(got.data, want.data)
    finally:
        ctx.timeout_ms = saved
        job.close()
    # The context still decodes and encodes.
    assert np.array_equal(P.Decoder.new().decode(pkt).data, want.data)
    f = P.Frame.new(352, 288, P.ChromaFormat.Yuv422, 10)
    f.data[:] = pic.data
    assert P.Encoder(P.Config(P.Profile.Hq)).encode(f) == pkt


def test_an_encode_job_times_out_and_recovers():
    import torch

    pic = O.test_frame(352, 288, 2, 10, 12, 9)
    k, msg, want = O.encode(O.Config(3), pic)
    assert k == 0, msg
    f = P.Frame.new(352, 288, P.ChromaFormat.Yuv422, 10)
    f.data[:] = pic.data
    ctx = P.context(0)
    saved = ctx.timeout_ms
    job = P.EncodeJob([f], P.Config(P.Profile.Hq))
    stream = torch.cuda.Stream()
    try:
        ctx.timeout_ms = 150
        _hold_stream(stream, 1)
        job.launch(stream)
        with pytest.raises(P.Error.Timeout):
            job.fetch(stream)
        stream.synchronize()
        assert job.fetch(stream)[0] == want
    finally:
        ctx.timeout_ms = saved
        job.close()


def test_the_limit_is_the_contexts_and_zero_means_none():
    ctx = P.context(0)
    saved = ctx.timeout_ms
    assert saved == 60000
    try:
        ctx.timeout_ms = 0
        assert ctx.timeout_ms == 0
        pic = O.test_frame(64, 32, 2, 10, 0, 1)
        k, msg, pkt = O.encode(O.Config(3), pic)
        assert np.array_equal(P.Decoder.new().decode(pkt).data, O.decode(pkt)[2].data)
    finally:
        ctx.timeout_ms = saved
