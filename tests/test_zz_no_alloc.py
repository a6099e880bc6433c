"""prores_decode_noalloc: decoding with no device allocation, for callers
that cannot allocate while they decode (a real-time playback thread, where
cudaMalloc can stall and cudaFree waits for the whole device; an
application whose device memory all comes from its own pool allocator).

Its output must equal the allocating prores_decode's, on consecutive calls
that share its one static scratch array. This file is collected last, so a
run that stops at the first failure has run every other test before it."""

import ctypes

import numpy as np
import pytest

import rivet_prores_b200 as P
from oracle import oracle as O
from rivet_prores_b200 import _abi

pytestmark = pytest.mark.gpu


def _entry():
    f = _abi.lib().prores_decode_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_int, ctypes.c_char_p, ctypes.c_size_t, ctypes.c_uint32, ctypes.c_void_p,
                  ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]
    return f


def _packets():
    hd = O.test_frame(1920, 1080, 2, 10, 24, 7)
    k, msg, hd_pkt = O.encode(O.Config(3), hd)
    assert k == 0, msg
    small = O.test_frame(352, 288, 3, 12, 10, 3)
    small.interlace = 1
    small.alpha = ((np.arange(352 * 288) * 37) % 4096).astype(np.uint16)
    k, msg, small_pkt = O.encode(O.Config(5), small)
    assert k == 0, msg
    return [hd_pkt, small_pkt]


def _device_memory():
    """(free bytes on the device, bytes the device's default memory pool has
    reserved): what any device allocation would change."""
    import torch

    rt = ctypes.CDLL("libcudart.so.12")
    pool = ctypes.c_void_p()
    assert rt.cudaDeviceGetDefaultMemPool(ctypes.byref(pool), 0) == 0
    reserved = ctypes.c_uint64()
    assert rt.cudaMemPoolGetAttribute(pool, 5, ctypes.byref(reserved)) == 0  # cudaMemPoolAttrReservedMemCurrent
    torch.cuda.synchronize()
    return torch.cuda.mem_get_info(0)[0], reserved.value


def test_decode_without_allocation_equals_the_allocating_decode():
    import torch

    decode = _entry()
    packets = _packets()
    wants = [P.Decoder.new().decode(p) for p in packets]
    outs = []
    for p in packets:
        info = _abi.Frame_()
        assert _abi.lib().prores_probe(p, len(p), 0, ctypes.byref(info)) == _abi.OK
        planes = torch.empty(info.data_len, dtype=torch.int16, device="cuda")
        alpha = torch.empty(max(info.alpha_len, 1), dtype=torch.int16, device="cuda")
        outs.append((info, planes, alpha))
    # One call first (it sets the device up and loads the kernels), and
    # everything else the loop below runs once (torch loads its kernels on
    # first use too); from then on nothing may change what the device has
    # allocated.
    for info, planes, alpha in outs:
        planes.fill_(-1)
        alpha.fill_(-1)
        planes.cpu()
        alpha.cpu()
    info, planes, alpha = outs[0]
    assert decode(0, packets[0], len(packets[0]), 0, planes.data_ptr(), info.data_len, None, 0, None) == _abi.OK
    before = _device_memory()
    # Two calls in a row on each frame, then the frames interleaved: every
    # call shares the scratch the previous call left behind.
    for i in [0, 0, 1, 1, 0, 1]:
        info, planes, alpha = outs[i]
        planes.fill_(-1)
        alpha.fill_(-1)
        p = packets[i]
        rc = decode(0, p, len(p), 0, planes.data_ptr(), info.data_len,
                    alpha.data_ptr() if info.alpha_len else None, info.alpha_len, None)
        assert rc == _abi.OK, _abi.last_error()
        got = planes.cpu().numpy().view(np.uint16)
        assert np.array_equal(got, wants[i].data), f"frame {i}"
        if info.alpha_len:
            assert np.array_equal(alpha.cpu().numpy().view(np.uint16)[: info.alpha_len], wants[i].alpha)
    assert _device_memory() == before, "a call allocated device memory"


def test_frames_beyond_the_scratch_are_refused():
    import torch

    decode = _entry()
    uhd = O.test_frame(3840, 2160, 2, 10, 0, 1)
    k, msg, pkt = O.encode(O.Config(3), uhd)
    assert k == 0, msg
    info = _abi.Frame_()
    assert _abi.lib().prores_probe(pkt, len(pkt), 0, ctypes.byref(info)) == _abi.OK
    planes = torch.empty(info.data_len, dtype=torch.int16, device="cuda")
    rc = decode(0, pkt, len(pkt), 0, planes.data_ptr(), info.data_len, None, 0, None)
    assert rc == _abi.CONFIG
    assert "prores_decode_noalloc" in _abi.last_error()
