"""Frames across ranks: the shares cover every frame once and balance the
macroblocks; the slowest rank's time is what every rank reports (gloo,
world size 2, on the CPU)."""

import os
import socket

import pytest
import torch.multiprocessing as mp

from rivet_prores_b200.sharding import macroblocks, max_over_ranks, shard_by_macroblocks


def test_shards_cover_every_frame_once_and_balance():
    sizes = [(3840, 2160)] * 5 + [(1920, 1080)] * 7 + [(720, 486)] * 3 + [(4096, 2160)]
    for world in (1, 2, 3, 8):
        shards = shard_by_macroblocks(sizes, world)
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(len(sizes)))
        loads = [sum(macroblocks(*sizes[i]) for i in s) for s in shards]
        assert max(loads) - min(loads) <= max(macroblocks(*s) for s in sizes)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, q):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    sizes = [(3840, 2160), (1920, 1080), (1280, 720), (720, 486), (3840, 2160)]
    mine = shard_by_macroblocks(sizes, world)[rank]
    # Each rank's "time" is its macroblocks; everyone reports the maximum.
    t = float(sum(macroblocks(*sizes[i]) for i in mine))
    got = max_over_ranks([t, -t], dist)
    dist.barrier()
    q.put((rank, mine, got))
    dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_ranks_split_the_frames_and_agree_on_the_slowest():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=100) for _ in range(2))
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    (_, a, ga), (_, b, gb) = res
    assert sorted(a + b) == list(range(5)) and not set(a) & set(b)
    assert ga == gb


def test_the_split_is_the_librarys():
    """shard_by_macroblocks (ranks under torchrun) and prores_shard_frames
    (the library's multi-device batch calls) split alike."""
    import ctypes

    import numpy as np

    from rivet_prores_b200 import _abi

    rng = np.random.Generator(np.random.PCG64(5))
    kinds = [(3840, 2160), (4096, 2160), (1920, 1080), (1280, 720), (720, 486), (16, 16), (33, 17)]
    for trial in range(50):
        n = int(rng.integers(0, 40))
        sizes = [kinds[int(k)] for k in rng.integers(0, len(kinds), n)]
        world = int(rng.integers(1, 9))
        w = (ctypes.c_uint32 * max(n, 1))(*[s[0] for s in sizes])
        h = (ctypes.c_uint32 * max(n, 1))(*[s[1] for s in sizes])
        part = (ctypes.c_int * max(n, 1))()
        assert _abi.lib().prores_shard_frames(w, h, n, world, part) == _abi.OK
        lib_split = [[i for i in range(n) if part[i] == r] for r in range(world)]
        assert lib_split == shard_by_macroblocks(sizes, world), (trial, sizes, world)
