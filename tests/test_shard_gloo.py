"""The multi-rank host path on CPU: two gloo ranks split one recovery set by
byte slabs (no data exchange), each encodes its slab, and rank 0 gathers
them; the result must equal the whole-set encode.  The per-slab encode here
is the oracle (the CPU stands in for the GPU); the partitioning, the
max-over-ranks timing and the gather are the code under test."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from par2gpu.shard import TILE, column_slabs, rank_sets


def test_column_slabs_cover_once_aligned():
    for S in (2, 2048, 2050, 4096, 65536, 1 << 20, 6144 + 64):
        for world in (1, 2, 3, 4, 8):
            slabs = column_slabs(S, world)
            assert len(slabs) == world
            assert slabs[0][0] == 0 and slabs[-1][1] == S
            for (a, b), (c, _) in zip(slabs, slabs[1:]):
                assert b == c
            assert all(a % TILE == 0 and a <= b for a, b in slabs)
            sizes = [b - a for a, b in slabs if b < S]
            assert not sizes or max(sizes) - min(sizes) <= TILE


def test_rank_sets_partition():
    for n in (0, 1, 7, 256):
        for world in (1, 2, 4):
            got = sorted(i for r in range(world) for i in rank_sets(n, r, world))
            assert got == list(range(n))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    from oracle import oracle
    from par2gpu.shard import column_slabs, gather_slabs, max_over_ranks

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        rng = np.random.default_rng(5)
        k, S, r = 24, 3 * 2048 + 512, 5
        src = rng.integers(0, 256, (k, S), dtype=np.uint8)
        exps = np.arange(r, dtype=np.uint32)
        a, b = column_slabs(S, world)[rank]
        local = oracle.encode(np.ascontiguousarray(src[:, a:b]), exps)
        t = max_over_ranks(1.0 + rank)
        full = gather_slabs(local, (a, b), S)
        if rank == 0:
            q.put(("ok", bool(np.array_equal(full, oracle.encode(src, exps))), t))
    except Exception as e:  # reported to the parent
        q.put(("error", repr(e), None))
        raise
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(180)
def test_two_rank_slab_encode_gathers_to_whole_set():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    status, same, t = q.get(timeout=10)
    assert status == "ok", same
    assert same
    assert t == 2.0   # the max of the two ranks' values
    assert all(p.exitcode == 0 for p in procs)
