"""Template sharding over two ranks (gloo, CPU): shard ranges, gathered peaks, max-over-ranks."""
import os
import socket

import pytest
import torch
import torch.multiprocessing as mp

from fastfft_b200.sharding import gather_peaks, max_over_ranks, shard_range


def test_shard_range_covers_exactly():
    for n in (0, 1, 7, 64, 1024, 1025):
        for w in (1, 2, 3, 8):
            spans = [shard_range(n, w, r) for r in range(w)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(spans[k][1] == spans[k + 1][0] for k in range(w - 1))
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard_range(4, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, n_total, q):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        a, b = shard_range(n_total, world, rank)
        # stand-in per-template results: value = template id * 1.5, index = 1000 + id
        ids = torch.arange(a, b)
        v, i = gather_peaks(ids.double() * 1.5, ids + 1000, n_total)
        t = max_over_ranks(10.0 + rank)
        q.put((rank, v.tolist(), i.tolist(), t))
    finally:
        dist.destroy_process_group()


def test_gather_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    n_total = 11
    procs = [ctx.Process(target=_worker, args=(r, 2, port, n_total, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, v, i, t in res:
        assert v == [k * 1.5 for k in range(n_total)]
        assert i == [1000 + k for k in range(n_total)]
        assert t == 11.0
