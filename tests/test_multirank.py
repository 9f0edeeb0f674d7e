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


# --- the sharded search on real per-rank results -------------------------------------
# Each rank correlates only its shard_range() of the templates against its own copy of the
# image spectrum (the oracle stands in for the GPU pass on CPU ranks), keeps (peak value,
# peak index) per template, and gather_peaks() assembles the batch in template order; the
# result must equal one rank searching every template.
SEARCH_N, SEARCH_L, SEARCH_W, SEARCH_T = 128, 24, 48, 7


def _search_inputs():
    import numpy as np

    from oracle import fastfft_oracle as O

    img = O.gaussian_blob_image(SEARCH_N, n_blobs=3, seed=O.SEED_BASE + 31)
    fout = (SEARCH_N, SEARCH_N, 1)
    spec = O.fwd(O.real_to_padded(img, fout, dtype=np.float64), fout, fout)
    rng = np.random.default_rng(O.SEED_BASE + 32)
    templates = [rng.standard_normal((SEARCH_L, SEARCH_L)) for _ in range(SEARCH_T)]
    return spec, templates


def _search_peaks(spec, templates, a, b):
    import numpy as np

    from oracle import fastfft_oracle as O

    fin, fout, iout = (SEARCH_L, SEARCH_L, 1), (SEARCH_N, SEARCH_N, 1), (SEARCH_W, SEARCH_W, 1)
    plan = O.Plan(fin, fout, fout, iout)
    vals, idxs = [], []
    for t in templates[a:b]:
        win = O.real_from_padded(O.fwd_image_inv(O.real_to_padded(t, fin), spec, plan, out_dtype=np.float64), iout)
        i, top, _ = O.peak(win)
        vals.append(top)
        idxs.append(i)
    return torch.tensor(vals, dtype=torch.float64), torch.tensor(idxs, dtype=torch.int64)


def _search_worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        spec, templates = _search_inputs()          # replicated inputs, prepared locally
        a, b = shard_range(SEARCH_T, world, rank)
        v, i = _search_peaks(spec, templates, a, b)
        gv, gi = gather_peaks(v, i, SEARCH_T)
        q.put((rank, (a, b), gv.tolist(), gi.tolist()))
    finally:
        dist.destroy_process_group()


def test_sharded_search_equals_single_rank():
    spec, templates = _search_inputs()
    ref_v, ref_i = _search_peaks(spec, templates, 0, SEARCH_T)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_search_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=180) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    spans = sorted(r[1] for r in res)
    assert spans == [(0, 4), (4, 7)]
    for _, _, v, i in res:
        assert v == ref_v.tolist()
        assert i == ref_i.tolist()
