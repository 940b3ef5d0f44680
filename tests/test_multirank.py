"""The N > 1 path of bench.py on CPU: two gloo ranks, each with its own frame
seed, combine their timings with a max, their ray counts with a sum, and
their films (sample slices of one image) with a sum-reduce into rank 0."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    from magik_b200 import dist as D
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms = [10.0 + rank, 5.0 * (2 - rank)]  # per-rank step times
        mx = D.max_over_ranks(ms)
        rays = D.sum_over_ranks([1000 * (rank + 1)])
        import torch
        film = torch.full((6,), float(rank + 1), dtype=torch.float32)
        film[0] = 10.0 * (rank + 1)
        D.reduce_film(film)
        q.put((rank, D.frame_seed(0x5EED, rank), mx, rays, film.tolist()))
    finally:
        dist.destroy_process_group()


def test_two_rank_weak_scaling_aggregation():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    seeds = {o[1] for o in out}
    assert len(seeds) == 2
    for rank, _, mx, rays, film in out:
        assert mx == [11.0, 10.0]
        assert rays == [3000.0]
        if rank == 0:  # mean of the two sample slices
            assert film == [15.0, 1.5, 1.5, 1.5, 1.5, 1.5]


def test_frame_seed_rank0_is_base():
    from magik_b200 import dist as D
    assert D.frame_seed(0x5EED, 0) == 0x5EED
