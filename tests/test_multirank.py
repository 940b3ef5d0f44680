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


# ------------------------------------------- data-parallel surrogate training
class _LinearNet:
    """A linear least-squares model with the surrogate's step interface
    (shuffle / gradient_step / adam_step): the host logic of the data-parallel
    training loop without a GPU.  Its 'Adam step' is plain gradient descent on
    the same cosine step-size schedule."""
    grad_dtype = None  # set to torch.float64 on construction

    def __init__(self, dim):
        import torch
        self.grad_dtype = torch.float64
        self.w = torch.zeros(dim, dtype=torch.float64)
        self.order = None

    @property
    def param_count(self):
        return self.w.numel()

    def shuffle(self, seed, epoch, n, stream=None):
        import numpy as np
        import torch
        self.order = torch.from_numpy(np.random.default_rng([int(seed), int(epoch)]).permutation(n))

    def gradient_step(self, cfg, feat, lab, first, n, grad, loss, stream=None):
        rows = self.order[first:first + n]
        X, y = feat[rows], lab[rows]
        r = X @ self.w - y
        grad.copy_((2.0 / n) * (X.T @ r))
        loss += (r * r).mean()

    def adam_step(self, cfg, grad, scale, progress, stream=None):
        import math
        lr = cfg.lr_final + 0.5 * (cfg.lr - cfg.lr_final) * (1.0 + math.cos(math.pi * progress))
        self.w -= lr * (grad * scale)


def _shard(rank, n=4096, dim=5):
    import torch
    g = torch.Generator().manual_seed(100 + rank)
    X = torch.randn(n, dim, generator=g, dtype=torch.float64)
    w_true = torch.arange(1, dim + 1, dtype=torch.float64)
    return X, X @ w_true + 0.01 * torch.randn(n, generator=g, dtype=torch.float64)


def _train_cfg():
    from types import SimpleNamespace
    return SimpleNamespace(batch=2048, epochs=3, seed=0x7EA1, lr=0.3, lr_final=0.05)


def _union_batch_training(world, cfg):
    """The expected run: every step a gradient step on the union of the
    ranks' batches (the mean of the ranks' batch-mean gradients)."""
    import math
    import numpy as np
    import torch
    from magik_b200 import dist as D
    shards = [_shard(r) for r in range(world)]
    b = cfg.batch // world
    n = shards[0][0].shape[0]
    nb = n // b
    w = torch.zeros(shards[0][0].shape[1], dtype=torch.float64)
    losses = []
    for ep in range(cfg.epochs):
        orders = [torch.from_numpy(np.random.default_rng([D.frame_seed(cfg.seed, r), ep]).permutation(n))
                  for r in range(world)]
        tot = 0.0
        for k in range(nb):
            gs = []
            for r, (X, y) in enumerate(shards):
                rows = orders[r][k * b:(k + 1) * b]
                res = X[rows] @ w - y[rows]
                gs.append((2.0 / b) * (X[rows].T @ res))
                tot += float((res * res).mean())
            g = gs[0]
            for h in gs[1:]:
                g = g + h
            lr = cfg.lr_final + 0.5 * (cfg.lr - cfg.lr_final) * (1.0 + math.cos(math.pi * (ep * nb + k) / (cfg.epochs * nb)))
            w = w - lr * (g * (1.0 / world))
        losses.append(tot / (nb * world))
    return w, losses


def _dp_worker(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    from magik_b200 import dist as D
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        net = _LinearNet(5)
        X, y = _shard(rank)
        losses = D.train_data_parallel(net, _train_cfg(), X, y)
        q.put((rank, net.w.tolist(), [float(v) for v in losses]))
    finally:
        dist.destroy_process_group()


def test_two_rank_data_parallel_training_is_union_batch_training():
    """Two gloo ranks with their own shards end with the same parameters,
    those of training on the union batches, and report the mean loss of
    both ranks' batches."""
    import numpy as np
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_dp_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    w_want, loss_want = _union_batch_training(2, _train_cfg())
    assert out[0][1] == out[1][1]  # every rank holds the same parameters
    np.testing.assert_allclose(out[0][1], w_want.tolist(), rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(out[0][2], loss_want, rtol=1e-6)
    assert out[0][2][-1] < 0.1 * out[0][2][0]  # it trains


def test_one_rank_data_parallel_training_and_batch_checks():
    import numpy as np
    from magik_b200 import dist as D
    cfg = _train_cfg()
    net = _LinearNet(5)
    X, y = _shard(0)
    losses = D.train_data_parallel(net, cfg, X, y)
    w_want, loss_want = _union_batch_training(1, cfg)
    np.testing.assert_allclose(net.w.numpy(), w_want.numpy(), rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(losses, loss_want, rtol=1e-6)
    cfg.batch = 1000
    with pytest.raises(ValueError):
        D.train_data_parallel(_LinearNet(5), cfg, X, y)
    cfg.batch = 8192
    with pytest.raises(ValueError):  # fewer samples than one batch
        D.train_data_parallel(_LinearNet(5), cfg, X, y)


def _strong_worker(rank, world, port, q):
    """One rank of bench.py's strong split with the CPU oracle standing in
    for the GPU render: bench.scene_config gives the rank its slice of the
    frame's samples, the oracle renders it, and dist.reduce_slices (the
    exchange step of run_gpu) assembles the frame in rank 0."""
    import argparse
    import datetime
    import sys
    import numpy as np
    import torch
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import bench
    import magik_b200 as M
    from magik_b200 import dist as D
    from oracle import oracle_py as O
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        bench.ARGS = argparse.Namespace(split="spp", width=24, height=16, spp=6)
        s = bench.scene_config(M, rank, world)
        stars = M.star_catalog(0x57A25, 20000)
        w = M.xyz_weights(s.n_bins)
        film, _ = O.render_pixels(s, stars, w, 0, s.width * s.height, nthreads=2)
        f = torch.from_numpy(np.ascontiguousarray(film, dtype=np.float64).ravel())
        D.reduce_slices(f, s.spp, 6)
        q.put((rank, int(s.sample_offset), int(s.spp), int(s.seed), f.numpy().tolist() if rank == 0 else None))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 4])
def test_strong_split_assembles_the_one_rank_frame(world):
    import numpy as np
    import magik_b200 as M
    from oracle import oracle_py as O
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_strong_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # contiguous, disjoint slices of the 6 samples, one seed
    offs = [(o[1], o[2]) for o in out]
    assert sum(c for _, c in offs) == 6 and all(offs[i][0] + offs[i][1] == offs[i + 1][0] for i in range(world - 1))
    assert len({o[3] for o in out}) == 1
    s = M.scene_defaults(width=24, height=16, spp=6)
    s.seed = out[0][3]
    full, _ = O.render_pixels(s, M.star_catalog(0x57A25, 20000), M.xyz_weights(s.n_bins), 0, 24 * 16, nthreads=2)
    got = np.array(out[0][4]).reshape(-1, 3)
    assert np.abs(full).sum() > 0
    np.testing.assert_allclose(got, full, rtol=1e-6, atol=1e-6 * np.abs(full).max())


def test_sample_slice_bounds():
    from magik_b200 import dist as D
    assert [D.sample_slice(16, r, 8) for r in range(8)] == [(2 * r, 2) for r in range(8)]
    assert [D.sample_slice(5, r, 2) for r in range(2)] == [(0, 3), (3, 2)]
    with pytest.raises(ValueError):
        D.sample_slice(2, 0, 4)
