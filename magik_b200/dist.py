"""Multi-GPU plumbing of the render: one process per GPU over
torch.distributed (NCCL on GPUs, gloo on CPU).  Rays are independent, so a
frame splits into sample slices, and the one exchange step is a sum-reduce of
the XYZ films into rank 0.  Two splits:

* strong (sample_slice / reduce_slices): the ranks share one frame.  Rank r
  renders a contiguous slice of its spp samples per pixel (mgk_scene's
  sample_offset and spp), all pixels, the same seed; each film, weighted by
  its share of the samples, sums into the film of the whole frame.  N ranks
  render the same frame N times faster.
* weak (frame_seed / reduce_film): every rank renders all pixels and all spp
  samples with its own jitter seed, and the mean of the films is the image at
  N x spp samples per pixel.

Timings are combined with a max over ranks."""


def sample_slice(spp, rank, world):
    """(sample_offset, count): the samples of a frame of `spp` samples per
    pixel that `rank` of `world` renders in the strong split, contiguous and
    as even as the division allows (every rank needs at least one)."""
    spp, rank, world = int(spp), int(rank), int(world)
    if world < 1 or not 0 <= rank < world or spp < world:
        raise ValueError(f"{spp} samples per pixel do not split over {world} ranks")
    base, extra = divmod(spp, world)
    return rank * base + min(rank, extra), base + (1 if rank < extra else 0)


def reduce_slices(film, count, spp, dst=0):
    """The film of the whole frame into rank `dst`, in place: each rank's
    film (the mean over its `count` of the frame's `spp` samples) weighted by
    count / spp, then sum-reduced (NCCL over NVLink on GPUs).  The other
    ranks' films are scratch afterwards.  Identity with one rank."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return film
    film.mul_(float(count) / float(spp))
    dist.reduce(film, dst=dst, op=dist.ReduceOp.SUM)
    return film


def frame_seed(base_seed, rank):
    """Seed of the frames a rank renders: distinct per rank, so N ranks
    together render N x spp samples per pixel of the same image."""
    return (int(base_seed) + 0x9E3779B97F4A7C15 * int(rank)) & 0xFFFFFFFFFFFFFFFF


def max_over_ranks(values, device="cpu"):
    """Element-wise max of a list of floats over all ranks (identity when
    torch.distributed is not initialised)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def sum_over_ranks(values, device="cpu"):
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return t.tolist()


def reduce_film(film, dst=0):
    """Mean of the ranks' films into rank `dst`, in place: a sum-reduce
    (NCCL reduce over NVLink on GPUs) then a division by the world size.
    Each rank rendered a sample slice of the same image with its own seed,
    so the result is the image at world x spp samples per pixel.  The other
    ranks' films are scratch afterwards (gloo reduces through them).
    Identity when torch.distributed is not initialised or has one rank."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return film
    world = dist.get_world_size()
    dist.reduce(film, dst=dst, op=dist.ReduceOp.SUM)
    if dist.get_rank() == dst:
        film.mul_(1.0 / world)
    return film


def train_data_parallel(net, cfg, d_feat, d_lab, stream=None):
    """Data-parallel Adam training of the deflection surrogate, one process
    per GPU.  Every rank holds its own shard of the sample set (d_feat [n, 7],
    d_lab [n], the same n on every rank) and takes cfg.batch / world rows of
    it per step; the ranks' batch gradients are summed by an all-reduce (NCCL
    over NVLink on GPUs) and the Adam step scales the sum by 1 / world, so each
    step is a step on the union batch of cfg.batch rows and every rank keeps
    the same parameters.  A rank shuffles its shard with frame_seed(cfg.seed,
    rank): with one rank this is the loop of Surrogate.train
    (mgk_surrogate_train).  Returns the mean batch loss of each epoch over all
    ranks (numpy float32).

    `net` is a Surrogate, or any object with its shuffle / gradient_step /
    adam_step methods, a `param_count` and optionally a `grad_dtype` (float32
    by default); d_feat and d_lab are tensors on the net's device."""
    import numpy as np
    import torch
    import torch.distributed as dist
    multi = dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1
    world = dist.get_world_size() if multi else 1
    rank = dist.get_rank() if multi else 0
    if cfg.batch == 0 or cfg.batch % world or (cfg.batch // world) % 1024:
        raise ValueError(f"batch {cfg.batch} is not {world} ranks x a multiple of 1024")
    b = cfg.batch // world
    n = int(d_feat.shape[0])
    nb = n // b
    if multi:  # the same number of steps on every rank, or the collectives would not pair up
        t = torch.tensor([nb, -nb], dtype=torch.int64, device=d_feat.device)
        dist.all_reduce(t, op=dist.ReduceOp.MIN)
        if int(t[0]) != nb or -int(t[1]) != nb:
            raise ValueError("the ranks' shards give different numbers of steps per epoch")
    if nb == 0:
        raise ValueError(f"{n} samples are fewer than one batch of {b} rows")
    grad = torch.empty(int(net.param_count), dtype=getattr(net, "grad_dtype", torch.float32), device=d_feat.device)
    loss = torch.zeros(max(int(cfg.epochs), 1), dtype=grad.dtype, device=d_feat.device)
    seed = frame_seed(cfg.seed, rank)
    for ep in range(int(cfg.epochs)):
        net.shuffle(seed, ep, n, stream=stream)
        for k in range(nb):
            net.gradient_step(cfg, d_feat, d_lab, k * b, b, grad, loss[ep:ep + 1], stream=stream)
            if multi:
                dist.all_reduce(grad, op=dist.ReduceOp.SUM)
            net.adam_step(cfg, grad, 1.0 / world, (ep * nb + k) / (int(cfg.epochs) * nb), stream=stream)
    if multi:
        dist.all_reduce(loss, op=dist.ReduceOp.SUM)
    return (loss[: int(cfg.epochs)] / float(nb * world)).cpu().numpy().astype(np.float32)
