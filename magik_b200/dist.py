"""Multi-GPU plumbing of the render: one process per GPU over
torch.distributed (NCCL on GPUs, gloo on CPU).  Rays are independent, so the
frame is split into sample slices: every rank renders all pixels with its own
jitter seed (a different set of samples of the same image) and the one
exchange step is a sum-reduce of the XYZ films into rank 0, which divides by
the number of ranks.  Timings are combined with a max over ranks."""


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
