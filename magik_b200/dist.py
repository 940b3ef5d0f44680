"""Multi-GPU plumbing of the render: one process per GPU, no data-path
collective.  Rays are independent and frames need no exchange, so each rank
renders whole frames of its own (its own jitter seed, i.e. a different set of
samples of the same image); the only collective is the max over ranks of the
measured times, over torch.distributed (NCCL on GPUs, gloo on CPU)."""


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
