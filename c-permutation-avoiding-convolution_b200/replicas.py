"""Multi-GPU plumbing: replicas, one process per GPU.

The convolutions of a batch are independent, so a batch shards across ranks
with no collective on the data path: every rank convolves its own slice of
problems on its own GPU.  The only collectives are host-side plumbing of the
benchmark (a barrier and the max over ranks of the timed region), over
torch.distributed (NCCL on GPUs, gloo on CPU).
"""


def shard(batch, world, rank):
    """Contiguous slice of `batch` problems owned by `rank` (sizes differ by
    at most one when world does not divide batch)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    base, extra = divmod(batch, world)
    start = rank * base + min(rank, extra)
    return slice(start, start + base + (1 if rank < extra else 0))


def max_over_ranks(value, dist=None, device=None):
    """The largest `value` over all ranks (the timed region of the slowest
    rank); `value` itself with no process group."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
