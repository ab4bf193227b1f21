"""Multi-GPU plumbing: one process per GPU, disorder samples sharded across ranks.

The twist-mesh pipeline exchanges nothing between samples (every sample's mesh is solved
independently, rlm/main_rlm_cpu.cpp:109), so N GPUs run N independent replicas on disjoint
sample ranges; torch.distributed carries only the gathering of the per-sample results and
the max-over-ranks timing.  Works with the "nccl" backend on GPUs and "gloo" on CPUs.
"""
import numpy as np


def shard(n_samples, world_size, rank):
    """Contiguous, balanced block of sample indices of `rank`: (first, count)."""
    if world_size <= 0 or not 0 <= rank < world_size or n_samples < 0:
        raise ValueError("invalid shard request")
    base, extra = divmod(n_samples, world_size)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def gather_samples(local, n_samples, dist, device="cpu"):
    """All-gather per-sample rows from every rank's shard into the full [n_samples, ...]
    array (sample order), returned on every rank.  `local` is [count, ...] float64."""
    import torch
    world, rank = dist.get_world_size(), dist.get_rank()
    first, count = shard(n_samples, world, rank)
    local = np.ascontiguousarray(local, dtype=np.float64)
    assert local.shape[0] == count
    width = int(np.prod(local.shape[1:])) if local.ndim > 1 else 1
    maxc = shard(n_samples, world, 0)[1]
    buf = torch.zeros((maxc, width), dtype=torch.float64, device=device)
    buf[:count] = torch.from_numpy(local.reshape(count, width)).to(device)
    parts = [torch.zeros_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf)
    out = np.empty((n_samples, width))
    for r in range(world):
        f, c = shard(n_samples, world, r)
        out[f:f + c] = parts[r][:c].cpu().numpy()
    return out.reshape((n_samples,) + local.shape[1:])


def max_over_ranks(value, dist, device="cpu"):
    """The largest of the ranks' values (step times are reported as the max over ranks)."""
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
