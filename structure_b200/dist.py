"""Multi-GPU plumbing for independent chains (replicas, weak scaling).

The sweep has no cross-GPU exchange: each rank advances its own batch of
chains; the only collectives are the timing barrier and the max-over-ranks
reduction of the measured device time.  Works with the "nccl" backend on GPUs
and "gloo" on CPU.
"""
import os


def rank_env():
    """(rank, world_size, local_rank) from the torch.distributed launcher."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def chain_seeds(rank, nchains, base=2000):
    """Chain seeds of one rank: disjoint across ranks for up to 1000 chains each."""
    if nchains > 1000:
        raise ValueError("at most 1000 chains per rank")
    return [base + 1000 * rank + r for r in range(nchains)]


def max_over_ranks(value, device=None):
    """Max of a float over all ranks (identity when not distributed)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value, device=None):
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
