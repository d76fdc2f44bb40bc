"""Multi-GPU replicas: independent commits / proofs sharded across ranks with
no data-path collective (one proof is a sequential Fiat-Shamir chain that fits
one GPU).  The only collectives are for reporting: the max of per-rank times
and the sum of per-rank work, over torch.distributed (NCCL on GPUs, gloo on
CPU)."""
import torch
import torch.distributed as dist


def shard(items, rank: int, world: int):
    """Round-robin share of `items` for `rank` (every item on exactly one rank)."""
    if not 0 <= rank < world:
        raise ValueError("rank out of range")
    return list(items)[rank::world]


def _reduce(value: float, op, device=None) -> float:
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(value: float, device=None) -> float:
    """Job time = the slowest rank's time."""
    return _reduce(value, dist.ReduceOp.MAX, device)


def sum_over_ranks(value: float, device=None) -> float:
    return _reduce(value, dist.ReduceOp.SUM, device)


def job_throughput(units_this_rank: float, seconds_this_rank: float, device=None) -> float:
    """Whole-job units per second: all ranks' units over the slowest rank's time."""
    total = sum_over_ranks(units_this_rank, device)
    slowest = max_over_ranks(seconds_this_rank, device)
    return total / slowest if slowest > 0 else 0.0
