"""Multi-GPU plumbing: one process per GPU; profiles are independent, so a
batch is sharded by profile with no data-path collective.  torch.distributed
carries only barriers and the max-over-ranks of timings."""


def shard(costs, rank, world):
    """Indices of the profiles rank `rank` computes: greedy longest-first
    assignment of per-profile costs (e.g. layer points) to `world` ranks,
    deterministic on every rank."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    owner = [0] * len(costs)
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        owner[i] = r
        load[r] += costs[i]
    return [i for i in range(len(costs)) if owner[i] == rank]


def max_over_ranks(value, device=None):
    """Max of a float over all ranks (identity when not distributed)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
