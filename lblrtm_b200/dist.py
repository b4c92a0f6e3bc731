"""Multi-GPU plumbing: one process per GPU; profiles are independent, so a
batch is sharded by profile with no data-path collective.  torch.distributed
carries only barriers, the max-over-ranks of timings and (optionally) the
gathering of small per-profile summaries."""


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


def sharded_run(costs, work, rank=0, world=1, device=None, gather=False):
    """Run `work(indices)` on this rank's shard of the profiles.

    `work` returns (elapsed_ms, summary) for its shard, timed on the device
    by the caller's own clock.  Returns (indices, max elapsed over ranks,
    summaries) where summaries is the list of every rank's summary when
    `gather` is set (rank order), else [this rank's].  Every rank takes the
    same collective steps (one max reduction, optionally one gather), so a
    rank with an empty shard still joins them."""
    import torch.distributed as dist
    mine = shard(costs, rank, world)
    ms, summary = work(mine)
    ms = max_over_ranks(ms, device)
    out = [summary]
    if gather and dist.is_available() and dist.is_initialized():
        out = [None] * world
        dist.all_gather_object(out, summary)
    return mine, ms, out
