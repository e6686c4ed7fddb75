"""Start-sharded solves over several GPUs, one process per GPU.

Starting points are independent, so the AM path shards by start: every rank
holds the data matrix, solves a contiguous share of the global start indices
on its own GPU, and one exchange at the end picks the best start of all ranks.
That exchange gathers each rank's best objective, takes the first maximum in
rank order (which is the reference's first-maximum rule over the global start
order, since shares are contiguous), and broadcasts that rank's loadings.
No collective runs on the per-iteration path.
"""
import numpy as np


def shard(total_starts, world, rank):
    """The contiguous share [first, first + count) of rank `rank` among `world`
    ranks; the first total_starts % world ranks take one start more."""
    base, extra = divmod(int(total_starts), int(world))
    count = base + (1 if rank < extra else 0)
    first = rank * base + min(rank, extra)
    return first, count


def best_of_ranks(fval, x, group=None):
    """Returns (best fval, its loadings x, the rank that held it), identical on
    every rank.  fval is this rank's best objective (NaN counts as no result),
    x its loadings (numpy, same length on every rank)."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    mine = torch.tensor([float(fval)], dtype=torch.float64)
    every = [torch.zeros(1, dtype=torch.float64) for _ in range(world)]
    dist.all_gather(every, mine, group=group)
    vals = [float(t.item()) for t in every]
    best_rank, best = 0, -np.inf
    for r, v in enumerate(vals):
        if not np.isnan(v) and v > best:  # strict: the first maximum wins
            best_rank, best = r, v
    buf = torch.from_numpy(np.ascontiguousarray(x, dtype=np.float32).copy())
    src = dist.get_global_rank(group, best_rank) if group is not None else best_rank
    dist.broadcast(buf, src=src, group=group)
    return (best if np.isfinite(best) else float("nan")), buf.numpy(), best_rank


def solve_sharded(solve_share, total_starts, start_points, group=None):
    """Runs this rank's share and the exchange.  solve_share(starts) solves the
    given n x count injected starts on this rank's GPU and returns (x, fval);
    start_points is the global n x total_starts matrix (every rank holds it, or
    at least its own columns).  Returns (x, fval, best rank, (first, count))."""
    import torch.distributed as dist
    first, count = shard(total_starts, dist.get_world_size(group), dist.get_rank(group))
    if count > 0:
        x, fval = solve_share(np.asfortranarray(start_points[:, first:first + count]))
    else:
        x, fval = np.zeros(start_points.shape[0], np.float32), float("nan")
    best, xb, r = best_of_ranks(fval, x, group)
    return xb, best, r, (first, count)
