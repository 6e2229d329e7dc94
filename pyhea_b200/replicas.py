"""Replica bookkeeping for multi-GPU runs of the swap search.

Solutions and structures are independent (the reference splits solutions
over MPI ranks, pyhea/cpp/accelerate.cpp:728, and gathers them on rank 0,
pyhea/model/opt.py:73-80), so N GPUs run N independent replicas: each rank
searches with its own seeds, and only the timing and counters are combined --
there is no collective on the data path.  A batch of structures can instead
be split across ranks (shard): each rank searches its share with the seeds
the structures have in the whole batch.
"""
import torch


def replica_seed(rank, index, stride=1_000_003):
    """Seed of the index-th search of a rank; disjoint across ranks."""
    return stride * int(rank) + int(index)


def shard(work, rank, world):
    """Indices of the items rank `rank` of `world` searches: items taken in
    descending work (ties by index) and each given to the rank with the least
    work so far (lowest rank on ties).  Deterministic, the same on every rank;
    every item goes to exactly one rank."""
    load = [0.0] * int(world)
    mine = []
    for i in sorted(range(len(work)), key=lambda i: (-float(work[i]), i)):
        r = min(range(int(world)), key=lambda r: (load[r], r))
        load[r] += float(work[i])
        if r == int(rank):
            mine.append(i)
    return sorted(mine)


def combine(local_ms, local_evals, group=None, device=None):
    """Whole-job figures of a replica run: (slowest rank's time in ms, total
    evaluations).  local_* are this rank's numbers; with torch.distributed
    uninitialised the local numbers are returned."""
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized():
        return float(local_ms), float(local_evals)
    t = torch.tensor([float(local_ms)], dtype=torch.float64, device=device)
    e = torch.tensor([float(local_evals)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    dist.all_reduce(e, op=dist.ReduceOp.SUM, group=group)
    return t.item(), e.item()


def gather_best(fitness, occupancy, group=None):
    """Rank-0 merge of replica results, as opt.py:73-80 merges MPI ranks:
    every rank's (fitness list, occupancy list) gathered and sorted ascending
    (stable, lower rank first on ties).  Returns (fitness, occupancy) on every
    rank."""
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized():
        pairs = list(zip(list(fitness), list(occupancy)))
    else:
        out = [None] * dist.get_world_size(group)
        dist.all_gather_object(out, (list(fitness), [list(map(int, o)) for o in occupancy]), group=group)
        pairs = [(f, o) for fs, os in out for f, o in zip(fs, os)]
    pairs.sort(key=lambda p: p[0])
    return [p[0] for p in pairs], [p[1] for p in pairs]
