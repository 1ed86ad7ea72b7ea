"""Multi-GPU replicas for DM-trial searches.

DM trials are independent spectra, so the search shards by spectrum with no
data-path collective: each rank (one process per GPU) searches the trials
assigned to it, and only the timing reduction and the gathering of candidate
lists to rank 0 cross process boundaries (torch.distributed; NCCL on GPUs,
gloo on CPU)."""


def shard(n_items, rank, world):
    """Indices of the items a rank searches (round robin over ranks)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    return list(range(rank, n_items, world))


def max_over_ranks(value, dist=None, device="cpu"):
    """Largest value over all ranks (the step time of a weak-scaling run)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_to_rank0(obj, dist=None):
    """List of every rank's object on rank 0 (None elsewhere)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return [obj]
    out = [None] * dist.get_world_size() if dist.get_rank() == 0 else None
    dist.gather_object(obj, out, dst=0)
    return out


def merge_candidates(per_rank, trial_ids):
    """Candidate lists of all trials in trial order from per-rank results
    (per_rank[r] is a list of (trial_id, candidates))."""
    byid = {}
    for res in per_rank:
        for tid, cands in res:
            byid[tid] = cands
    return [byid[t] for t in trial_ids]
