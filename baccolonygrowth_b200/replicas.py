"""Replica (ensemble) runs over several GPUs: one colony per rank, no
collective in the step.  The only cross-rank work is the end-of-run
aggregation: job time = the slowest rank's device time, job work = the sum
of the ranks' cell-steps."""
import torch
import torch.distributed as dist


def aggregate(times_s, works, device="cpu"):
    """times_s: this rank's timings (seconds) -> max over ranks;
    works: this rank's work counters -> sum over ranks.  Every rank calls
    this with lists of the same length (same collectives, same order)."""
    t = torch.tensor(list(times_s), dtype=torch.float64, device=device)
    w = torch.tensor(list(works), dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.all_reduce(w, op=dist.ReduceOp.SUM)
    return t.tolist(), w.tolist()


def replica_seed(base, rank):
    """Seed of the colony a rank simulates (independent replicas)."""
    return base + 2 * rank
