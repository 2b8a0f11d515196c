"""Many independent drapes over several GPUs: one process per GPU, each solving its share of the drapes with
drape_solve_batch. The drapes share nothing, so the data path has no collective; the ranks combine only their
results at the end (the slowest rank's time, summed counters, every drape's time for the percentiles).

The share is balanced by work: drapes are taken largest first (rows, then index) and each goes to the rank with
the fewest rows so far (ties to the lower rank), the longest-processing-time rule on rows."""
import numpy as np


def partition(rows, ranks):
    """Index lists, one per rank (each in increasing order), of drapes with `rows` block rows each."""
    if ranks < 1:
        raise ValueError("ranks must be at least 1")
    load = [0] * ranks
    shares = [[] for _ in range(ranks)]
    for i in sorted(range(len(rows)), key=lambda k: (-rows[k], k)):
        r = min(range(ranks), key=lambda q: (load[q], q))
        shares[r].append(i)
        load[r] += rows[i]
    return [sorted(s) for s in shares]


def combine(total_s, counters, seconds, indices, count, dist=None, device=None):
    """Whole-job results from each rank's batch time, counters (name -> number, summed over ranks) and per-drape
    seconds of its `indices`. Returns (max total_s over ranks, summed counters, seconds of all `count` drapes in
    drape order). With `dist` (torch.distributed, initialised) the ranks reduce; without it this rank's values are
    the job's."""
    everything = np.zeros(count)
    everything[np.asarray(indices, int)] = seconds
    names = sorted(counters)
    if dist is None:
        return float(total_s), {k: counters[k] for k in names}, everything
    import torch

    t = torch.tensor([float(total_s)], dtype=torch.float64, device=device)
    c = torch.tensor([float(counters[k]) for k in names], dtype=torch.float64, device=device)
    s = torch.tensor(everything, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(c, op=dist.ReduceOp.SUM)
    dist.all_reduce(s, op=dist.ReduceOp.SUM)  # each drape's slot is non-zero on its own rank only
    return float(t.item()), dict(zip(names, c.cpu().tolist())), s.cpu().numpy()
