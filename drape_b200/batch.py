"""Many drapes at once (the batched configuration): every drape of batch_scenes solved cold to the equilibrium
tolerance through drape_solve_batch, `workers` at a time, reporting solves/s and the p50/p99 per-drape times.

    python -m drape_b200.batch [--drapes 128] [--workers 32] [--budget s] [--preconditioner learned]
    torchrun --nproc-per-node N -m drape_b200.batch ...   # the drapes split over N GPUs (drape_b200.batch_shards)
"""
import argparse
import json
import os
import sys

import numpy as np

from drape_b200 import api, batch_shards
from drape_b200.scenes import batch_scenes


def batch_workload(drapes, workers, budget, preconditioner, absolute=1e-6, forcing=1):
    """Every drape of the batched configuration solved cold to |grad E_s| <= `absolute`, `workers` at a time. Under
    torchrun (WORLD_SIZE > 1, one process per GPU) each rank solves its row-balanced share on its own GPU
    (drape_b200.batch_shards) and the ranks combine only their results; rank 0 returns the job's line."""
    world, rank = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    scenes = batch_scenes(drapes)
    mine = batch_shards.partition([n * n for n, _, _, _ in scenes], world)[rank]
    dist, device = None, None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as td

        torch.cuda.set_device(local)
        td.init_process_group("nccl", timeout=datetime.timedelta(seconds=600 + 2 * budget))
        dist, device = td, f"cuda:{local}"
    net = api.Network.trained(device=local) if preconditioner == 2 else None
    ds = []
    for i in mine:
        n, seed, radius, young = scenes[i]
        d = api.Drape.sheet(n, seed=seed, radius=radius, young=young, plane=True, device=local,
                            options=api.default_options(preconditioner=preconditioner, time_budget_s=budget,
                                                        equilibrium_absolute=absolute, forcing=forcing))
        if net is not None:
            d.set_network(net)
        ds.append(d)
    logs, seconds, total = api.solve_batch(ds, workers, check=False) if ds else ([], np.zeros(0), 0.0)
    local_counts = {"solved": sum(g["reason"] == "tolerance" for g in logs),
                    "newton": sum(g["newton_iterations"] for g in logs),
                    "pcg": sum(g["pcg_iterations"] for g in logs), "fallbacks": sum(g["fallbacks"] for g in logs),
                    "sum_device_s": sum(g["device_seconds"] for g in logs)}
    for g in logs:
        key = "reason_" + g["reason"]
        local_counts[key] = local_counts.get(key, 0) + 1
    for k in ("reason_tolerance", "reason_cap", "reason_stalled", "reason_time_budget"):
        local_counts.setdefault(k, 0)
    total, counts, seconds_all = batch_shards.combine(total, local_counts, seconds, mine, drapes, dist, device)
    for d in ds:
        d.close()
    if dist is not None:
        dist.destroy_process_group()
    sizes = [s[0] for s in scenes]
    per_n = {}
    for n in sorted(set(sizes)):
        idx = [i for i in range(drapes) if sizes[i] == n]
        per_n[str(n)] = {"drapes": len(idx), "median_s": float(np.median(seconds_all[idx]))}
    solved = int(round(counts["solved"]))
    return {"workload": "batch", "drapes": drapes, "workers": workers, "n_gpus": world,
            "preconditioner": preconditioner, "budget_s": budget, "tolerance_N": absolute,
            "forcing": ["fixed rtol 1e-6", "eisenstat-walker"][forcing], "solved": solved,
            "total_s": total, "solves_per_s": solved / total if total > 0 else 0.0,
            "p50_s": float(np.percentile(seconds_all, 50)), "p99_s": float(np.percentile(seconds_all, 99)),
            "max_s": float(seconds_all.max()), "sum_device_s": counts["sum_device_s"],
            "newton": int(round(counts["newton"])), "pcg": int(round(counts["pcg"])),
            "fallbacks": int(round(counts["fallbacks"])),
            "reasons": {k[len("reason_"):]: int(round(v)) for k, v in counts.items() if k.startswith("reason_") and v},
            "per_columns": per_n}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--drapes", type=int, default=128)
    ap.add_argument("--workers", type=int, default=32, help="drapes solved at a time")
    ap.add_argument("--preconditioner", default="learned", choices=["jacobi", "multilevel", "learned"])
    ap.add_argument("--budget", type=float, default=0.0, help="the solver's own time budget per drape, s (0: none)")
    ap.add_argument("--absolute", type=float, default=1e-6, help="stop at |grad E_s| <= this (N)")
    ap.add_argument("--forcing", type=int, default=1, choices=[0, 1],
                    help="1 (default): Eisenstat-Walker forcing of the Newton directions; 0: fixed PCG rtol 1e-6")
    args = ap.parse_args(argv)
    # more hardware queues than the default 8, for streams of many drapes (read when CUDA starts)
    os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
    pre = {"jacobi": 0, "multilevel": 1, "learned": 2}[args.preconditioner]
    out = batch_workload(args.drapes, args.workers, args.budget, pre, args.absolute, args.forcing)
    if int(os.environ.get("RANK", "0")) == 0:
        print(json.dumps(out), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
