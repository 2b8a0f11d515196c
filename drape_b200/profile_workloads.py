"""Small, self-contained GPU workloads for profiling one part of the solve (ncu captures, CUDA-event timings).

    python -m drape_b200.profile_workloads cycle   [--n 129] [--steps 20]   # multilevel V-cycle and PCG iteration
    python -m drape_b200.profile_workloads network [--n 129] [--steps 20]   # preconditioner network forward
    python -m drape_b200.profile_workloads spmv    [--drapes 128]          # batched and n257 BSR SpMV, autotuned
    python -m drape_b200.profile_workloads solve   [--n 129] [--preconditioner learned] [--out state.npy] [--budget s]
    python -m drape_b200.profile_workloads batch   [--drapes 128] [--workers 32] [--budget s]   # concurrent solves
    torchrun --nproc-per-node N -m drape_b200.profile_workloads batch ...   # the drapes split over N GPUs

batch solves the same `drapes` sheets cold (learned preconditioner unless --preconditioner says otherwise) through
drape_solve_batch, `workers` at a time, and reports solves/s and the p50/p99 of the per-drape solve times.

spmv builds the batched configuration: `drapes` sheets with n drawn from {33, 49, 65, 97, 129}, sphere radius
U(0.15, 0.35) m, E log-uniform in [1e5, 2e6] Pa (master seed 7), each assembled on the GPU at its start state
(h = 1e-2 s), concatenated block-diagonally; and the single n257 sheet's matrix. For each it times every
lanes-per-row x threads shape of the SpMV kernel, keeps the fastest, checks its y against numpy (f64 of the same
f32 blocks) and reports algorithmic GB/s (40 B per block + 28 B per row) against the measured HBM peak.

Both drive `steps` PTC steps of the n x n sheet drape (sphere + ground plane) with the multilevel preconditioner,
assemble the projected (SPD) PTC system at that state, and then:
  cycle    times stand-alone V-cycles and flexible PCG iterations on it (drape_time_multilevel) and a fine SpMV;
  network  runs the shipped network's forward (drape_network_gradient) and one preconditioner-2 PCG solve on it.
"""
import argparse
import ctypes
import json
import os
import sys

import numpy as np

from drape_b200 import api, batch_shards

GRAVITY = np.array([0.0, -9.81, 0.0])


def system(n, steps):
    d = api.Drape.sheet(n, seed=0, plane=True, options=api.default_options(max_steps=steps, preconditioner=1))
    d.solve_equilibrium(check=False)
    x, h = d.state, d.final_h()
    x_hat = x + h * h * np.tile(GRAVITY, d.V)
    d.set_options(api.default_options(tangent=1))
    g, blocks = d.assemble(x, x_hat=x_hat, h=h, mode=0, curvature=False)
    return d, blocks, -g


def sheet_matrix(n, seed, radius, young):
    """(row_ptr, col_idx, 9B f32 blocks) of the sheet drape's PTC system at its start state (h = 1e-2 s)."""
    import tempfile
    d = api.Drape.sheet(n, seed=seed, radius=radius, young=young, plane=True)
    x = d.state
    h = 1e-2
    _, blocks = d.assemble(x, x_hat=x + h * h * np.tile(GRAVITY, d.V), h=h, mode=0)
    with tempfile.TemporaryDirectory() as t:
        api.write_sheet_problem(t, n, seed=seed, radius=radius, young=young, plane=True)
        _, arr = api.read_problem_arrays(t)
    d.close()
    return arr["row_ptr"].astype(np.int64), arr["col_idx"].astype(np.int64), blocks


def batch_scenes(drapes):
    """(columns, seed, sphere radius, E) of the batched configuration's drapes, master seed 7."""
    rng = np.random.default_rng(7)
    out = []
    for _ in range(drapes):
        n = int(rng.choice([33, 49, 65, 97, 129]))
        out.append((n, int(rng.integers(1, 1 << 30)), float(rng.uniform(0.15, 0.35)),
                    float(np.exp(rng.uniform(np.log(1e5), np.log(2e6))))))
    return out


def batch_workload(drapes, workers, budget, preconditioner):
    """Every drape of the batched configuration solved cold to |grad E_s| <= 1e-6 N, `workers` at a time. Under
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
                            options=api.default_options(preconditioner=preconditioner, time_budget_s=budget))
        if net is not None:
            d.set_network(net)
        ds.append(d)
    logs, seconds, total = api.solve_batch(ds, workers, check=False) if ds else ([], np.zeros(0), 0.0)
    local_counts = {"solved": sum(g["status"] == 0 for g in logs), "newton": sum(g["newton_iterations"] for g in logs),
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
            "preconditioner": preconditioner, "budget_s": budget, "solved": solved, "total_s": total,
            "solves_per_s": solved / total if total > 0 else 0.0,
            "p50_s": float(np.percentile(seconds_all, 50)), "p99_s": float(np.percentile(seconds_all, 99)),
            "max_s": float(seconds_all.max()), "sum_device_s": counts["sum_device_s"],
            "newton": int(round(counts["newton"])), "pcg": int(round(counts["pcg"])),
            "fallbacks": int(round(counts["fallbacks"])),
            "reasons": {k[len("reason_"):]: int(round(v)) for k, v in counts.items() if k.startswith("reason_") and v},
            "per_columns": per_n}


def spmv_workload(drapes):
    import json as _json
    import os
    parts, offset = [], 0
    sizes = []
    for n, seed, radius, young in batch_scenes(drapes):
        rp, ci, blk = sheet_matrix(n, seed, radius, young)
        parts.append((rp, ci + offset, blk))
        offset += len(rp) - 1
        sizes.append(n)
    rp_all = [np.zeros(1, np.int64)]
    base = 0
    for rp, _, _ in parts:
        rp_all.append(rp[1:] + base)
        base += rp[-1]
    batch = (np.concatenate(rp_all), np.concatenate([p[1] for p in parts]), np.concatenate([p[2] for p in parts]))
    single = sheet_matrix(257, 0, 0.25, 5e5)
    try:
        peak = _json.load(open(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                            "MEASURED_PEAKS.json")))["hbm_gbs"]
    except Exception:
        peak = 6650.0
    out = {}
    for name, (rp, ci, blk) in (("batched", batch), ("n257", single)):
        R, B = len(rp) - 1, len(ci)
        x = np.random.default_rng(1).standard_normal(3 * R).astype(np.float32)
        shapes = {}
        for lanes in (4, 8, 16, 32):
            for threads in (128, 256):
                shapes[f"{lanes}x{threads}"] = api.spmv_benchmark(rp, ci, blk, x, 20, lanes, threads)
        best = min(shapes, key=shapes.get)
        lanes, threads = (int(v) for v in best.split("x"))
        ms, y = api.spmv_benchmark(rp, ci, blk, x, 20, lanes, threads, result=True)
        Bm = blk.reshape(-1, 3, 3).astype(np.float64)
        rows = np.repeat(np.arange(R), np.diff(rp))
        ref = np.zeros((R, 3))
        np.add.at(ref, rows, np.einsum("kab,kb->ka", Bm, x.reshape(-1, 3).astype(np.float64)[ci]))
        err = float(np.linalg.norm(y - ref.reshape(-1)) / np.linalg.norm(ref))
        bytes_ = 40 * B + 28 * R
        out[name] = {"rows": R, "blocks": B, "algorithmic_MB": bytes_ / 1e6, "best_shape": best, "ms": ms,
                     "GB_per_s": bytes_ / (ms * 1e-3) / 1e9, "fraction_of_peak": bytes_ / (ms * 1e-3) / 1e9 / peak,
                     "peak_GB_per_s": peak, "relative_error_vs_numpy": err, "all_shapes_ms": shapes}
    out["batched"]["drapes"] = drapes
    out["batched"]["columns_histogram"] = {str(n): sizes.count(n) for n in sorted(set(sizes))}
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("workload", choices=["cycle", "network", "spmv", "solve", "batch"])
    ap.add_argument("--workers", type=int, default=32, help="batch: drapes solved at a time")
    ap.add_argument("--preconditioner", default="learned", choices=["jacobi", "multilevel", "learned"])
    ap.add_argument("--out", default=None, help="solve: .npy file for the converged positions")
    ap.add_argument("--absolute", type=float, default=1e-6, help="solve: stop at |grad E_s| <= this (N)")
    ap.add_argument("--budget", type=float, default=0.0,
                    help="solve, batch: the solver's own time budget per drape, s (0: none)")
    ap.add_argument("--n", type=int, default=129)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--drapes", type=int, default=128)
    args = ap.parse_args(argv)
    if args.workload == "spmv":
        print(json.dumps(spmv_workload(args.drapes)), flush=True)
        return 0
    if args.workload == "batch":
        # more hardware queues than the default 8, for streams of many drapes (read when CUDA starts)
        os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
        pre = {"jacobi": 0, "multilevel": 1, "learned": 2}[args.preconditioner]
        out = batch_workload(args.drapes, args.workers, args.budget, pre)
        if int(os.environ.get("RANK", "0")) == 0:
            print(json.dumps(out), flush=True)
        return 0
    if args.workload == "solve":
        # the bench scene's full cold solve; the converged positions go to --out for an f64 error check
        pre = {"jacobi": 0, "multilevel": 1, "learned": 2}[args.preconditioner]
        d = api.Drape.sheet(args.n, seed=0, plane=True,
                            options=api.default_options(preconditioner=pre, equilibrium_absolute=args.absolute,
                                                        time_budget_s=args.budget))
        if pre == 2:
            d.set_network(api.Network.trained())
        log = d.solve_equilibrium(check=False)
        if args.out:
            np.save(args.out, d.state)
        keys = ("reason", "ptc_steps", "newton_iterations", "pcg_iterations", "fallbacks", "ms_pcg", "final_residual",
                "device_seconds", "static_energy")
        print(json.dumps({k: log[k] for k in keys}), flush=True)
        return 0
    d, blocks, b = system(args.n, args.steps)
    lib = api.load()
    out = {"workload": args.workload, "columns": args.n, "ptc_steps": args.steps}
    if args.workload == "cycle":
        d.set_options(api.default_options(preconditioner=1))
        _, info = d.pcg(b, 1e-6, 2000, blocks=blocks)
        out["pcg"] = info
        lib.drape_time_multilevel.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p]
        t = (ctypes.c_float * 3)()
        for its in (20, 200):
            assert lib.drape_time_multilevel(d.h, its, t) == 0, lib.drape_last_error(d.h)
            out[f"iterations_{its}"] = {"vcycle_ms": t[0], "pcg_iteration_ms": t[1], "pdl": t[2]}
        out["spmv_ms"] = d.time_spmv(200, 8, 256)
    else:
        net = api.Network.trained()
        d.set_options(api.default_options(preconditioner=1))
        sol, _ = d.pcg(b, 1e-8, 4000, blocks=blocks)
        loss, _, fac = net.gradient(d, blocks, b, sol)
        d.set_options(api.default_options(preconditioner=2))
        d.set_network(net)
        _, info = d.pcg(b, 1e-6, 2000, blocks=blocks)
        out.update({"loss": loss, "factor_min": float(fac.min()), "factor_max": float(fac.max()), "pcg": info})
    print(json.dumps(out), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
