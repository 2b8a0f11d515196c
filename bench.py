"""Benchmark of the quasi-static drape GPU stage (one JSON line on rank 0).

Workload: the 1.0 m sheet of n x n vertices (default n = 129: 16641 vertices, 32768 triangles, 48896 hinges,
180993 BSR blocks) over a sphere of radius 0.25 m and a ground plane at y = -0.25 m, isotropic StVK E = 5e5 Pa,
nu = 0.3, t = 5e-4 m, k_b = 1e-5 N m, IPC d_hat = 2e-3 m, kappa = 1e3; PTC from dt0 = 1e-3 s to
|grad E_s| <= 1e-6 N, PCG rtol 1e-6, <= 2000 iterations. One step = one full cold solve to the converged state.
Direction solver (--preconditioner): learned (default: the multilevel V-cycle flexible PCG with the shipped
network's fine smoother), multilevel (spectral Jacobi smoothing), jacobi (the reference's block-Jacobi PCG).
--compare jacobi (default) adds one device-timed block-Jacobi solve of the same workload after the timed steps, the
learned-vs-Jacobi comparison of the metric (all: also multilevel and learned; none: skip). Synthetic scene (the
reference ships no dataset; seeded jitter, seed 0).

value: seconds per converged solve with the problem resident in HBM (CUDA-event-timed solve, max over ranks).
e2e:   the same through the C ABI from host arrays: drape_create (host->device copies) + solve + drape_get_state
       (device->host), wall clock on the host.
--impl reference: the reference's CPU implementation of this path (the f64 oracle restatement; the Rust crate
       cannot be built here), single-threaded like the reference, on a bounded sample of the same solve: its
       seconds per Newton iteration times the Newton iterations of the whole solve (FULL_SOLVE_NEWTON);
       --full-solve times the oracle's whole solve instead.
Multi-GPU: replicas only (one independent drape per rank, no collective on the data path).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "n129 drape wall-time to converged state"


def peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "_fallback": True}


class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.path = tempfile.mktemp(suffix=".csv")
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.proc or not os.path.exists(self.path):
            return None
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [v.strip() for v in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.remove(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons), "samples": len(sm)}


def flush_l2(torch, device):
    """Writes 512 MiB (> the 126 MB L2) so every timed solve starts cold."""
    buf = torch.empty(128 * 1024 * 1024, dtype=torch.float32, device=device)
    buf.fill_(1.0)
    torch.cuda.synchronize(device)
    del buf


def multilevel_bytes_per_iteration(n, R, B):
    """Algorithmic bytes of one multilevel flexible PCG iteration: the fine matrix read three times (pre-smoothing
    residual in the restriction, post-smoothing residual, the direction SpMV: 40 B per block + 28 B per row each),
    each coarse level's 5 x 5 stencil of 48-byte blocks read twice (restriction, prolongation), and the level-0
    vectors of the direction and update steps (x, r, p, q, z: 100 B per row)."""
    total = 3 * (40 * B + 28 * R) + 100 * R
    while n > 5 and (n - 1) % 2 == 0:
        n = (n - 1) // 2 + 1
        total += 2 * (25 * 48 + 48) * n * n
    return total


PRECOND = {"jacobi": "block-Jacobi PCG", "multilevel": "multilevel V-cycle flexible PCG (omega-Jacobi smoothing)",
           "learned": "multilevel V-cycle flexible PCG with the network-predicted fine smoother"}


def run_gpu(args):
    import numpy as np
    import torch

    from drape_b200 import api

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    def options_for(name):
        return api.default_options(pcg_max_iterations=args.pcg_max, max_steps=args.max_steps,
                                   preconditioner={"jacobi": 0, "multilevel": 1, "learned": 2}[name])

    net = api.Network.trained(device=local) if args.preconditioner == "learned" or args.compare == "all" else None
    # Host arrays for the end-to-end leg (built outside every timed region).
    pdir = tempfile.mkdtemp(prefix="drape_bench_")
    api.write_sheet_problem(pdir, args.n, seed=args.seed, plane=bool(args.plane))
    meta, arr = api.read_problem_arrays(pdir)
    host = dict(start=arr["rest_positions_f64"], row_vertex=arr["row_vertex"], unit_mass=arr["row_unit_mass_f64"],
                row_ptr=arr["row_ptr"], col_idx=arr["col_idx"], tri=arr["elem_vertices"], geom=arr["elem_geom_f64"],
                hinge=arr["hinge_vertices"], hinge_k=arr["hinge_stiffness_f64"],
                material=(meta["material"]["wale_N_per_m"], meta["material"]["course_N_per_m"],
                          meta["material"]["coupling_N_per_m"], meta["material"]["shear_N_per_m"]),
                gravity=tuple(meta["gravity_vector"]), colliders=arr["colliders"][4:].astype(np.float64),
                dhat=meta["contact"]["dhat_m"], kappa=meta["contact"]["kappa"], columns=args.n)
    h2d = sum(v.nbytes for v in host.values() if hasattr(v, "nbytes"))
    d2h = 3 * int(meta["vertices"]) * 8

    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()

    def one_step(name=args.preconditioner):
        """One step through the public C ABI from host buffers: drape_create (host->device copies of the problem),
        the solve (timed on the device with CUDA events on the library's stream, bracketed by a synchronize), and
        drape_get_state (device->host copy of the converged positions)."""
        flush_l2(torch, local)
        barrier()
        t0 = time.perf_counter()
        drape = api.Drape.from_arrays(**host, options=options_for(name), device=local)
        if name == "learned":
            drape.set_network(net)
        torch.cuda.synchronize()
        log = drape.solve_equilibrium(check=False)
        state = drape.state
        t1 = time.perf_counter()
        barrier()
        drape.close()
        # The solve's time: CUDA events recorded by the library on its stream at the start and end of the solve
        # (with a synchronize before the end event is read); the host decisions between launches are inside.
        return log, log["device_seconds"], t1 - t0, state

    for _ in range(args.warmup):
        one_step()
    logs, secs, e2e = [], [], []
    with ClockSampler(local) as clock:
        for _ in range(args.steps):
            log, s, w, state = one_step()
            logs.append(log)
            secs.append(s)
            e2e.append(w)
    clocks = clock.summary()
    t = sum(secs) / len(secs)
    t_e2e = sum(e2e) / len(e2e)
    if dist:
        v = torch.tensor([t, t_e2e], device=f"cuda:{local}")
        dist.all_reduce(v, op=dist.ReduceOp.MAX)
        t, t_e2e = v.tolist()
    last = logs[-1]
    R, B = int(meta["rows"]), int(meta["blocks"])
    pk = peaks()
    traffic = None
    if args.preconditioner == "jacobi":
        kernel = "pcg_kernel (persistent block-Jacobi PCG)"
        bytes_per_iter = 40 * B + 196 * R
        tpath = os.path.join(ROOT, "profiles", "pcg_traffic.json")
        if os.path.exists(tpath):
            tr = json.load(open(tpath))
            if tr.get("columns") == args.n:
                # One launch stages the matrix into shared memory once: its DRAM traffic is per launch, not per
                # iteration (ncu capture summarised in profiles/pcg_kernel_n129.md).
                traffic = tr["dram_bytes_per_launch"]
    else:
        kernel = "multilevel flexible PCG iteration (restrict/tail/prolong/direction/update kernels, one graph)"
        bytes_per_iter = multilevel_bytes_per_iteration(args.n, R, B)
    achieved = (bytes_per_iter * last["pcg_iterations"]) / (last["ms_pcg"] / 1e3) / 1e9 if last["ms_pcg"] > 0 else 0.0
    comparison = {}
    others = {"none": (), "jacobi": ("jacobi",), "all": ("jacobi", "multilevel", "learned")}[args.compare]
    if others:  # every rank runs the same comparison solves (replicas; one_step holds the barriers), rank 0 reports
        for other in others:
            if other == args.preconditioner:
                continue
            log_o, s_o, _, _ = one_step(other)
            comparison[other] = {"seconds": s_o, "ptc_steps": log_o["ptc_steps"],
                                 "newton_iterations": log_o["newton_iterations"],
                                 "pcg_iterations": log_o["pcg_iterations"],
                                 "pcg_per_newton": log_o["pcg_iterations"] / max(1, log_o["newton_iterations"]),
                                 "fallbacks_to_jacobi": log_o["fallbacks"], "converged": log_o["reason"] == "tolerance",
                                 "final_residual_N": log_o["final_residual"]}
        if "jacobi" in comparison:
            comparison["jacobi_seconds_over_this"] = comparison["jacobi"]["seconds"] / t
    out = {
        "metric": METRIC, "value": t, "unit": "s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t * 1e3, "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": f"sheet n{args.n} over sphere r=0.25 + ground plane y=-0.25, {PRECOND[args.preconditioner]}, "
                               f"PTC dt0=1e-3 s to |grad E_s|<=1e-6 N", "columns": args.n, "rows": R, "blocks": B,
                   "seed": args.seed, "preconditioner": args.preconditioner, "parallelism": f"replicas{world}",
                   "l2": "flushed (512 MiB write) before every timed solve"},
        "solve": {"converged": last["reason"] == "tolerance", "reason": last["reason"],
                  "final_residual_N": last["final_residual"], "ptc_steps": last["ptc_steps"],
                  "newton_iterations": last["newton_iterations"], "pcg_iterations": last["pcg_iterations"],
                  "pcg_per_newton": last["pcg_iterations"] / max(1, last["newton_iterations"]),
                  "rejected_attempts": last["rejected_attempts"], "static_energy_J": last["static_energy"],
                  "fallbacks_to_jacobi": last["fallbacks"], "mg_levels": last["mg_levels"],
                  "phase_ms": {k: last[k] for k in ("ms_assembly", "ms_pcg", "ms_line_search", "ms_ccd", "ms_other")}},
        "e2e": {"value": t_e2e, "unit": "s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": int(sum(l["kernel_launches"] for l in logs)),
        "roofline": {"bound": "hbm", "kernel": kernel, "achieved": achieved,
                     "peak": pk["hbm_gbs"], "unit": "GB/s", "frac": achieved / pk["hbm_gbs"],
                     "traffic": traffic, "peak_source": "fallback" if pk.get("_fallback") else "measured",
                     "algorithmic_bytes_per_pcg_iteration": bytes_per_iter,
                     "algorithmic_bytes_per_launch": bytes_per_iter * last["pcg_iterations"] / max(1, last["pcg_launches"]),
                     "avg_launch_ms": last["ms_pcg"] / max(1, last["pcg_launches"])},
        "clocks": clocks,
    }
    if comparison:
        comparison["this_run"] = args.preconditioner
        out["comparison"] = comparison
    if rank == 0 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(args, last)
    if dist:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)


# Newton iterations of the whole cold solve of a bench workload, keyed by (n, plane, seed), and where the count
# comes from: the f64 oracle's own whole solve (`python bench.py --impl reference --full-solve`, no CPU budget) where
# it has been run, else the block-Jacobi GPU solve of the same workload (the reference's method, f32 PCG; 424 PTC
# steps at n129).
FULL_SOLVE_NEWTON = {(129, 1, 0): (3162, "the block-Jacobi GPU solve of this workload")}


def full_newton_count(args, gpu_log=None):
    """(Newton iterations of the whole solve, where the count comes from), or (None, ...) when neither the table
    nor this run's GPU solve gives one."""
    known = FULL_SOLVE_NEWTON.get((args.n, int(args.plane), args.seed))
    if known is not None:
        return known
    if gpu_log:
        return int(gpu_log["newton_iterations"]), "this run's GPU solve"
    return None, "none"


def cpu_baseline(args, gpu_log=None, budget_s=None):
    """The f64 oracle (port of the reference crate's method: exact tangent, LM, f64 block-Jacobi PCG rtol 1e-6
    <= 2000 iterations, inner-count PTC from dt0 = 1e-3 s) timed on the host. It runs the cold solve until `budget_s`
    of CPU time has passed (0: to the end) and reports the whole solve's time as its seconds per Newton iteration
    times the Newton iterations of the whole solve: the counted whole solve of this workload, else this run's
    GPU solve. With neither, the solve runs to the end and its own time is the value."""
    from tests import oracle_py

    budget = budget_s if budget_s is not None else args.cpu_budget
    full_newton, source = full_newton_count(args, gpu_log)
    if full_newton is None:
        budget = 0.0
    s = oracle_py.Scene("sheet", args.n, seed=args.seed, plane=bool(args.plane))
    # The cold solve, stopped at the first PTC step that ends past the CPU budget.
    _, st = s.ptc(h0=1e-3, doubling=False, absolute=1e-6, pcg=True, rtol=1e-6, maxit=2000, budget_s=budget)
    steps, elapsed, newton = int(st["steps"]), st["seconds"], int(st["newton"])
    if budget == 0.0:
        return {"value": elapsed, "unit": "s", "cores": 1, "kind": "port", "newton_iterations": newton,
                "converged": bool(st["converged"]),
                "sample": f"the whole n{args.n} solve ({steps} PTC steps, {newton} Newton iterations) on 1 host core",
                "host_cpu": _cpu_model()}
    per_newton = elapsed / max(1, newton)
    return {"value": per_newton * full_newton, "unit": "s", "cores": 1, "kind": "port",
            "sample": f"{steps} PTC steps ({newton} Newton iterations) of the n{args.n} solve in {elapsed:.1f} s on 1 "
                      f"host core; value = {per_newton:.3f} s per Newton iteration x {full_newton} Newton iterations "
                      f"of the whole solve ({source})",
            "host_cpu": _cpu_model()}


def _cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except Exception:
        pass
    return "unknown"


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from tests import oracle_py

    oracle_py.build()
    results = []
    budget = 0.0 if args.full_solve else args.cpu_budget
    for i in range(args.warmup if args.full_solve else 0, args.warmup + args.steps):  # a full solve needs no warm-up
        r = cpu_baseline(args, None, budget_s=budget)
        if i >= args.warmup:
            results.append(r)
    v = sum(r["value"] for r in results) / len(results)
    out = {"metric": METRIC, "value": v, "unit": "s", "n_gpus": int(os.environ.get("WORLD_SIZE", "1")),
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": v * 1e3, "higher_is_better": False,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
           "config": {"workload": f"sheet n{args.n} over sphere r=0.25 + ground plane y=-0.25, f64 oracle port "
                                  f"(exact tangent, LM, block-Jacobi PCG rtol 1e-6 <= 2000)", "columns": args.n},
           "cpu_baseline": {"value": v, "unit": "s", "cores": 1, "kind": "port", "sample": results[-1]["sample"]},
           "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if "newton_iterations" in results[-1]:
        out["newton_iterations"] = results[-1]["newton_iterations"]
        out["converged"] = results[-1]["converged"]
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="drape_b200", choices=["drape_b200", "reference"])
    ap.add_argument("--n", type=int, default=129)
    ap.add_argument("--plane", type=int, default=1)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--pcg-max", type=int, default=2000)
    ap.add_argument("--max-steps", type=int, default=1000)
    ap.add_argument("--cpu-budget", type=float, default=20.0)
    ap.add_argument("--full-solve", action="store_true",
                    help="--impl reference: time the oracle's whole solve instead of a bounded sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--preconditioner", default="learned", choices=["jacobi", "multilevel", "learned"])
    ap.add_argument("--compare", default="jacobi", choices=["none", "jacobi", "all"],
                    help="after the timed steps, one device-timed solve of the same workload with each other solver")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
