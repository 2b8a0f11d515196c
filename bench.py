"""Benchmark of the quasi-static drape GPU stage (one JSON line on rank 0).

Workload: the 1.0 m sheet of n x n vertices (default n = 129: 16641 vertices, 32768 triangles, 48896 hinges,
180993 BSR blocks) over a sphere of radius 0.25 m and a ground plane at y = -0.25 m, isotropic StVK E = 5e5 Pa,
nu = 0.3, t = 5e-4 m, k_b = 1e-5 N m, IPC d_hat = 2e-3 m, kappa = 1e3; PTC from dt0 = 1e-3 s; Newton directions
to the Eisenstat-Walker forcing tolerance in [1e-7, 1e-2], the reference GPU stage's own setting (run-e7.ts:22,
e4_rules.rs:15-22; --forcing 0: a fixed PCG rtol 1e-6), <= 2000 PCG iterations. One step = one full cold solve to
the converged state: |grad E_s| <= 5e-8 N (--absolute), a residual at which the converged state lies within 1e-4 m
of the f64 equilibrium (the vertex error grows about in proportion to the final residual, ~1.3e3 m/N at n129: a solve
stopped at 1e-7 N ends between 0.5e-7 and 1e-7 N and so 0.6e-4 to 1.3e-4 m off); the solve's time to the scene's
1e-6 N Newton tolerance is reported beside it ("secondary": the same run, read from its step records).
Direction solver (--preconditioner): learned (default: the multilevel V-cycle flexible PCG with the shipped
network's fine smoother), multilevel (spectral Jacobi smoothing), jacobi (the reference's block-Jacobi PCG).
--compare all (default) adds one device-timed solve of the same workload with each other direction solver after the
timed steps: block Jacobi (the learned-vs-Jacobi comparison of the metric) and the multilevel preconditioner without
the network (what the network adds); jacobi: block Jacobi only; none: skip. Synthetic scene (the
reference ships no dataset; seeded jitter, seed 0).

value: seconds per converged solve with the problem resident in HBM (CUDA-event-timed solve, max over ranks).
e2e:   the same through the C ABI from host arrays: drape_create (host->device copies) + solve + drape_get_state
       (device->host), wall clock on the host.
error: after the timed steps, the f64 oracle polishes the last converged state on the host (band-Cholesky Newton
       to 1e-8 N) and the line gives the max vertex distance, the relative static-energy error and the f64 residual.
--impl reference: the reference's CPU implementation of this path (the f64 oracle restatement; the Rust crate
       cannot be built here), single-threaded like the reference, on a bounded sample of the same solve, scaled
       by the oracle's own whole solve of this workload (FULL_SOLVE: its time to the sample's step over its time
       to the end, measured once on one core); --full-solve times the oracle's whole solve instead.
--probe cycle|network|spmv|solve: the stand-alone workloads the profiles were captured on (see probe()).
Multi-GPU: replicas only (one independent drape per rank, no collective on the data path).
"""
import argparse
import json
import os
import re
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


def tolerance_crossing(records, tolerance):
    """The solve's figures at the first moment its |grad E_s| was <= `tolerance`, from the step records of a solve
    run to a tighter tolerance (the solve is deterministic, so a solve stopped at `tolerance` ends exactly there):
    host seconds, PTC steps, Newton and PCG iterations up to that moment; None if the solve never got there."""
    for k, r in enumerate(records):
        if r["residual"] <= tolerance:
            done = records[:k]
            return {"tolerance_N": tolerance, "seconds": done[-1]["seconds"] if done else 0.0, "ptc_steps": k,
                    "newton_iterations": int(sum(d["inner"] for d in done)),
                    "pcg_iterations": int(sum(d["pcg_iterations"] for d in done))}
    return None


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
                                   equilibrium_absolute=args.absolute, prolongation=args.prolongation,
                                   forcing=args.forcing,
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
        records = drape.step_records()
        drape.close()
        # The solve's time: CUDA events recorded by the library on its stream at the start and end of the solve
        # (with a synchronize before the end event is read); the host decisions between launches are inside.
        return log, log["device_seconds"], t1 - t0, state, records

    for _ in range(args.warmup):
        one_step()
    logs, secs, e2e = [], [], []
    with ClockSampler(local) as clock:
        for _ in range(args.steps):
            log, s_dev, w, state, records = one_step()
            logs.append(log)
            secs.append(s_dev)
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
        tpath = os.path.join(ROOT, "profiles", "multilevel_traffic.json")
        if os.path.exists(tpath):
            tr = json.load(open(tpath))
            if tr.get("columns") == args.n:
                # DRAM bytes of one flexible PCG iteration (the sum over its kernels, ncu capture of the stand-alone
                # cycle workload, bench.py --probe cycle), expressed per launch of the solve graph like `achieved`.
                traffic = tr["dram_bytes_per_iteration"] * last["pcg_iterations"] / max(1, last["pcg_launches"])
    achieved = (bytes_per_iter * last["pcg_iterations"]) / (last["ms_pcg"] / 1e3) / 1e9 if last["ms_pcg"] > 0 else 0.0
    # Device-time equivalent of the secondary tolerance's host seconds (the solve's device/host time ratio).
    scale = last["device_seconds"] / last["seconds"] if last["seconds"] > 0 else 1.0
    secondary = tolerance_crossing(records, args.secondary)
    if secondary:
        secondary["device_seconds"] = secondary["seconds"] * scale
    comparison = {}
    others = {"none": (), "jacobi": ("jacobi",), "all": ("jacobi", "multilevel", "learned")}[args.compare]
    if others:  # every rank runs the same comparison solves (replicas; one_step holds the barriers), rank 0 reports
        for other in others:
            if other == args.preconditioner:
                continue
            log_o, s_o, _, _, rec_o = one_step(other)
            sec_o = tolerance_crossing(rec_o, args.secondary)
            if sec_o:
                sec_o["device_seconds"] = sec_o["seconds"] * (log_o["device_seconds"] / max(log_o["seconds"], 1e-9))
            comparison[other] = {"seconds": s_o, "ptc_steps": log_o["ptc_steps"],
                                 "newton_iterations": log_o["newton_iterations"],
                                 "pcg_iterations": log_o["pcg_iterations"],
                                 "pcg_per_newton": log_o["pcg_iterations"] / max(1, log_o["newton_iterations"]),
                                 "fallbacks_to_jacobi": log_o["fallbacks"], "converged": log_o["reason"] == "tolerance",
                                 "final_residual_N": log_o["final_residual"], "secondary": sec_o}
        if "jacobi" in comparison:
            comparison["jacobi_seconds_over_this"] = comparison["jacobi"]["seconds"] / t
            if secondary and comparison["jacobi"]["secondary"]:
                comparison["jacobi_over_this_at_secondary"] = (comparison["jacobi"]["secondary"]["device_seconds"] /
                                                               max(secondary["device_seconds"], 1e-9))
    out = {
        "metric": METRIC, "value": t, "unit": "s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t * 1e3, "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": f"sheet n{args.n} over sphere r=0.25 + ground plane y=-0.25, {PRECOND[args.preconditioner]}, "
                               f"PTC dt0=1e-3 s to |grad E_s|<={args.absolute:g} N, "
                               f"{'Eisenstat-Walker forcing' if args.forcing else 'PCG rtol 1e-6'}",
                   "columns": args.n, "rows": R,
                   "blocks": B, "seed": args.seed, "preconditioner": args.preconditioner,
                   "tolerance_N": args.absolute, "prolongation": ["bilinear", "smoothed"][args.prolongation],
                   "forcing": ["fixed rtol 1e-6", "eisenstat-walker"][args.forcing],
                   "parallelism": f"replicas{world}",
                   "l2": "flushed (512 MiB write) before every timed solve"},
        "solve": {"converged": last["reason"] == "tolerance", "reason": last["reason"],
                  "final_residual_N": last["final_residual"], "ptc_steps": last["ptc_steps"],
                  "newton_iterations": last["newton_iterations"], "pcg_iterations": last["pcg_iterations"],
                  "pcg_per_newton": last["pcg_iterations"] / max(1, last["newton_iterations"]),
                  "rejected_attempts": last["rejected_attempts"], "static_energy_J": last["static_energy"],
                  "fallbacks_to_jacobi": last["fallbacks"], "mg_levels": last["mg_levels"],
                  "phase_ms": {k: last[k] for k in ("ms_assembly", "ms_pcg", "ms_line_search", "ms_ccd", "ms_other")}},
        "secondary": secondary,
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
        out["cpu_baseline"], out["error"] = cpu_leg(args, state)
    if dist:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)


# The f64 oracle's own whole cold solve of a bench workload, keyed by (n, plane, seed, tolerance in N): its time,
# counts, and its cumulative time at the end of each of its first PTC steps (the scale of a bounded sample). Run
# once with `python bench.py --impl reference --full-solve --record` on one core of the build container (Intel Xeon
# @ 2.7 GHz), not on the GPU box. None where it has not been run.
FULL_SOLVE = {
    (33, 1, 0, 1e-07): {
        "seconds": 30.231,
        "steps": 76,
        "newton": 494,
        "seconds_to_1e-6": 29.961,
        "host": "Intel(R) Xeon(R) Processor @ 2.70GHz (build container), 1 core",
        "seconds_at_step": [0.01, 0.02, 0.031, 0.043, 0.06, 0.084, 0.113, 0.366, 0.615, 0.985, 1.03, 1.23, 1.807,
            1.884, 2.429, 3.55, 3.699, 4.047, 4.328, 4.616, 4.735, 5.064, 5.323, 5.359, 5.48, 5.856, 6.297, 6.353,
            6.434, 7.072, 7.274, 7.783, 8.45, 8.944, 9.397, 9.626, 9.888, 9.924, 9.981, 10.312, 10.741, 10.832,
            11.537, 11.771, 12.602, 12.872, 13.568, 13.943, 14.064, 14.433, 14.639, 14.923, 15.368, 16.065, 16.396,
            16.661, 17.251, 18.468, 18.843, 19.546, 20.746, 21.452, 21.662, 22.632, 23.599, 24.356, 25.289, 25.68,
            26.142, 26.613, 27.442, 28.568, 28.888, 29.68, 29.961, 30.231],
    },
    (129, 1, 0, 1e-07): {
        "seconds": 8965.712,
        "steps": 431,
        "newton": 3237,
        "seconds_to_1e-6": 8472.771,
        "host": "Intel(R) Xeon(R) Processor (build container, no clock in its CPU name), 1 core",
        "seconds_at_step": [
            0.366, 0.785, 1.292, 1.955, 2.884, 4.157, 7.064, 39.91, 49.63, 60.976, 75.578, 77.355, 83.323,
            102.033, 147.126, 168.781, 211.59, 236.475, 270.9, 317.883, 337.182, 376.098, 407.167, 424.768,
            452.334, 491.779, 520.002, 557.394, 573.288, 605.738, 616.951, 650.855, 658.577, 686.719, 697.442,
            724.934, 738.759, 766.848, 782.684, 816.623, 847.555, 859.376, 884.996, 895.156, 918.974, 930.145,
            956.158, 972.904, 1000.422, 1016.028, 1045.767, 1065.109, 1091.45, 1103.847, 1137.064, 1161.043,
            1190.085, 1207.554, 1247.183, 1268.312, 1298.316, 1313.962, 1342.654, 1369.212, 1415.393, 1446.949,
            1479.8, 1507.294, 1517.52, 1541.615, 1573.308, 1598.021, 1604.048, 1630.966, 1636.861, 1656.489,
            1685.51, 1712.012, 1721.576, 1741.144, 1766.459, 1789.404, 1796.173, 1812.526, 1838.282, 1866.343,
            1885.819, 1889.903, 1900.014, 1926.695, 1935.9, 1961.043, 1978.794, 2009.695, 2020.099, 2053.388,
            2059.87, 2096.711, 2106.306, 2140.13, 2151.13, 2185.051, 2195.781, 2221.775, 2229.619, 2261.79,
            2270.308, 2300.819, 2309.233, 2337.192, 2346.582, 2384.263, 2410.179, 2414.277, 2422.433, 2450.38,
            2463.091, 2490.254, 2504.239, 2529.289, 2553.123, 2557.752, 2569.641, 2600.317, 2610.187, 2644.243,
            2656.823, 2692.477, 2701.367, 2729.738, 2740.825, 2775.218, 2790.942, 2820.022, 2835.408, 2873.889,
            2886.011, 2917.516, 2926.682, 2952.542, 2974.35, 3006.1, 3020.875, 3051.847, 3067.346, 3101.975,
            3106.224, 3149.233, 3160.137, 3200.28, 3224.53, 3260.222, 3277.43, 3316.132, 3337.037, 3367.234,
            3394.34, 3417.197, 3437.013, 3467.221, 3480.286, 3515.739, 3544.973, 3550.751, 3568.507, 3601.066,
            3616.833, 3649.984, 3670.063, 3674.519, 3696.005, 3699.037, 3724.183, 3754.382, 3766.618, 3800.24,
            3810.846, 3850.346, 3864.678, 3892.855, 3901.142, 3936.882, 3944.365, 3981.211, 4005.19, 4008.95,
            4020.785, 4053.378, 4065.284, 4097.417, 4116.42, 4145.252, 4160.847, 4172.001, 4189.752, 4218.832,
            4233.571, 4272.941, 4276.733, 4305.249],
    },
    (129, 1, 0, 5e-08): {
        "seconds": 9193.558,
        "steps": 436,
        "newton": 3279,
        "seconds_to_1e-6": 8649.817,
        "host": "Intel(R) Xeon(R) Processor (build container, no clock in its CPU name), 1 core",
        "seconds_at_step": [
            0.252, 0.612, 1.096, 1.582, 2.365, 3.349, 5.371, 33.773, 40.415, 47.943, 59.426, 61.023, 66.331,
            78.808, 114.158, 134.0, 169.197, 186.085, 216.042, 259.513, 277.803, 313.968, 338.487, 349.592,
            369.932, 397.142, 416.001, 443.805, 455.403, 477.934, 487.788, 515.175, 522.002, 544.106, 553.037,
            575.63, 587.111, 609.718, 621.84, 650.712, 681.015, 693.89, 721.145, 731.462, 757.417, 769.124,
            798.536, 817.143, 844.958, 861.303, 887.201, 902.953, 929.686, 941.799, 973.687, 999.004, 1023.507,
            1042.622, 1076.475, 1096.883, 1126.009, 1142.787, 1169.243, 1193.203, 1232.283, 1256.089, 1288.835,
            1317.036, 1330.465, 1355.946, 1388.652, 1417.296, 1423.726, 1452.473, 1459.956, 1479.496, 1508.75,
            1535.79, 1547.649, 1573.039, 1605.517, 1637.682, 1646.987, 1666.15, 1699.002, 1732.166, 1755.795,
            1761.438, 1771.386, 1804.027, 1815.003, 1846.583, 1865.054, 1896.579, 1907.436, 1939.068, 1947.003,
            1984.09, 1994.73, 2028.816, 2040.063, 2073.508, 2085.412, 2113.371, 2120.736, 2146.498, 2157.908,
            2189.732, 2198.322, 2228.088, 2237.589, 2267.755, 2291.004, 2294.499, 2304.595, 2334.036, 2345.801,
            2375.588, 2386.53, 2410.338, 2436.403, 2442.512, 2455.995, 2484.389, 2493.58, 2524.913, 2537.127,
            2577.346, 2588.525, 2626.421, 2636.767, 2669.054, 2683.327, 2713.382, 2728.029, 2764.962, 2774.044,
            2802.209, 2810.59, 2839.018, 2862.827, 2891.149, 2904.568, 2937.023, 2949.91, 2984.113, 2989.636,
            3029.815, 3039.927, 3075.211, 3095.64, 3126.841, 3142.973, 3174.855, 3194.216, 3226.962, 3251.485,
            3276.493, 3299.24, 3334.378, 3347.114, 3379.064, 3406.31, 3413.33, 3434.548, 3471.193, 3486.602,
            3521.737, 3544.813, 3549.583, 3572.984, 3576.27, 3604.912, 3643.004, 3659.79, 3694.014, 3704.601,
            3744.314, 3759.744, 3792.812, 3803.279, 3838.689, 3846.635, 3880.548, 3903.499, 3905.987, 3916.138,
            3952.336, 3966.76, 4003.56, 4022.422, 4060.229, 4082.336, 4093.159, 4116.376, 4146.725, 4158.566,
            4194.236, 4197.347, 4222.262],
    },
}


def _oracle_solve(args, budget):
    """The oracle's cold solve of the bench workload (port of the reference crate's method: exact tangent, LM, f64
    block-Jacobi PCG rtol 1e-6 <= 2000 iterations, inner-count PTC from dt0 = 1e-3 s), stopped at the first PTC step
    that ends past `budget` s (0: to the tolerance). Returns its statistics (oracle_py.Scene.ptc)."""
    from tests import oracle_py

    s = oracle_py.Scene("sheet", args.n, seed=args.seed, plane=bool(args.plane))
    _, st = s.ptc(h0=1e-3, doubling=False, absolute=args.absolute, pcg=True, rtol=1e-6, maxit=2000, budget_s=budget)
    return st


def cpu_baseline(args, budget_s=None):
    """The f64 oracle timed on this host, single-threaded like the reference crate: a bounded sample of the cold
    solve (the PTC steps that end within `budget_s`), scaled by the oracle's own whole solve of this workload
    (FULL_SOLVE: whole-solve seconds over its seconds to the same step). Without a whole-solve record (or with
    budget 0) the solve runs to the end and its own time is the value."""
    budget = budget_s if budget_s is not None else args.cpu_budget
    key = (args.n, int(args.plane), args.seed, args.absolute)
    whole = FULL_SOLVE.get(key)
    if whole is None and args.n <= 33:
        budget = 0.0  # small enough to run whole (n33: ~30 s on one core)
    st = _oracle_solve(args, budget)
    steps, elapsed, newton = int(st["steps"]), st["seconds"], int(st["newton"])
    base = {"unit": "s", "cores": 1, "kind": "port", "host_cpu": _cpu_model()}
    if whole is None and budget != 0.0:
        # No whole-solve record to scale by: the sample is reported as what it is, a lower bound.
        return dict(base, value=elapsed, sample_only=True,
                    sample=f"{steps} PTC steps ({newton} Newton iterations) of the n{args.n} solve in {elapsed:.1f} s "
                           f"on 1 host core; no whole-solve record of this workload, so the value is the sample's "
                           f"time alone (a lower bound of the whole solve's)")
    if budget == 0.0:
        return dict(base, value=elapsed, newton_iterations=newton, converged=bool(st["converged"]),
                    sample=f"the whole n{args.n} solve to {args.absolute:g} N ({steps} PTC steps, {newton} Newton "
                           f"iterations) on 1 host core")
    at = whole["seconds_at_step"]
    k = min(steps, len(at))
    ratio = whole["seconds"] / at[k - 1]
    return dict(base, value=elapsed * ratio, extrapolated=True,
                sample=f"{steps} PTC steps ({newton} Newton iterations) of the n{args.n} solve in {elapsed:.1f} s on 1 "
                       f"host core, x {ratio:.2f} = the oracle's own whole solve to {args.absolute:g} N "
                       f"({whole['steps']} PTC steps, {whole['newton']} Newton iterations, {whole['seconds']:.0f} s on "
                       f"{whole['host']}) over its first {k} steps ({at[k - 1]:.1f} s there)",
                whole_solve_measured={"seconds": whole["seconds"], "ptc_steps": whole["steps"],
                                      "newton_iterations": whole["newton"], "host": whole["host"],
                                      "seconds_to_1e-6_N": whole.get("seconds_to_1e-6")})


def cpu_leg(args, gpu_state):
    """Rank 0, after the timed steps: the CPU baseline, and the f64 error of the last converged GPU state (the oracle
    polishes it with band-Cholesky Newton to 1e-8 N; max vertex distance, relative static-energy error, the f64
    residual at the GPU state)."""
    from tests import oracle_py
    from tests.polish_state import polished_error

    oracle_py.build()
    base = cpu_baseline(args)
    t0 = time.perf_counter()
    oracle = oracle_py.Scene("sheet", args.n, seed=args.seed, plane=bool(args.plane))
    err, e_rel, r64, _, st = polished_error(oracle, gpu_state, require_converged=False)
    error = {"max_vertex_m": err, "relative_energy": e_rel, "f64_residual_N": r64,
             "polish_converged": bool(st["converged"]), "polish_newton": int(st["newton"]),
             "polish_cpu_s": time.perf_counter() - t0, "bound_m": 1e-4, "within_bound": bool(err <= 1e-4)}
    return base, error


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
        r = cpu_baseline(args, budget_s=budget)
        if i >= args.warmup:
            results.append(r)
    v = sum(r["value"] for r in results) / len(results)
    out = {"metric": METRIC, "value": v, "unit": "s", "n_gpus": int(os.environ.get("WORLD_SIZE", "1")),
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": v * 1e3, "higher_is_better": False,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
           "config": {"workload": f"sheet n{args.n} over sphere r=0.25 + ground plane y=-0.25, f64 oracle port "
                                  f"(exact tangent, LM, block-Jacobi PCG rtol 1e-6 <= 2000), PTC dt0=1e-3 s to "
                                  f"|grad E_s|<={args.absolute:g} N", "columns": args.n, "tolerance_N": args.absolute},
           "cpu_baseline": {k: results[-1][k] for k in results[-1] if k != "value"} | {"value": v},
           "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if "newton_iterations" in results[-1]:
        out["newton_iterations"] = results[-1]["newton_iterations"]
        out["converged"] = results[-1]["converged"]
    print(json.dumps(out), flush=True)


def record_full_solve(args):
    """--impl reference --full-solve --record: the oracle's whole solve with per-step times (its progress lines),
    printed as the FULL_SOLVE entry for this workload."""
    from tests import oracle_py

    oracle_py.build()
    cmd = [sys.executable, "-c",
           "import sys; sys.path.insert(0, %r); from tests import oracle_py; "
           "s = oracle_py.Scene('sheet', %d, seed=%d, plane=%s); "
           "s.ptc(h0=1e-3, doubling=False, absolute=%r, pcg=True, rtol=1e-6, maxit=2000, progress=True)"
           % (ROOT, args.n, args.seed, bool(args.plane), args.absolute)]
    proc = subprocess.run(cmd, stderr=subprocess.PIPE, text=True, check=True)
    print(json.dumps(parse_progress(proc.stderr.splitlines(), _cpu_model())), flush=True)


def parse_progress(lines, host):
    """FULL_SOLVE entry from the oracle's progress lines ('state after K steps: residual R N at T s, N Newton
    iterations'): cumulative seconds at the end of each of the first 200 steps, the whole solve, and the time at
    which the residual first fell to 1e-6 N."""
    pat = re.compile(r"state after (\d+) steps: residual ([0-9.eE+-]+) N at ([0-9.]+) s, (\d+) Newton")
    at, t6, last = [], None, None
    for line in lines:
        m = pat.search(line)
        if not m:
            continue
        k, r, sec, newton = int(m.group(1)), float(m.group(2)), float(m.group(3)), int(m.group(4))
        if k >= 1 and len(at) < 200:
            at.append(sec)
        if t6 is None and r <= 1e-6:
            t6 = sec
        last = (k, sec, newton)
    return {"seconds": last[1], "steps": last[0], "newton": last[2], "seconds_to_1e-6": t6, "host": host,
            "seconds_at_step": at}


def probe(args):
    """Stand-alone workloads the profiles were captured on (ncu needs kernels outside the solve's conditional
    graph, and small, repeatable cases):
      cycle    PTC steps of the n x n sheet drape with the multilevel preconditioner, then the projected PTC system
               at that state: stand-alone V-cycles and flexible PCG iterations on it (drape_time_multilevel), a
               fine SpMV;
      network  the same system: the shipped network's forward (drape_network_gradient) and one learned PCG solve;
      spmv     `drapes` sheets of the batched configuration concatenated block-diagonally, and the n257 sheet's
               matrix: every lanes-per-row x threads shape of the SpMV kernel timed, the fastest checked against
               numpy and reported in algorithmic GB/s (40 B per block + 28 B per row) against the measured HBM peak;
      solve    the bench scene's cold solve to --absolute; the converged positions go to --out (an .npy file)."""
    import ctypes

    import numpy as np

    from drape_b200 import api
    from drape_b200.scenes import GRAVITY, batch_scenes, sheet_matrix

    pre = {"jacobi": 0, "multilevel": 1, "learned": 2}[args.preconditioner]
    if args.probe == "solve":
        d = api.Drape.sheet(args.n, seed=args.seed, plane=bool(args.plane),
                            options=api.default_options(preconditioner=pre, equilibrium_absolute=args.absolute,
                                                        time_budget_s=args.budget, prolongation=args.prolongation,
                                                        forcing=args.forcing, progress=1))
        if pre == 2:
            d.set_network(api.Network.trained())
        log = d.solve_equilibrium(check=False)
        if args.out:
            np.save(args.out, d.state)
        keys = ("reason", "ptc_steps", "newton_iterations", "pcg_iterations", "fallbacks", "ms_pcg", "ms_assembly",
                "ms_other", "final_residual", "device_seconds", "static_energy", "kernel_launches")
        return {k: log[k] for k in keys}
    if args.probe == "spmv":
        parts, offset = [], 0
        for n, seed, radius, young in batch_scenes(args.drapes):
            rp, ci, blk = sheet_matrix(n, seed, radius, young)
            parts.append((rp, ci + offset, blk))
            offset += len(rp) - 1
        rp_all, base = [np.zeros(1, np.int64)], 0
        for rp, _, _ in parts:
            rp_all.append(rp[1:] + base)
            base += rp[-1]
        batch = (np.concatenate(rp_all), np.concatenate([p[1] for p in parts]), np.concatenate([p[2] for p in parts]))
        peak = peaks()["hbm_gbs"]
        out = {}
        for name, (rp, ci, blk) in (("batched", batch), ("n257", sheet_matrix(257, 0, 0.25, 5e5))):
            R, B = len(rp) - 1, len(ci)
            x = np.random.default_rng(1).standard_normal(3 * R).astype(np.float32)
            shapes = {f"{lanes}x{threads}": api.spmv_benchmark(rp, ci, blk, x, 20, lanes, threads)
                      for lanes in (4, 8, 16, 32) for threads in (128, 256)}
            best = min(shapes, key=shapes.get)
            lanes, threads = (int(v) for v in best.split("x"))
            ms, y = api.spmv_benchmark(rp, ci, blk, x, 20, lanes, threads, result=True)
            rows = np.repeat(np.arange(R), np.diff(rp))
            ref = np.zeros((R, 3))
            np.add.at(ref, rows, np.einsum("kab,kb->ka", blk.reshape(-1, 3, 3).astype(np.float64),
                                           x.reshape(-1, 3).astype(np.float64)[ci]))
            bytes_ = 40 * B + 28 * R
            out[name] = {"rows": R, "blocks": B, "algorithmic_MB": bytes_ / 1e6, "best_shape": best, "ms": ms,
                         "GB_per_s": bytes_ / (ms * 1e-3) / 1e9, "fraction_of_peak": bytes_ / (ms * 1e-3) / 1e9 / peak,
                         "peak_GB_per_s": peak,
                         "relative_error_vs_numpy": float(np.linalg.norm(y - ref.reshape(-1)) / np.linalg.norm(ref)),
                         "all_shapes_ms": shapes}
        return out
    d = api.Drape.sheet(args.n, seed=args.seed, plane=bool(args.plane),
                        options=api.default_options(max_steps=args.probe_steps, preconditioner=1))
    d.solve_equilibrium(check=False)
    x, h = d.state, d.final_h()
    d.set_options(api.default_options(tangent=1))
    g, blocks = d.assemble(x, x_hat=x + h * h * np.tile(GRAVITY, d.V), h=h, mode=0, curvature=False)
    b = -g
    lib = api.load()
    out = {"probe": args.probe, "columns": args.n, "ptc_steps": args.probe_steps}
    if args.probe == "cycle":
        d.set_options(api.default_options(preconditioner=1, prolongation=args.prolongation))
        _, info = d.pcg(b, 1e-6, 2000, blocks=blocks)
        out["pcg"] = info
        lib.drape_time_multilevel.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p]
        tm = (ctypes.c_float * 6)()
        for its in (20, 200):
            assert lib.drape_time_multilevel(d.h, its, tm) == 0, lib.drape_last_error(d.h)
            out[f"iterations_{its}"] = {"vcycle_ms": tm[0], "pcg_iteration_ms": tm[1], "pdl": tm[2],
                                        "pcg_iteration_stream_ms": tm[3], "setup_fresh_ms": tm[4],
                                        "setup_reuse_ms": tm[5]}
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
    return out


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
    ap.add_argument("--absolute", type=float, default=5e-8, help="stop at |grad E_s| <= this (N)")
    ap.add_argument("--secondary", type=float, default=1e-6,
                    help="also report the time at which the solve first reached |grad E_s| <= this (N)")
    ap.add_argument("--cpu-budget", type=float, default=20.0)
    ap.add_argument("--full-solve", action="store_true",
                    help="--impl reference: time the oracle's whole solve instead of a bounded sample")
    ap.add_argument("--record", action="store_true",
                    help="--impl reference --full-solve: print the FULL_SOLVE entry (per-step times) of the solve")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--preconditioner", default="learned", choices=["jacobi", "multilevel", "learned"])
    ap.add_argument("--forcing", type=int, default=1, choices=[0, 1],
                    help="Newton direction tolerance: 1 (default) Eisenstat-Walker, the reference GPU stage's setting "
                         "(run-e7.ts:22 forcing: true; e4_rules.rs:15-22); 0 a fixed PCG rtol 1e-6")
    ap.add_argument("--prolongation", type=int, default=0, choices=[0, 1],
                    help="multilevel fine-to-coarse prolongation: 0 bilinear (default), 1 smoothed once")
    ap.add_argument("--compare", default="all", choices=["none", "jacobi", "all"],
                    help="after the timed steps, one device-timed solve of the same workload with each other solver")
    ap.add_argument("--probe", default=None, choices=["cycle", "network", "spmv", "solve"],
                    help="run one stand-alone profiling workload instead of the benchmark (see probe())")
    ap.add_argument("--probe-steps", type=int, default=20, help="--probe cycle/network: PTC steps before the system")
    ap.add_argument("--drapes", type=int, default=128, help="--probe spmv: drapes of the batched configuration")
    ap.add_argument("--budget", type=float, default=0.0, help="--probe solve: the solver's time budget, s")
    ap.add_argument("--out", default=None, help="--probe solve: .npy file for the converged positions")
    args = ap.parse_args()
    if args.probe:
        print(json.dumps(probe(args)), flush=True)
    elif args.impl == "reference":
        if args.full_solve and args.record:
            record_full_solve(args)
        else:
            run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
