"""Small, self-contained GPU workloads for profiling one part of the solve (ncu captures, CUDA-event timings).

    python -m drape_b200.profile_workloads cycle   [--n 129] [--steps 20]   # multilevel V-cycle and PCG iteration
    python -m drape_b200.profile_workloads network [--n 129] [--steps 20]   # preconditioner network forward

Both drive `steps` PTC steps of the n x n sheet drape (sphere + ground plane) with the multilevel preconditioner,
assemble the projected (SPD) PTC system at that state, and then:
  cycle    times stand-alone V-cycles and flexible PCG iterations on it (drape_time_multilevel) and a fine SpMV;
  network  runs the shipped network's forward (drape_network_gradient) and one preconditioner-2 PCG solve on it.
"""
import argparse
import ctypes
import json
import sys

import numpy as np

from drape_b200 import api

GRAVITY = np.array([0.0, -9.81, 0.0])


def system(n, steps):
    d = api.Drape.sheet(n, seed=0, plane=True, options=api.default_options(max_steps=steps, preconditioner=1))
    d.solve_equilibrium(check=False)
    x, h = d.state, d.final_h()
    x_hat = x + h * h * np.tile(GRAVITY, d.V)
    d.set_options(api.default_options(tangent=1))
    g, blocks = d.assemble(x, x_hat=x_hat, h=h, mode=0, curvature=False)
    return d, blocks, -g


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("workload", choices=["cycle", "network"])
    ap.add_argument("--n", type=int, default=129)
    ap.add_argument("--steps", type=int, default=20)
    args = ap.parse_args(argv)
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
