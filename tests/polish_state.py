"""f64 error of a converged GPU state (checker, runs on the host only):

    python -m tests.polish_state --n 257 state.npy

The oracle's f64 PTC with band-Cholesky Newton (tests/oracle_py.py Scene.ptc: h0 = 1 s, no step doubling) polishes
the state of the n x n sheet drape (sphere + ground plane, seed 0) to |grad E_s| <= 1e-8 N; the line printed
gives the f64 |grad E_s| at the GPU state, the largest vertex distance between the two states and the relative
static-energy error."""
import argparse
import json
import time

import numpy as np

from tests import oracle_py


def polished_error(oracle, x_g, require_converged=True):
    """The frictionless drape has many equilibria (folds on the floor, wrinkles), and which one a solve reaches
    depends on its path: the f32 PCG directions and the f64 band Cholesky ones take different paths from the
    same cold start. The error of a converged GPU state is therefore measured by the f64 oracle itself: its f64
    residual at the GPU state, and its own Newton/PTC solve started there and run to 1e-8 N, which lands on the
    f64 equilibrium of that basin. Returns (max vertex error m, relative static-energy error, f64 residual N,
    the polished state, the polish's statistics)."""
    r64 = float(np.linalg.norm(oracle.static_gradient(x_g)))
    x_o, st = oracle.ptc(start=x_g, h0=1.0, doubling=False, absolute=1e-8, pcg=False, max_steps=200)
    if require_converged:
        assert st["converged"] == 1.0, st
    err = float(np.abs(x_g - x_o).reshape(-1, 3).max())
    e_o = oracle.static_energy(x_o)
    return err, abs(oracle.static_energy(x_g) - e_o) / abs(e_o), r64, x_o, st


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("state", nargs="+", help=".npy files of 3V f64 positions")
    ap.add_argument("--n", type=int, default=129)
    args = ap.parse_args(argv)
    oracle = oracle_py.Scene("sheet", args.n, seed=0, plane=True)
    for path in args.state:
        x_g = np.load(path)
        t = time.time()
        err, e_rel, r64, _, st = polished_error(oracle, x_g, require_converged=False)
        print(json.dumps({"state": path, "r64_N": r64, "polish": st, "max_vertex_error_m": err,
                          "rel_energy_error": e_rel, "cpu_s": time.time() - t}), flush=True)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
