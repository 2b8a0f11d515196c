"""f64 error of a converged GPU state (checker, runs on the host only):

    python -m tests.polish_state --n 257 state.npy [--absolute 1e-8]

The oracle's f64 PTC with band-Cholesky Newton (tests/oracle_py.py Scene.ptc: h0 = 1 s, no step doubling) polishes
the state of the n x n sheet drape (sphere + ground plane, seed 0) to |grad E_s| <= `absolute`; the line printed
gives the f64 |grad E_s| at the GPU state, the largest vertex distance between the two states and the relative
static-energy error."""
import argparse
import json
import time

import numpy as np

from tests import oracle_py


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("state", nargs="+", help=".npy files of 3V f64 positions")
    ap.add_argument("--n", type=int, default=129)
    ap.add_argument("--absolute", type=float, default=1e-8)
    args = ap.parse_args(argv)
    oracle = oracle_py.Scene("sheet", args.n, seed=0, plane=True)
    for path in args.state:
        x_g = np.load(path)
        t = time.time()
        r64 = float(np.linalg.norm(oracle.static_gradient(x_g)))
        x_o, st = oracle.ptc(start=x_g, h0=1.0, doubling=False, absolute=args.absolute, pcg=False, max_steps=200)
        err = float(np.abs(x_g - x_o).reshape(-1, 3).max())
        e_o = oracle.static_energy(x_o)
        print(json.dumps({"state": path, "r64_N": r64, "polish": st, "max_vertex_error_m": err,
                          "rel_energy_error": abs(oracle.static_energy(x_g) - e_o) / abs(e_o),
                          "cpu_s": time.time() - t}), flush=True)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
