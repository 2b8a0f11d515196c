"""Trains the preconditioner network on tuples that drape solves emit on the GPU and writes the shipped weights
(drape_b200/preconditioner_network.bin).

    python -m drape_b200.train_preconditioner [--out PATH] [--seeds 8] [--steps 1200] [--json PATH]

Training set: sheets over a sphere of radius U(0.15, 0.35) m and the ground plane, E log-uniform in
[1e5, 2e6] Pa, n in {33, 65}, seeds 1..S (seed 0, the n129 bench scene, is held out). From each drape, the
pseudo-transient systems at several depths of its solve: the projected tangent (SPD) with its inertia term,
right-hand side = the Newton right-hand side there, solution = multilevel PCG to 1e-8; per system also two random
error probes e (b = A e: the high-frequency error the fine smoother acts on) and, twice, the dominant eigenvector
of D^{-1} A (its one-cycle error nears 1 where a row's smoothing turns unstable, so the loss keeps the learned
damping inside the stable range). Loss per tuple: the A-norm error of one V-cycle, ||x - M b||_A^2 / ||x||_A^2;
Adam on the GPU (hand-written kernels, nn.cu).
Evaluation: the held-out n129 seed-0 systems (loss and PCG iterations, multilevel vs learned).
"""
import argparse
import json
import math
import os
import sys
import time

import numpy as np

from drape_b200 import api

GRAVITY = np.array([0.0, -9.81, 0.0])


def _system(d):
    x = d.state
    h = d.final_h()
    x_hat = x + h * h * np.tile(GRAVITY, d.V)
    d.set_options(api.default_options(tangent=1))
    g, blocks = d.assemble(x, x_hat=x_hat, h=h, mode=0, curvature=False)
    return blocks, -g


def _spmv(row_ptr, col_idx, blocks, v):
    """A v for 9B row-major f32 blocks (f64 arithmetic)."""
    B = np.asarray(blocks, np.float64).reshape(-1, 3, 3)
    rows = np.repeat(np.arange(len(row_ptr) - 1), np.diff(row_ptr))
    out = np.zeros((len(row_ptr) - 1, 3))
    np.add.at(out, rows, np.einsum("kab,kb->ka", B, v.reshape(-1, 3)[col_idx]))
    return out.reshape(-1)


def _top_mode(row_ptr, col_idx, blocks, steps=60):
    """Dominant eigenvector of D^{-1} A (power method, f64): the mode a too-strong smoother amplifies."""
    B = np.asarray(blocks, np.float64).reshape(-1, 3, 3)
    R = len(row_ptr) - 1
    rows = np.repeat(np.arange(R), np.diff(row_ptr))
    Dinv = np.linalg.inv(B[(rows == col_idx)])
    v = np.random.default_rng(R).standard_normal(3 * R)
    for _ in range(steps):
        v = np.einsum("kab,kb->ka", Dinv, _spmv(row_ptr, col_idx, blocks, v).reshape(-1, 3)).reshape(-1)
        v /= np.linalg.norm(v)
    return v


def drape_tuples(n, seed, radius, young, depths, probes=2, rng=None):
    """A drape, its (blocks, rhs, PCG solution) tuples at the given PTC depths and `probes` random error probes
    (blocks, A e, e) per system."""
    d = api.Drape.sheet(n, seed=seed, radius=radius, young=young, plane=True,
                        options=api.default_options(preconditioner=1))
    meta, arr = None, None
    out, probe_out, done = [], [], 0
    for depth in depths:
        d.set_options(api.default_options(max_steps=depth - done, preconditioner=1))
        d.solve_equilibrium(start=d.state if done else None, h0=d.final_h() if done else 0.0, check=False)
        done = depth
        blocks, b = _system(d)
        d.set_options(api.default_options(preconditioner=1))
        sol, info = d.pcg(b, 1e-8, 4000, blocks=blocks)
        if info["status"] == "converged":
            out.append((blocks, b, sol))
        if probes and rng is not None:
            if arr is None:
                import tempfile
                with tempfile.TemporaryDirectory() as t:
                    api.write_sheet_problem(t, n, seed=seed, radius=radius, young=young, plane=True)
                    meta, arr = api.read_problem_arrays(t)
            rp, ci = arr["row_ptr"].astype(np.int64), arr["col_idx"].astype(np.int64)
            for _ in range(probes):
                e = rng.standard_normal(3 * d.R)
                probe_out.append((blocks, _spmv(rp, ci, blocks, e), e))
            # the top mode twice: its one-cycle error nears 1 where the smoothing turns unstable
            top = _top_mode(rp, ci, blocks)
            probe_out.extend([(blocks, _spmv(rp, ci, blocks, top), top)] * 2)
    return d, out, probe_out


def pcg_iterations(d, tuples, preconditioner, net=None):
    d.set_options(api.default_options(preconditioner=preconditioner))
    if net is not None:
        d.set_network(net)
    return [d.pcg(b, 1e-6, 2000, blocks=blocks)[1]["iterations"] for blocks, b, _ in tuples]


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=api.NETWORK_FILE)
    ap.add_argument("--seeds", type=int, default=8)
    ap.add_argument("--steps", type=int, default=1200)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--json", default=None)
    args = ap.parse_args(argv)
    rng = np.random.default_rng(2024)
    t0 = time.time()
    groups = {}
    for n, depths in ((33, (5, 20, 60)), (65, (5, 20, 60, 150))):
        for seed in range(1, args.seeds + 1):
            radius = float(rng.uniform(0.15, 0.35))
            young = float(math.exp(rng.uniform(math.log(1e5), math.log(2e6))))
            d, tup, probes = drape_tuples(n, seed, radius, young, depths, 2, rng)
            g = groups.setdefault(n, [d, []])
            g[1].extend(tup + probes)
    t_data = time.time() - t0
    held_d, held, held_probes = drape_tuples(129, 0, 0.25, 5e5, (20, 80, 200), 1, np.random.default_rng(99))
    net = api.Network(seed=0)
    held_before = [net.gradient(held_d, *t)[0] for t in held + held_probes]
    losses = {}
    t1 = time.time()
    rounds = 6
    per = max(1, args.steps // (rounds * len(groups)))
    for r in range(rounds):
        for n, (d, tup) in groups.items():
            losses.setdefault(n, []).extend(net.train(d, tup, per, args.lr).tolist())
    t_train = time.time() - t1
    held_after = [net.gradient(held_d, *t)[0] for t in held + held_probes]
    it_ml = pcg_iterations(held_d, held, 1)
    it_nn = pcg_iterations(held_d, held, 2, net)
    net.save(args.out)
    report = {
        "tuples": {str(n): len(t) for n, (_, t) in groups.items()}, "held_out_tuples": len(held),
        "data_seconds": t_data, "train_seconds": t_train, "steps": per * rounds * len(groups),
        "train_loss_first": {str(n): float(np.mean(l[:len(groups[n][1])])) for n, l in losses.items()},
        "train_loss_last": {str(n): float(np.mean(l[-len(groups[n][1]):])) for n, l in losses.items()},
        "held_out_loss_untrained (solutions, then probes)": held_before, "held_out_loss_trained": held_after,
        "held_out_pcg_iterations_multilevel": it_ml, "held_out_pcg_iterations_learned": it_nn,
        "weights": os.path.relpath(args.out, os.path.dirname(os.path.dirname(os.path.abspath(__file__)))),
    }
    print(json.dumps(report), flush=True)
    if args.json:
        with open(args.json, "w") as f:
            json.dump(report, f, indent=1)
    return 0


if __name__ == "__main__":
    sys.exit(main())
