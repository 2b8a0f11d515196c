"""The reference comparer's verdict on one GPU run (engine/oracle/src/e7_compare.rs:276-363), restated as a test
checker over the `drape` command's gpu-<mode>/ files and the f64 oracle:

  intersection_free        every kept f32 state (in f64) and every accepted step's recorded minimum distance
                           stays outside the colliders (e7_compare.rs:264-273)
  rules_replayed_ok        Eisenstat-Walker forcing (<= 1e-5), the PTC controller, the rejections, and on probe
                           files alpha_max, resolution and line-search acceptance (e7_compare.rs:240-261)
  static_energy_ok         E_s rises by at most 1e-6 of max |E_s| between kept states (e7_compare.rs:100-104)
  final_state_residual_ok  the final f32 state's f64 r/L <= max(1e-3, 2 x the representation floor: r/L of the
                           oracle's cold equilibrium rounded to f32) (e7_compare.rs:276-290)
  oracle_converged         the oracle's own run of the mode converged (its reference-<mode>.json), when present
  start_feasible           a warm or prolong run's start state lies outside the colliders (e7_compare.rs:145-156)
and the diagnostics: energy gap and largest vertex gap against the oracle's cold equilibrium (e7_compare.rs:293-299),
the f64 r/L of the final state, the smallest distance over d_hat. `python -m tests.e7_compare --dir D --mode M
[--start prefix]` prints the verdict and writes gpu-<mode>/result.json (schema e7-result/1)."""
import argparse
import json
import os

import numpy as np

from drape_b200 import api
from tests import e7_replays, oracle_py

ENERGY_LIMIT = 1e-6
RESIDUAL_FLOOR_ALLOWANCE = 1e-3
FLOOR_FACTOR = 2.0


def distances(colliders, x):
    """Smallest vertex-collider distance per vertex (colliders packed 8 per entry: kind 1 plane n.x = w, 2 sphere
    |x - c| = w)."""
    p = x.reshape(-1, 3)
    best = np.full(len(p), np.inf)
    for c in np.asarray(colliders, np.float64).reshape(-1, 8):
        a = c[1:4]
        d = p @ a - c[4] if c[0] == 1 else np.linalg.norm(p - a, axis=1) - c[4]
        best = np.minimum(best, d)
    return best


def _state(prefix):
    meta = json.load(open(prefix + ".json"))
    return np.fromfile(prefix + ".bin", np.float32 if meta["dtype"] == "f32" else np.float64).astype(np.float64)


def compare(case_dir, mode, oracle, start=None):
    """(verdict, details) of the run in case_dir/gpu-<mode>; `oracle` the case's oracle_py.Scene; `start` the start
    state prefix of a warm or prolong run."""
    out = os.path.join(case_dir, f"gpu-{mode}")
    res, fields, it, rb, at, ptc = e7_replays.read_run(out)
    meta, arr = api.read_problem_arrays(case_dir)
    problem = json.load(open(os.path.join(case_dir, "problem.json")))
    colliders, dhat = arr["colliders"][4:].astype(np.float64), meta["contact"]["dhat_m"]
    free = arr["row_vertex"].astype(int)
    V = arr["rest_positions"].size // 3
    states = np.fromfile(os.path.join(out, "gpu-states.bin"), np.float32).astype(np.float64).reshape(-1, 3 * V)
    verdict, details = {}, {}
    # intersection-free
    ratios = [distances(colliders, x)[free].min() / dhat for x in states]
    ratios += [r / dhat for r in ptc[:, 6] if np.isfinite(r)]
    probe_path = os.path.join(out, "gpu-probe-iterates.bin")
    if os.path.exists(probe_path):
        probes = np.fromfile(probe_path, np.float32).astype(np.float64).reshape(-1, 3 * V)
        ratios += [distances(colliders, x)[free].min() / dhat for x in probes]
    details["min_distance_over_dhat"] = float(min(ratios))
    verdict["intersection_free"] = details["min_distance_over_dhat"] > 0
    # replays
    rules = {"ptc": {k: v for k, v in problem.get("ptc", {}).items()}}
    o = api.default_options()
    for key, value in (("growth", o.growth), ("shrink", o.shrink), ("inner_max_iterations", o.inner_max),
                       ("h0", o.h0), ("h_min_factor", o.h_min_factor), ("h_max", o.h_max)):
        rules["ptc"].setdefault(key, value)
    forcing = e7_replays.forcing_replay(it, rb, fields, at)
    replays = {"forcing_replay_error": float(forcing), "controller_replay_ok": bool(e7_replays.controller_replay(rules, ptc)),
               "rejection_replay_ok": bool(e7_replays.rejection_replay(it, at))}
    probe_ok = True
    if os.path.exists(probe_path):
        pit = np.fromfile(os.path.join(out, "gpu-probe-iterations.bin"), np.float64).reshape(-1, 9)
        prb = np.fromfile(os.path.join(out, "gpu-probe-robust.bin"), np.float64).reshape(-1, len(fields))
        pairs = np.fromfile(os.path.join(out, "gpu-probe-directions.bin"), np.float32).reshape(-1, 2, 3 * V)
        trials = np.fromfile(os.path.join(out, "gpu-probe-search.bin"), np.float64).reshape(-1, 8)
        alpha = max(e7_replays.alpha_errors(pit, prb, fields, pairs, oracle.max_step), default=0.0)
        probe_ok = (e7_replays.resolution_replay(pit, prb, fields, probes, free) and alpha <= 1e-4 and
                    e7_replays.acceptance_replay(trials, problem.get("newton", {}).get("armijo", o.armijo)))
        replays["probe_alpha_worst_error"] = float(alpha)
    replays["probe_replays_ok"] = bool(probe_ok)
    details["replays"] = replays
    verdict["rules_replayed_ok"] = bool(forcing <= 1e-5 and replays["controller_replay_ok"] and
                                        replays["rejection_replay_ok"] and probe_ok)
    # static energy along the kept states
    if len(states) > 2:
        energies = np.array([oracle.static_energy(x) for x in states])
        rise = float(np.max(np.diff(energies)) / np.abs(energies).max())
        details["energy_rise_relative"] = rise
        verdict["static_energy_ok"] = rise <= ENERGY_LIMIT
    # final state and the oracle's references
    final = states[-1]
    r_over_l = float(np.linalg.norm(oracle.static_gradient(final)) / oracle.gravity_load)
    details["final_residual_over_load_f64"] = r_over_l
    floor = 0.0
    own = os.path.join(case_dir, f"reference-{mode}.json")
    if os.path.exists(own):
        ref = json.load(open(own))
        verdict["oracle_converged"] = bool(ref["converged"]) and ref.get("mu_cap_steps", 0) == 0
        details["oracle"] = {k: ref.get(k) for k in ("converged", "ptc_steps", "newton_iterations", "rejected_attempts")}
        floor = ref.get("representation_floor", 0.0) or 0.0
    cold_eq = os.path.join(case_dir, "equilibrium-cold")
    if not floor and os.path.exists(cold_eq + ".json"):
        # the representation floor: r/L of the oracle's own equilibrium rounded to f32 (the f32 state files hold no
        # better), as the reference records it beside its cold solve
        xr = _state(cold_eq).astype(np.float32).astype(np.float64)
        floor = float(np.linalg.norm(oracle.static_gradient(xr)) / oracle.gravity_load)
    details["representation_floor"] = floor
    verdict["final_state_residual_ok"] = r_over_l <= max(RESIDUAL_FLOOR_ALLOWANCE, FLOOR_FACTOR * floor)
    if start is not None:
        x0 = _state(start)
        d0 = float(distances(colliders, x0)[free].min() / dhat)
        details["start_residual_over_load"] = float(np.linalg.norm(oracle.static_gradient(x0)) / oracle.gravity_load)
        details["start_min_distance_over_dhat"] = d0
        verdict["start_feasible"] = d0 > 0
    if os.path.exists(cold_eq + ".json"):
        xc = _state(cold_eq)
        e_c = oracle.static_energy(xc)
        details["energy_gap_over_cold"] = float((oracle.static_energy(final) - e_c) / abs(e_c))
        side = np.ptp(arr["rest_positions"].astype(np.float64).reshape(-1, 3)[:, 0])
        details["max_vertex_gap_over_side"] = float(np.linalg.norm((final - xc).reshape(-1, 3), axis=1).max() / side)
    return verdict, details


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--dir", required=True)
    ap.add_argument("--mode", default="cold")
    ap.add_argument("--start", default=None, help="start state prefix of a warm or prolong run")
    args = ap.parse_args(argv)
    problem = json.load(open(os.path.join(args.dir, "problem.json")))
    n = int(problem["grid_columns"])
    oracle = oracle_py.Scene("reference", n, edit=problem.get("edit", "base"))
    verdict, details = compare(args.dir, args.mode, oracle, args.start)
    out = {"verdict": verdict, "schema": "e7-result/1", "case": problem.get("case"), "mode": args.mode, **details}
    with open(os.path.join(args.dir, f"gpu-{args.mode}", "result.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(json.dumps(out))
    return 0 if all(verdict.values()) else 1


if __name__ == "__main__":
    raise SystemExit(main())
