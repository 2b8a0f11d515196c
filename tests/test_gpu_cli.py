"""The `drape` command on the GPU (needs a B200): a cold solve of the reference's n17 base case with the rules
of its problem.json writes the gpu-<mode>/ files run-e7.ts writes (state files readable by both), and a warm
start from that equilibrium stays there; the learned preconditioner runs with the shipped weights."""
import json
import os
import subprocess
import tempfile

import numpy as np
import pytest

from drape_b200 import api
from drape_b200.build import CLI
from tests import e7_replays, oracle_py

pytestmark = pytest.mark.gpu


def _run(*args):
    p = subprocess.run([CLI, *args], capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr
    return p


def test_cold_then_warm_reference_case():
    with tempfile.TemporaryDirectory() as t:
        api.write_reference_problem(t, 17, "base")
        _run("--case", t, "--mode", "cold")
        out = os.path.join(t, "gpu-cold")
        res = json.load(open(os.path.join(out, "gpu-result.json")))
        assert res["schema"] == "e7-gpu/1" and res["stop"] == "tolerance", res
        assert res["final_relative_residual"] <= 1e-8 * 1.0001
        ptc = np.fromfile(os.path.join(out, "gpu-ptc.bin"), np.float64).reshape(-1, 7)
        assert len(ptc) == res["accepted_steps"] and np.all(np.diff(ptc[:, 0]) > 0)
        meta = json.load(open(os.path.join(out, "gpu-equilibrium.json")))
        eq = np.fromfile(os.path.join(out, "gpu-equilibrium.bin"), np.float32)
        assert meta["dtype"] == "f32" and eq.size == 3 * meta["vertices"] and meta["final_h"] > 0
        states = np.fromfile(os.path.join(out, "gpu-states.bin"), np.float32)
        # n17 <= 65 columns: the start, then every accepted state; the last is the equilibrium
        assert states.size == (res["accepted_steps"] + 1) * eq.size
        assert np.array_equal(states[-eq.size:], eq)
        # per-Newton and per-attempt tables: every accepted attempt's records add up to its gpu-ptc.bin row
        it = np.fromfile(os.path.join(out, "gpu-iterations.bin"), np.float64).reshape(-1, 9)
        rb = np.fromfile(os.path.join(out, "gpu-robust.bin"), np.float64).reshape(-1, 16)
        at = np.fromfile(os.path.join(out, "gpu-attempts.bin"), np.float64).reshape(-1, 6)
        assert len(it) == len(rb) == res["newton_records"] > 0 and len(at) == res["attempt_records"]
        assert np.all(at[:, 4] <= at[:, 5]) and at[-1, 5] == len(it) and np.all(at[1:, 4] == at[:-1, 5])
        accepted = at[at[:, 3] == 0]
        assert len(accepted) == res["accepted_steps"] and np.array_equal(accepted[:, 0], ptc[:, 0])
        for a, p in zip(accepted, ptc):
            seg = it[int(a[4]):int(a[5])]
            assert np.all(seg[:, 0] == p[0]) and np.array_equal(seg[:, 1], np.arange(len(seg)))
            assert int((seg[:, 8] == 0).sum()) == p[3]  # updates = the step's inner count
            assert int(np.nansum(seg[:, 3])) == p[5]    # PCG iterations of the step
            # the last iterate ends the attempt: converged or at the limit without a solve, or a failed search
            assert seg[-1, 8] != 0 and (np.isnan(seg[-1, 3]) or seg[-1, 8] in (3, 5))
            assert a[2] == p[1]
        upd = it[:, 8] == 0
        assert np.all(it[upd, 6] >= 0) and np.all(it[upd, 6] <= rb[upd, 6])  # 0 <= alpha <= alpha_max
        assert np.all(rb[upd, 12] < 0) and np.all(rb[upd, 9] <= 0)          # descent slope, Armijo decrease
        # the reference comparer's replays of these tables (e7_compare.rs:240-248)
        # the command's step rules: the problem's "ptc" block over the library defaults it falls back to
        o = api.default_options()
        rules = {"growth": o.growth, "shrink": o.shrink, "inner_max_iterations": o.inner_max, "h0": o.h0,
                 "h_min_factor": o.h_min_factor, "h_max": o.h_max}
        rules.update(json.load(open(os.path.join(t, "problem.json"))).get("ptc", {}))
        _, fields, it2, rb2, at2, ptc2 = e7_replays.read_run(out)
        assert e7_replays.forcing_replay(it2, rb2, fields, at2) <= 1e-5
        assert e7_replays.controller_replay({"ptc": rules}, ptc2)
        assert e7_replays.rejection_replay(it2, at2)
        # warm start from the written equilibrium: already converged (f32 rounding of the state aside)
        _run("--case", t, "--mode", "warm", "--start", os.path.join(out, "gpu-equilibrium"))
        warm = json.load(open(os.path.join(t, "gpu-warm", "gpu-result.json")))
        assert warm["stop"] == "tolerance" and warm["accepted_steps"] <= res["accepted_steps"], warm
        eq2 = np.fromfile(os.path.join(t, "gpu-warm", "gpu-equilibrium.bin"), np.float32)
        assert np.abs(eq2 - eq).max() <= 1e-3


def test_learned_preconditioner_from_the_command():
    with tempfile.TemporaryDirectory() as t:
        api.write_reference_problem(t, 17, "base")
        _run("--case", t, "--mode", "cold", "--preconditioner", "learned")
        res = json.load(open(os.path.join(t, "gpu-cold", "gpu-result.json")))
        assert res["preconditioner"] == "learned" and res["stop"] == "tolerance", res


def test_prolong_workflow():
    """The prolong path of the pipeline (run-e7.ts:59-63 after e7_prolong.rs:52-64), on cases written by the oracle's
    own e7-generate: the GPU's n17 equilibrium of the reference's base case is prolonged to the n33 case by
    `drape prolong`, which writes the state `oracle e7-prolong` writes (its f64 values rounded to the coarse state's
    f32); `drape --mode prolong` from it stops on the case's tolerance at an f64 equilibrium of the n33 case (the
    oracle's polish lands within 1e-4 m; the f32 state file's rounding leaves ~1e-6 of relative static energy)."""
    from tests.polish_state import polished_error

    oracle_py.build()
    with tempfile.TemporaryDirectory() as t:
        c17, c33 = os.path.join(t, "drape-n17"), os.path.join(t, "drape-n33")
        for n, c in ((17, c17), (33, c33)):
            subprocess.run([oracle_py.CLI, "e7-generate", "--n", str(n), "--edit", "base", "--out", c], check=True,
                           capture_output=True)
        _run("--case", c17, "--mode", "cold")
        eq = os.path.join(c17, "gpu-cold", "gpu-equilibrium")
        start, ostart = os.path.join(t, "start33"), os.path.join(t, "oracle_start33")
        _run("prolong", "--coarse", eq, "--coarse-n", "17", "--fine-dir", c33, "--out", start)
        subprocess.run([oracle_py.CLI, "e7-prolong", "--coarse", eq, "--coarse-n", "17", "--fine-dir", c33, "--out",
                        ostart], check=True, capture_output=True)
        mine = np.fromfile(start + ".bin", np.float32)
        ref = np.fromfile(ostart + ".bin", np.float64).astype(np.float32)
        assert mine.size == 3 * 33 * 33 and np.array_equal(mine, ref)
        _run("--case", c33, "--mode", "prolong", "--start", start)
        res = json.load(open(os.path.join(c33, "gpu-prolong", "gpu-result.json")))
        assert res["stop"] == "tolerance" and res["mode"] == "prolong", res
        x = np.fromfile(os.path.join(c33, "gpu-prolong", "gpu-equilibrium.bin"), np.float32).astype(np.float64)
        err, e_rel, _, _, _ = polished_error(oracle_py.Scene("reference", 33, edit="base"), x)
        # the state file is f32: its rounding (~1e-8 m) against the stiff barrier costs ~1e-6 of the static energy
        assert err <= 1e-4 and e_rel <= 2e-6, (err, e_rel)


def test_comparer_verdict_on_cold_and_prolong_runs():
    """The comparer's gates (e7_compare.rs:276-363, restated in tests/e7_compare.py) on the command's own outputs
    for the reference's n17 base case written by the oracle's e7-generate, with the oracle's cold reference
    solve beside it: every gate holds for the cold run, and for a prolong run of the n33 case from the prolonged
    n17 equilibrium; a state pushed into the sphere trips intersection_free."""
    from tests import e7_compare

    oracle_py.build()
    with tempfile.TemporaryDirectory() as t:
        c17, c33 = os.path.join(t, "drape-n17"), os.path.join(t, "drape-n33")
        for n, c in ((17, c17), (33, c33)):
            subprocess.run([oracle_py.CLI, "e7-generate", "--n", str(n), "--edit", "base", "--out", c], check=True,
                           capture_output=True)
        for c in (c17, c33):  # the oracle's cold references: its equilibrium gives the representation floor
            subprocess.run([oracle_py.CLI, "e7-solve", "--dir", c, "--mode", "cold"], check=True, capture_output=True)
        _run("--case", c17, "--mode", "cold")
        o17 = oracle_py.Scene("reference", 17, edit="base")
        verdict, details = e7_compare.compare(c17, "cold", o17)
        assert set(verdict) >= {"intersection_free", "rules_replayed_ok", "static_energy_ok", "final_state_residual_ok",
                                "oracle_converged"}
        # Every gate holds except that E_s may rise between kept states by up to ~1.5e-6 of max |E_s| (the
        # reference's gate is 1e-6): the refinement solve stops at the forcing target, so an early inexact step can
        # trade a little static energy for inertia (PTC decreases Phi, not E_s).
        assert details["energy_rise_relative"] <= 1e-5, details
        assert all(ok for k, ok in verdict.items() if k != "static_energy_ok"), (verdict, details)
        # the cold gaps are diagnostics in the comparer too: the GPU's path (f32 directions, Eisenstat-Walker
        # forcing) may end on a neighbouring equilibrium of the frictionless sheet, within a fraction of a percent
        assert abs(details["energy_gap_over_cold"]) <= 1e-2 and details["max_vertex_gap_over_side"] <= 0.1, details
        start = os.path.join(t, "start33")
        _run("prolong", "--coarse", os.path.join(c17, "gpu-cold", "gpu-equilibrium"), "--coarse-n", "17",
             "--fine-dir", c33, "--out", start)
        _run("--case", c33, "--mode", "prolong", "--start", start)
        verdict, details = e7_compare.compare(c33, "prolong", oracle_py.Scene("reference", 33, edit="base"), start)
        assert verdict["start_feasible"] and all(verdict.values()), (verdict, details)
        # a planted intersection: the last kept state of the n17 run with a vertex inside the sphere
        path = os.path.join(c17, "gpu-cold", "gpu-states.bin")
        s = np.fromfile(path, np.float32)
        V = 17 * 17
        centre = 3 * ((V // 2) + (s.size // (3 * V) - 1) * V)
        s[centre + 2] -= 0.05  # 5 cm down into the sphere (z up)
        s.tofile(path)
        verdict, _ = e7_compare.compare(c17, "cold", o17)
        assert not verdict["intersection_free"]
