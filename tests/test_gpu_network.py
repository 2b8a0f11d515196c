"""The preconditioner network on the GPU against its numpy oracle (tests/network_ref.py), its training, and full
solves with the learned preconditioner (needs a B200).

Tolerances: both sides round the dense layers' operands to bf16; the device accumulates in f32 and runs the
V-cycle in f32, the oracle in f64: factors within 2e-3, the loss within 2e-3 relative, the parameter gradient
within 2e-2 relative L2.
"""
import os
import tempfile

import numpy as np
import pytest
import scipy.sparse.linalg as spla

from drape_b200 import api
from tests import multilevel_ref as ml
from tests import network_ref as nr
from tests import oracle_py

pytestmark = pytest.mark.gpu


def _tuple(d, n, seed):
    """(blocks, b, x) of the projected (SPD) PTC system at the drape's current state; x solved in f64."""
    log_h = d.final_h()
    x = d.state
    x_hat = x + log_h * log_h * np.tile([0.0, -9.81, 0.0], d.V)
    d.set_options(api.default_options(tangent=1, prolongation=0))
    g, blocks = d.assemble(x, x_hat=x_hat, h=log_h, mode=0, curvature=False)
    d.set_options(api.default_options(prolongation=0))
    rp, ci = oracle_py.Scene("sheet", n, seed=seed, plane=True).pattern()
    A = ml.bsr_matrix(rp, ci, blocks)
    b = -g
    return blocks, b, spla.spsolve(A.tocsc(), b), rp, ci


def _drape_at(n, steps, seed=0):
    d = api.Drape.sheet(n, seed=seed, plane=True, options=api.default_options(max_steps=steps))
    d.solve_equilibrium(check=False)
    return d


def test_network_gradient_matches_the_oracle():
    d = _drape_at(17, 10)
    blocks, b, x, rp, ci = _tuple(d, 17, 0)
    net = api.Network(seed=1)
    p = nr.init_params(7, scale_out=0.5)
    net.parameters = p
    loss, grad, fac = net.gradient(d, blocks, b, x)
    L, g, f = nr.network_loss(p.astype(np.float64), rp, ci, blocks, 17, b, x, bf=True)
    assert np.ptp(f) > 1e-2
    assert np.abs(fac - f).max() <= 2e-3, np.abs(fac - f).max()
    assert abs(loss - L) <= 2e-3 * L, (loss, L)
    assert np.linalg.norm(grad - g) <= 2e-2 * np.linalg.norm(g), np.linalg.norm(grad - g) / np.linalg.norm(g)


def test_untrained_network_stays_just_below_the_spectral_smoother():
    d = _drape_at(17, 10)
    blocks, b, x, _, _ = _tuple(d, 17, 0)
    net = api.Network(seed=5)
    _, _, fac = net.gradient(d, blocks, b, x)
    assert np.abs(fac - 0.9).max() <= 1e-6  # o = 0: f = 0.9, inside (0.8, 1)


def test_training_lowers_the_vcycle_error():
    """Adam on the GPU lowers the one-cycle A-norm error on random error probes e (b = A e) of three PTC systems
    (the probes carry the high-frequency error the fine smoother acts on)."""
    d = _drape_at(17, 5)
    rng = np.random.default_rng(4)
    tuples = []
    for extra in (0, 10, 25):
        if extra:
            d.set_options(api.default_options(max_steps=extra))
            d.solve_equilibrium(start=d.state, h0=d.final_h(), check=False)
        blocks, _, _, rp, ci = _tuple(d, 17, 0)
        A = ml.bsr_matrix(rp, ci, blocks)
        for _ in range(2):
            e = rng.standard_normal(A.shape[0])
            tuples.append((blocks, A @ e, e))
    net = api.Network(seed=2)
    before = [net.gradient(d, *t)[0] for t in tuples]
    net.train(d, tuples, steps=120, lr=3e-3)
    after = [net.gradient(d, *t)[0] for t in tuples]
    assert np.mean(after) < 0.95 * np.mean(before), (before, after)


def test_network_file_round_trip():
    net = api.Network(seed=3)
    p = nr.init_params(11, scale_out=0.3)
    net.parameters = p
    with tempfile.TemporaryDirectory() as t:
        path = os.path.join(t, "net.bin")
        net.save(path)
        other = api.Network(seed=4, path=path)
        assert np.array_equal(other.parameters, p)


@pytest.mark.parametrize("n", [17, 33])
def test_learned_preconditioner_solve_reaches_an_f64_equilibrium(n):
    """With the learned smoother (the shipped weights when present) the drape lands on an f64 equilibrium within
    1e-4 m, as with block Jacobi: the converged state does not depend on the network."""
    from tests.test_gpu_parity import _polished_error
    net = api.Network.trained() if os.path.exists(api.NETWORK_FILE) else api.Network(seed=0)
    gpu = api.Drape.sheet(n, seed=0, plane=True,
                          options=api.default_options(equilibrium_absolute=1e-7, preconditioner=2))
    gpu.set_network(net)
    log = gpu.solve_equilibrium()
    assert log["reason"] == "tolerance" and log["final_residual"] <= 1e-7, log
    oracle = oracle_py.Scene("sheet", n, seed=0, plane=True)
    err, e_rel, r64 = _polished_error(oracle, gpu.state)
    assert r64 <= 1.01e-7 and err <= 1e-4 and e_rel <= 1e-9, (r64, err, e_rel)


def test_what_the_shipped_network_gains_on_held_out_n129_systems(record_property):
    """The trained network against the identical method without it (the multilevel preconditioner with the
    spectral smoother), on held-out systems of the n129 bench scene (seed 0 is never trained on) at PTC depths 20
    and 80: flexible PCG iterations to rtol 1e-6 and the host time of each solve. The shipped network gains
    nothing on these systems (its factors sit near the lower bound of (0.8, 1), where the iteration count rises a
    little), so the test states that loss and bounds it: both converge and the network costs at most 25 % more
    iterations. The figures are recorded as test properties."""
    import time
    from drape_b200 import train_preconditioner as tp
    net = api.Network.trained()
    d, tuples, _ = tp.drape_tuples(129, 0, 0.25, 5e5, (20, 80), probes=0)
    assert tuples
    out = {}
    for name, pre in (("multilevel", 1), ("learned", 2)):
        d.set_options(api.default_options(preconditioner=pre))
        if pre == 2:
            d.set_network(net)
        its, secs = [], []
        for blocks, b, _ in tuples:
            d.pcg(b, 1e-6, 2000, blocks=blocks)  # warm: hierarchy, graph
            t0 = time.perf_counter()
            _, info = d.pcg(b, 1e-6, 2000, blocks=blocks)
            secs.append(time.perf_counter() - t0)
            assert info["status"] == "converged", (name, info)
            its.append(info["iterations"])
        out[name] = (its, secs)
    gain = [m / l for m, l in zip(out["multilevel"][0], out["learned"][0])]
    record_property("pcg_iterations_multilevel", out["multilevel"][0])
    record_property("pcg_iterations_learned", out["learned"][0])
    record_property("seconds_multilevel", out["multilevel"][1])
    record_property("seconds_learned", out["learned"][1])
    record_property("iteration_gain_multilevel_over_learned", gain)
    assert all(g >= 1 / 1.25 for g in gain), out
