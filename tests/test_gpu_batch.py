"""Concurrent solves of many drapes (drape_solve_batch) against the same drapes solved one at a time (needs a B200).

Each drape keeps its own stream and every reduction of the solve runs in a fixed order (per-CTA partials, no
floating-point atomics), so a drape solved inside a batch, its kernels interleaved with other drapes', must end
bit-identical to the same drape solved alone: the same state and the same step, Newton and PCG counts.
"""
import numpy as np
import pytest

from drape_b200 import api

pytestmark = pytest.mark.gpu

# (columns, seed, sphere radius m, Young's modulus Pa, preconditioner): uneven sizes and materials and all three
# direction solvers (0 block Jacobi, 1 multilevel, 2 learned)
CASES = [(17, 1, 0.20, 3e5, 2), (33, 2, 0.30, 1e6, 2), (17, 3, 0.25, 5e5, 0), (33, 4, 0.18, 2e5, 0),
         (9, 5, 0.30, 1e5, 1), (17, 6, 0.33, 2e6, 1)]
COUNTS = ("reason", "ptc_steps", "newton_iterations", "pcg_iterations", "rejected_attempts", "fallbacks")


def _drapes(net):
    out = []
    for n, seed, radius, young, pre in CASES:
        d = api.Drape.sheet(n, seed=seed, radius=radius, young=young, plane=True,
                            options=api.default_options(preconditioner=pre))
        if pre == 2:
            d.set_network(net)
        out.append(d)
    return out


@pytest.fixture(scope="module")
def net():
    n = api.Network.trained()
    yield n
    n.close()


def test_batch_matches_one_at_a_time(net):
    alone = _drapes(net)
    logs_alone = [d.solve_equilibrium() for d in alone]
    batch = _drapes(net)
    logs, seconds, total = api.solve_batch(batch, workers=4)
    for i, (a, b) in enumerate(zip(alone, batch)):
        assert logs[i]["status"] == 0, i
        assert logs[i]["reason"] == "tolerance", i
        for k in COUNTS:
            assert logs[i][k] == logs_alone[i][k], (i, k)
        assert np.array_equal(a.state, b.state), i
        assert logs[i]["final_residual"] == logs_alone[i]["final_residual"], i
    assert np.all(seconds > 0) and total >= seconds.max()
    for d in alone + batch:
        d.close()


def test_batch_more_workers_than_drapes_and_a_second_batch(net):
    batch = _drapes(net)[:3]
    first, _, _ = api.solve_batch(batch, workers=8)
    states = [d.state for d in batch]
    # a second batch starts from the converged states: every drape is already at its tolerance
    second, _, _ = api.solve_batch(batch, workers=8)
    for i, d in enumerate(batch):
        assert first[i]["status"] == 0 and second[i]["status"] == 0
        assert second[i]["newton_iterations"] == 0
        assert np.array_equal(d.state, states[i])
        d.close()


def test_batch_rejects_a_context_given_twice(net):
    d = _drapes(net)[0]
    with pytest.raises(api.DrapeError) as e:
        api.solve_batch([d, d], workers=2)
    assert e.value.status == 1
    d.close()
