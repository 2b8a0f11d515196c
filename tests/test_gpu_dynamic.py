"""The dynamic drape (backward Euler, drape.rs:403-439 / drape-e4.ts:45-52) on the GPU against the f64 oracle
(needs a B200): the n17 sheet falls from rest onto the sphere at h = 1/240 s, one drape_time_step per step from the
GPU's own previous state and velocity, each step checked against the oracle's step from the same (x, v).

Tolerances: both Newtons stop on their f64 residual |grad Phi| / |grad Phi(x_n)| (GPU 1e-8: f32 PCG directions with
one f64 refinement; oracle 1e-10 with band Cholesky, or its line search's f64 noise floor, below 1e-7 in contact). Phi's
Hessian is at least M/h^2 (~34 N/m per vertex here) and the scale at most ~4 N, so a step's positions agree within
1e-8 m and its velocity within 1e-8 m / h; over the 48 chained steps the two trajectories stay within 1e-6 m."""
import numpy as np
import pytest

from drape_b200 import api
from tests import oracle_py

pytestmark = pytest.mark.gpu
H = 1.0 / 240.0


@pytest.mark.parametrize("preconditioner", [0, 1])
def test_falling_sheet_matches_the_oracle_step_by_step(preconditioner):
    n = 17
    gpu = api.Drape.sheet(n, seed=0, plane=True, options=api.default_options(preconditioner=preconditioner))
    oracle = oracle_py.Scene("sheet", n, seed=0, plane=True)
    x_o, v_o = oracle.start(), np.zeros(3 * oracle.V)
    v = None
    for step in range(48):
        x = gpu.state
        # the oracle's step from the GPU's own (x, v): a per-step comparison
        x1, v1, st = oracle.time_step(x, v, H, tolerance=1e-10)
        assert st["status"] == 1 or st["final_relative_residual"] <= 1e-7, (step, st)
        v, log = gpu.time_step(H, v, tolerance=1e-8, max_iterations=30)
        assert log["status_name"] == "converged", (step, log)
        assert log["final_relative_residual"] <= 1e-8
        assert abs(log["scale"] - st["scale"]) <= 1e-9 * st["scale"], (step, log["scale"], st["scale"])
        xg = gpu.state
        assert np.abs(xg - x1).max() <= 1e-8, (step, np.abs(xg - x1).max())
        assert np.abs(v - v1).max() <= 1e-8 / H, (step, np.abs(v - v1).max())
        assert np.allclose(v, (xg - x) / H, rtol=0, atol=1e-12 / H)
        # the oracle's own trajectory, for the chained comparison
        x_o, v_o, _ = oracle.time_step(x_o, v_o, H, tolerance=1e-10)
    assert np.abs(gpu.state - x_o).max() <= 1e-6, np.abs(gpu.state - x_o).max()
    # the sheet reached the sphere: its centre vertex is within the barrier's reach of the sphere's top (y = 0.25)
    centre = gpu.state.reshape(-1, 3)[(n * n) // 2]
    assert centre[1] < 0.25 + 2e-3, centre
    records = gpu.newton_records()
    assert records and records[-1]["status"] == 1


def test_time_step_rejects_bad_arguments():
    gpu = api.Drape.sheet(9, seed=0, plane=True)
    with pytest.raises(api.DrapeError):
        gpu.time_step(0.0)
    with pytest.raises(api.DrapeError):
        gpu.time_step(H, tolerance=-1.0)
