"""Scene generators shared by the batched configuration, its driver and the tests.

batch_scenes: the many-drapes configuration (n drawn from {33, 49, 65, 97, 129}, sphere radius U(0.15, 0.35) m,
E log-uniform in [1e5, 2e6] Pa, master seed 7). sheet_matrix: one sheet's PTC system at its start state.
"""
import tempfile

import numpy as np

from drape_b200 import api

GRAVITY = np.array([0.0, -9.81, 0.0])


def sheet_matrix(n, seed, radius, young):
    """(row_ptr, col_idx, 9B f32 blocks) of the sheet drape's PTC system at its start state (h = 1e-2 s)."""
    d = api.Drape.sheet(n, seed=seed, radius=radius, young=young, plane=True)
    x = d.state
    h = 1e-2
    _, blocks = d.assemble(x, x_hat=x + h * h * np.tile(GRAVITY, d.V), h=h, mode=0)
    with tempfile.TemporaryDirectory() as t:
        api.write_sheet_problem(t, n, seed=seed, radius=radius, young=young, plane=True)
        _, arr = api.read_problem_arrays(t)
    d.close()
    return arr["row_ptr"].astype(np.int64), arr["col_idx"].astype(np.int64), blocks


def batch_scenes(drapes):
    """(columns, seed, sphere radius, E) of the batched configuration's drapes, master seed 7."""
    rng = np.random.default_rng(7)
    out = []
    for _ in range(drapes):
        n = int(rng.choice([33, 49, 65, 97, 129]))
        out.append((n, int(rng.integers(1, 1 << 30)), float(rng.uniform(0.15, 0.35)),
                    float(np.exp(rng.uniform(np.log(1e5), np.log(2e6))))))
    return out
