"""The preconditioner network's numpy oracle (tests/network_ref.py) checked on its own, on the CPU: its analytic
gradient through the V-cycle and the network against central finite differences (f64, no bf16 rounding), the
untrained network's factors (exactly 1), and the bf16 rounding helper."""
import numpy as np
import scipy.sparse.linalg as spla

from tests import multilevel_ref as ml
from tests import network_ref as nr
from tests import oracle_py


def _tuple(n=9, seed=1):
    sc = oracle_py.Scene("sheet", n, seed=seed, plane=True, projected=True)
    rp, ci = sc.pattern()
    x = sc.kernel_state() - 0.06 * np.tile(sc.gravity / np.linalg.norm(sc.gravity), sc.V)
    h = 0.01
    x_hat = x + h * h * np.tile(sc.gravity, sc.V)
    _, vals = sc.assemble(x, x_hat, h, 0.0, curvature=False)
    blocks = vals.astype(np.float32)
    A = ml.bsr_matrix(rp, ci, blocks)
    b = np.random.default_rng(seed).standard_normal(A.shape[0])
    sol = spla.spsolve(A.tocsc(), b)
    return rp, ci, blocks, b, sol


def test_analytic_gradient_matches_finite_differences():
    rp, ci, blocks, b, sol = _tuple()
    p = nr.init_params(7, scale_out=0.5).astype(np.float64)
    L, g, f = nr.network_loss(p, rp, ci, blocks, 9, b, sol, bf=False)
    assert 0.0 < L < 1.0 and np.ptp(f) > 1e-3
    rng = np.random.default_rng(0)
    for _ in range(3):
        d = rng.standard_normal(p.size)
        eps = 1e-6
        lp = nr.network_loss(p + eps * d, rp, ci, blocks, 9, b, sol, bf=False, grad=False)[0]
        lm = nr.network_loss(p - eps * d, rp, ci, blocks, 9, b, sol, bf=False, grad=False)[0]
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g @ d) <= 1e-5 * abs(fd) + 1e-10, (fd, g @ d)


def test_untrained_network_is_the_spectral_smoother():
    rp, ci, blocks, b, sol = _tuple()
    p = nr.init_params(3, scale_out=0.0)
    _, _, f = nr.network_loss(p, rp, ci, blocks, 9, b, sol, grad=False)
    assert np.abs(f - 1.0).max() <= 1e-6


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 65504.0], np.float32)
    r = nr.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == np.float32(1.0078125)
    assert abs(r[3] + 3.140625) < 1e-6 and r[4] == 65536.0
