"""The preconditioner network's numpy oracle (tests/network_ref.py) checked on its own, on the CPU: its analytic
gradient through the V-cycle and the network against central finite differences (f64, no bf16 rounding), the
untrained network's factors (exactly 1), the bf16 rounding helper, and the shipped weights' factors (below 1, the
V-cycle with them positive definite)."""
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


def test_untrained_network_stays_just_below_the_spectral_smoother():
    """A zero output layer gives o = 0: f = 0.8 + 0.2 sigmoid(0) = 0.9 on every row, and no input reaches 1."""
    rp, ci, blocks, b, sol = _tuple()
    p = nr.init_params(3, scale_out=0.0)
    _, _, f = nr.network_loss(p, rp, ci, blocks, 9, b, sol, grad=False)
    assert np.abs(f - 0.9).max() <= 1e-6
    p = nr.init_params(3, scale_out=50.0)
    _, _, f = nr.network_loss(p, rp, ci, blocks, 9, b, sol, grad=False)
    assert f.max() <= 1.0 + 1e-7 and f.min() >= 0.8 - 1e-7  # (0.8, 1) up to the f32 sum 0.8f + 0.2f


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 65504.0], np.float32)
    r = nr.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == np.float32(1.0078125)
    assert abs(r[3] + 3.140625) < 1e-6 and r[4] == 65536.0


def test_shipped_network_keeps_the_cycle_positive_definite():
    """The shipped weights (drape_b200/preconditioner_network.bin: 8-byte magic, int32 count, f32 parameters) give
    factors below 1 on a held-out kernel-state system, and the V-cycle with them keeps every eigenvalue of M A
    positive, as flexible PCG needs."""
    import os

    path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "drape_b200",
                        "preconditioner_network.bin")
    raw = open(path, "rb").read()
    assert raw[:8] == b"DRAPENN1" and int(np.frombuffer(raw[8:12], np.int32)[0]) == nr.N_PARAMS
    params = np.frombuffer(raw[12:], np.float32).astype(np.float64)
    n = 17
    sc = oracle_py.Scene("sheet", n, seed=0, plane=True, projected=True)
    rp, ci = sc.pattern()
    x = sc.kernel_state() - 0.06 * np.tile(sc.gravity / np.linalg.norm(sc.gravity), sc.V)
    h = 0.01
    _, vals = sc.assemble(x, x + h * h * np.tile(sc.gravity, sc.V), h, 0.0, curvature=False)
    blocks = vals.astype(np.float32)
    A = ml.bsr_matrix(rp, ci, blocks)
    Hh = ml.Hierarchy(A, n)
    feat, w = nr.features(rp, ci, blocks, Hh.omega[0])
    _, _, f = nr.forward(params, feat, rp, ci, w, True)
    assert 0.5 < f.min() and f.max() < 1.0
    Hh.S[0] = f[:, None, None] * Hh.S[0]
    M = np.stack([Hh.vcycle(e) for e in np.eye(A.shape[0])], axis=1)
    lam = np.linalg.eigvals(M @ A.toarray())
    assert lam.real.min() > 0.0 and np.abs(lam.imag).max() < 1e-8
