"""The Chebyshev fine smoother of the numpy restatement (multilevel_ref.chebyshev_apply), on the CPU: degree 1 is the
device's spectral damped-Jacobi smoother, the error polynomial keeps the Chebyshev bound on its interval, and a grid
tile plus a halo of 2 (degree - 1) vertices reproduces the global result, which is the data a one-launch kernel
has to read."""
import numpy as np

from tests import multilevel_ref as ml
from tests import oracle_py

N = 17
HALO_PER_SPMV = 2  # the fine matrix couples vertices up to two grid steps apart (hinges across an edge)


def _fine_system(n=N, seed=3):
    sc = oracle_py.Scene("sheet", n, seed=seed, plane=True, projected=True)
    rp, ci = sc.pattern()
    x = sc.kernel_state() - 0.06 * np.tile(sc.gravity / np.linalg.norm(sc.gravity), sc.V)
    h = 0.01
    x_hat = x + h * h * np.tile(sc.gravity, sc.V)
    _, vals = sc.assemble(x, x_hat, h, 0.0, curvature=False)
    A = ml.bsr_matrix(rp, ci, vals)
    r = np.random.default_rng(seed).standard_normal(A.shape[0])
    return rp, ci, A, r


def test_fine_stencil_radius_is_two():
    rp, ci, _, _ = _fine_system()
    rows = np.repeat(np.arange(len(rp) - 1), np.diff(rp))
    ci = np.asarray(ci)
    assert np.abs(ci % N - rows % N).max() == HALO_PER_SPMV
    assert np.abs(ci // N - rows // N).max() == HALO_PER_SPMV


def test_degree_one_is_the_spectral_jacobi_smoother():
    _, _, A, r = _fine_system()
    omega = ml.spectral_omega(A, 0)
    lo, hi = ml.chebyshev_interval(omega)
    Dinv = ml.jacobi_smoother(A, 1.0)
    z = ml.chebyshev_apply(A, Dinv, r, lo, hi, 1)
    ref = ml.block_apply(ml.jacobi_smoother(A, omega), r)
    assert np.allclose(z, ref, rtol=1e-13, atol=0.0)


def test_error_polynomial_keeps_the_chebyshev_bound():
    """On a diagonal test matrix with D = I every eigenvalue of D^{-1} A is known: the error factor
    1 - lambda p(lambda) of degree k stays within 1 / T_k((hi + lo) / (hi - lo)) on [lo, hi]."""
    lam = np.linspace(0.05, 1.0, 300)
    A = np.diag(np.repeat(lam, 3))
    Dinv = np.tile(np.eye(3), (lam.size, 1, 1))
    lo, hi = 0.05, 1.0
    for k in (1, 2, 3, 4):
        e = np.ones(3 * lam.size)
        err = e - ml.chebyshev_apply(A, Dinv, A @ e, lo, hi, k)
        bound = 1.0 / np.cosh(k * np.arccosh((hi + lo) / (hi - lo)))
        assert np.abs(err).max() <= bound * (1 + 1e-12), (k, np.abs(err).max(), bound)
        assert np.abs(err).max() >= 0.999 * bound  # equioscillation: the bound is reached


def _tiled(A, Dinv, r, lo, hi, degree, tile, halo):
    """Each tile evaluated from the rows and columns of its own tile grown by `halo` vertices only."""
    out = np.full_like(r, np.nan)
    X, Y = np.meshgrid(np.arange(N), np.arange(N), indexing="xy")
    X, Y = X.ravel(), Y.ravel()
    for y0 in range(0, N, tile):
        for x0 in range(0, N, tile):
            own = (X >= x0) & (X < x0 + tile) & (Y >= y0) & (Y < y0 + tile)
            ext = (X >= x0 - halo) & (X < x0 + tile + halo) & (Y >= y0 - halo) & (Y < y0 + tile + halo)
            v = np.flatnonzero(ext)
            dof = (3 * v[:, None] + np.arange(3)).ravel()
            z = ml.chebyshev_apply(A[dof][:, dof], Dinv[v], r[dof], lo, hi, degree)
            keep = own[v]
            out[(3 * v[keep][:, None] + np.arange(3)).ravel()] = z.reshape(-1, 3)[keep].ravel()
    return out


def test_tile_with_halo_reproduces_the_global_smoother():
    _, _, A, r = _fine_system()
    lo, hi = ml.chebyshev_interval(ml.spectral_omega(A, 0))
    Dinv = ml.jacobi_smoother(A, 1.0)
    for degree in (2, 3):
        full = ml.chebyshev_apply(A, Dinv, r, lo, hi, degree)
        scale = np.abs(full).max()
        halo = HALO_PER_SPMV * (degree - 1)
        tiled = _tiled(A, Dinv, r, lo, hi, degree, tile=6, halo=halo)
        assert np.abs(tiled - full).max() <= 1e-12 * scale
        # one vertex too few is caught; the two-step couplings are weak hinge terms along the grid axes, so the
        # error it leaves is small (~1e-8 to 1e-5 relative) but far above rounding
        short = _tiled(A, Dinv, r, lo, hi, degree, tile=6, halo=halo - 1)
        assert np.abs(short - full).max() > 1e-9 * scale
