"""The multilevel preconditioner on the GPU against its f64 numpy restatement (tests/multilevel_ref.py), and the
flexible PCG and full drape solves that use it (needs a B200).

Tolerances: the Galerkin products are f64 sums of the same f32 blocks on both sides (relative 1e-12 of the
level's largest entry); smoother blocks carry the damping of an f32 power method (2e-4); one V-cycle runs in f32 on the GPU
against f64 in numpy (relative L2 1e-3: the cycle amplifies the f32 rounding of its residuals by the spread of the
coarse operator); PCG solutions are judged by their f64 residual, as block-Jacobi ones are.
"""
import numpy as np
import pytest

from drape_b200 import api
from tests import multilevel_ref as ml
from tests import oracle_py

pytestmark = pytest.mark.gpu


def _mid_drape_system(n, steps=30, seed=0):
    """The PTC system after `steps` steps of the n x n sheet drape (over sphere + plane), with the projected
    tangent (clamped stress, Gauss-Newton hinge, no barrier curvature): SPD, so both PCGs must converge. (The exact
    tangent at mu = 0 is indefinite there; both PCGs then report breakdown and the Newton raises mu.)"""
    d = api.Drape.sheet(n, seed=seed, plane=True, options=api.default_options(max_steps=steps))
    log = d.solve_equilibrium(check=False)
    x = d.state
    h = log["final_h"]
    g_dir = np.array([0.0, -9.81, 0.0])
    x_hat = x + h * h * np.tile(g_dir, d.V)
    d.set_options(api.default_options(tangent=1))
    grad, blocks = d.assemble(x, x_hat=x_hat, h=h, mode=0, curvature=False)
    rp, ci = oracle_py.Scene("sheet", n, seed=seed, plane=True).pattern()  # the builder's pattern (test_host.py)
    return d, rp, ci, blocks, grad


@pytest.fixture(scope="module")
def system33():
    d, rp, ci, blocks, grad = _mid_drape_system(33)
    A = ml.bsr_matrix(rp, ci, blocks)
    return d, A, blocks, grad


def _reference(A, n, prolongation):
    """The host hierarchy the device builds: bilinear everywhere (0), or the fine prolongation smoothed once with
    level 1 kept as a 7 x 7 stencil (1)."""
    if prolongation:
        return ml.Hierarchy(A, n, smooth_prolongation=(0,), truncate=3)
    return ml.Hierarchy(A, n)


@pytest.mark.parametrize("prolongation", [0, 1])
def test_hierarchy_matches_galerkin_products(system33, prolongation):
    """Galerkin products: the bilinear ones are f64 sums of the same f32 blocks on both sides (1e-12 of the level's
    largest entry). The smoothed level 1 is formed on the device from Sp = omega_P D^{-1} in f32 and the f32 power
    method's lambda (2e-4, as the smoothers), by the symmetric form sum_k P(k, J) (W_k - Z_k)^T, which equals
    P_0^T A P_0 for the assembled (symmetric up to one f32 rounding) A."""
    d, A, blocks, _ = system33
    d.set_options(api.default_options(preconditioner=1, prolongation=prolongation))
    d.precondition(np.zeros(3 * d.R), blocks=blocks)  # set-up for these blocks
    H = _reference(A, 33, prolongation)
    for level in range(len(H.cols)):
        n, op, sm, w = d.multilevel_view(level, width=True)
        assert n == H.cols[level]
        if level > 0:
            assert w == H.width[level]
            ref = H.stencil(level)
            tol = 1e-12 if prolongation == 0 else 2e-4
            assert np.abs(op - ref).max() <= tol * np.abs(ref).max(), (level, np.abs(op - ref).max() / np.abs(ref).max())
        if level < len(H.cols) - 1:
            ref_s = H.S[level].reshape(-1, 9).T
            # the damping comes from an f32 power method on the device, f64 here
            assert np.abs(sm - ref_s).max() <= 2e-4 * np.abs(ref_s).max(), level


@pytest.mark.parametrize("prolongation", [0, 1])
def test_vcycle_matches_reference(system33, prolongation):
    d, A, blocks, grad = system33
    d.set_options(api.default_options(preconditioner=1, prolongation=prolongation))
    H = _reference(A, 33, prolongation)
    rng = np.random.default_rng(3)
    for r in (-grad, rng.standard_normal(3 * d.R)):
        z = d.precondition(r, blocks=blocks)
        zr = H.vcycle(r)
        assert np.linalg.norm(z - zr) <= 1e-3 * np.linalg.norm(zr), np.linalg.norm(z - zr) / np.linalg.norm(zr)


@pytest.mark.parametrize("n", [65, 129])
def test_vcycle_with_the_cluster_tail_matches_reference(n):
    """n65 and n129 have five and six levels, ending with 33, 17, 9, 5: their last three run in one 8-CTA
    thread-block cluster (tail3_kernel) instead of a restriction, tail_kernel and a prolongation. The cycle still
    matches the f64 one."""
    d, rp, ci, blocks, grad = _mid_drape_system(n, steps=12)
    A = ml.bsr_matrix(rp, ci, blocks)
    d.set_options(api.default_options(preconditioner=1))
    H = _reference(A, n, 0)
    assert [l.shape[0] // 3 for l in H.A][-4:] == [1089, 289, 81, 25]
    rng = np.random.default_rng(4)
    for r in (-grad, rng.standard_normal(3 * d.R)):
        z = d.precondition(r, blocks=blocks)
        zr = H.vcycle(r)
        assert np.linalg.norm(z - zr) <= 1e-3 * np.linalg.norm(zr), np.linalg.norm(z - zr) / np.linalg.norm(zr)


@pytest.mark.parametrize("prolongation", [0, 1])
def test_multilevel_pcg_converges_in_far_fewer_iterations(system33, prolongation):
    d, A, blocks, grad = system33
    b = -grad
    d.set_options(api.default_options(preconditioner=1, prolongation=prolongation))
    # The iteration count against the f64 cycle's at rtol 1e-4: below that the f32 solve approaches its attainable
    # accuracy on this system (its true f64 residual stays near 2e-4 of |b| however far the recursive one falls),
    # where f32 iterations grow beyond the f64 count without saying anything about the cycle.
    H = _reference(A, 33, prolongation)
    x, info = d.pcg(b, 1e-4, 2000, blocks=blocks)
    _, k_ref, st = ml.flexible_pcg(A, b, H.vcycle, 1e-4, 2000)
    assert info["status"] == "converged" and st == "converged", info
    assert abs(info["iterations"] - k_ref) <= 5 + 0.25 * k_ref, (info["iterations"], k_ref)
    x, info = d.pcg(b, 1e-6, 2000, blocks=blocks)
    assert info["status"] == "converged", info
    d.set_options(api.default_options(preconditioner=0))
    xj, jac = d.pcg(b, 1e-6, 20000, blocks=blocks)
    d.set_options(api.default_options(preconditioner=1, prolongation=prolongation))
    assert info["iterations"] * 3 < jac["iterations"], (info, jac)
    # Both stop on the recursive f32 residual; their true f64 residuals sit at the same f32 floor.
    res = np.linalg.norm(b - A @ x) / np.linalg.norm(b)
    res_j = np.linalg.norm(b - A @ xj) / np.linalg.norm(b)
    assert res <= max(10 * res_j, 1e-5), (res, res_j)


def test_multilevel_is_rejected_without_a_structured_grid():
    rp, ci, vals, rhs = oracle_py.linear_case("tension", 17)  # boundary vertices pinned: rows != vertices
    R = len(rp) - 1
    with pytest.raises(RuntimeError):
        api.Drape.from_arrays(np.zeros(3 * (R + 64)), np.arange(R), np.ones(R), rp, ci, columns=17,
                              options=api.default_options(preconditioner=1))


@pytest.mark.parametrize("n", [17, 33])
def test_sheet_solve_with_multilevel_reaches_an_f64_equilibrium(n):
    """The drape solved with the multilevel flexible PCG (smoothed prolongation, the default) lands on an f64
    equilibrium within 1e-4 m (the same bound as the block-Jacobi solve): the converged state does not depend on
    the preconditioner's quality."""
    from tests.test_gpu_parity import _polished_error
    o = api.default_options(equilibrium_absolute=1e-7, preconditioner=1)
    gpu = api.Drape.sheet(n, seed=0, plane=True, options=o)
    log = gpu.solve_equilibrium()
    assert log["reason"] == "tolerance" and log["final_residual"] <= 1e-7, log
    assert log["mg_levels"] >= 3
    oracle = oracle_py.Scene("sheet", n, seed=0, plane=True)
    err, e_rel, r64 = _polished_error(oracle, gpu.state)
    assert r64 <= 1.01e-7, r64
    assert err <= 1e-4, err
    assert e_rel <= 1e-9, e_rel
