"""The smoothed prolongation of the numpy restatement (multilevel_ref.smoothed_prolongation), on the CPU: with no
smoothing it is the device's bilinear prolongation, the level-1 operator it gives fits a 7 x 7 stencil (the layout a
device form needs), and the V-cycle with it needs fewer flexible-PCG iterations than the bilinear one."""
import numpy as np

from tests import multilevel_ref as ml
from tests import oracle_py

N = 17


def _system(n=N, seed=3):
    sc = oracle_py.Scene("sheet", n, seed=seed, plane=True, projected=True)
    rp, ci = sc.pattern()
    x = sc.kernel_state() - 0.06 * np.tile(sc.gravity / np.linalg.norm(sc.gravity), sc.V)
    h = 0.01
    _, vals = sc.assemble(x, x + h * h * np.tile(sc.gravity, sc.V), h, 0.0, curvature=False)
    return ml.bsr_matrix(rp, ci, vals)


def test_no_smoothing_is_the_bilinear_prolongation():
    A = _system()
    P = ml.prolongation(N)
    assert abs(ml.smoothed_prolongation(A, P, 0, c=0.0) - P).max() == 0.0


def test_level_one_operator_fits_a_seven_by_seven_stencil():
    """Entries two coarse steps out and beyond come only from the weak axial hinge couplings: the ring at three
    steps is small but not negligible (~1e-5 of the largest entry), the ring at four is at rounding level."""
    A = _system()
    H = ml.Hierarchy(A, N, smooth_prolongation=(0,))
    nc = H.cols[1]
    C = H.A[1].tocoo()
    i, j = C.row // 3, C.col // 3
    radius = np.maximum(np.abs(i % nc - j % nc), np.abs(i // nc - j // nc))
    big = np.abs(C.data).max()
    assert radius.max() <= 4
    assert 1e-8 * big < np.abs(C.data[radius == 3]).max() < 1e-4 * big
    assert np.abs(C.data[radius == 4]).max(initial=0.0) < 1e-10 * big
    # the bilinear hierarchy's level 1 stays within 5 x 5
    B = ml.Hierarchy(A, N).A[1].tocoo()
    bi, bj = B.row // 3, B.col // 3
    assert np.abs(bi % nc - bj % nc).max() <= 2 and np.abs(bi // nc - bj // nc).max() <= 2


def test_smoothed_prolongation_needs_fewer_iterations():
    A = _system()
    b = np.random.default_rng(99).standard_normal(A.shape[0])
    _, k_bilinear, s1 = ml.flexible_pcg(A, b, ml.Hierarchy(A, N).vcycle, 1e-6, 1000)
    _, k_smoothed, s2 = ml.flexible_pcg(A, b, ml.Hierarchy(A, N, smooth_prolongation=(0,)).vcycle, 1e-6, 1000)
    assert s1 == s2 == "converged"
    assert k_smoothed < k_bilinear, (k_smoothed, k_bilinear)
