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


def _device_form_level_one(A, n, Sp):
    """The device's level-1 product (galerkin_smoothed_kernel), restated row by row in numpy: per coarse row I at
    fine vertex c = 2I, B_i = P(i,I) Id - Sp_i sum_k A_ik P(k,I) over the 7 x 7 window, W = A B over 11 x 11,
    Z = A Sp W over 15 x 15, V = W - Z, A_1[I, J] = sum_k P(k,J) V_k^T for J within 3 of I. Returns [49 * 9][rows]."""
    nc = (n - 1) // 2 + 1
    R = n * n
    Ab = A.tobsr(blocksize=(3, 3))
    rows_of = {}
    for i in range(R):
        s, e = Ab.indptr[i], Ab.indptr[i + 1]
        rows_of[i] = list(zip(Ab.indices[s:e], Ab.data[s:e]))

    def w1(f, C):
        d = f - 2 * C
        return 1.0 if d == 0 else 0.5 if abs(d) == 1 else 0.0

    out = np.zeros((49 * 9, nc * nc))
    for I in range(nc * nc):
        X, Y = I % nc, I // nc
        cx, cy = 2 * X, 2 * Y

        def window(r):
            pts = {}
            for dy in range(-r, r + 1):
                for dx in range(-r, r + 1):
                    fx, fy = cx + dx, cy + dy
                    if 0 <= fx < n and 0 <= fy < n:
                        pts[fy * n + fx] = None
            return pts

        B = {}
        for i in window(3):
            acc = np.zeros((3, 3))
            for j, m in rows_of[i]:
                acc += w1(j % n, X) * w1(j // n, Y) * m
            B[i] = w1(i % n, X) * w1(i // n, Y) * np.eye(3) - Sp[i] @ acc
        W, Yv = {}, {}
        for j in window(5):
            acc = np.zeros((3, 3))
            for k, m in rows_of[j]:
                if k in B:
                    acc += m @ B[k]
            W[j], Yv[j] = acc, Sp[j] @ acc
        V = {}
        for r in window(7):
            acc = np.zeros((3, 3))
            for k, m in rows_of[r]:
                if k in Yv:
                    acc += m @ Yv[k]
            V[r] = W.get(r, np.zeros((3, 3))) - acc
        for o in range(49):
            JX, JY = X + o % 7 - 3, Y + o // 7 - 3
            if not (0 <= JX < nc and 0 <= JY < nc):
                continue
            blk = np.zeros((3, 3))
            for q in range(9):
                kx, ky = 2 * JX + q % 3 - 1, 2 * JY + q // 3 - 1
                if 0 <= kx < n and 0 <= ky < n:
                    blk += w1(kx, JX) * w1(ky, JY) * V[ky * n + kx].T
            out[o * 9:(o + 1) * 9, I] = blk.reshape(-1)
    return out


def test_device_form_of_level_one_is_the_galerkin_product():
    """The row-by-row form the device uses (symmetric A and Sp blocks) gives P_0^T A P_0 truncated to 7 x 7."""
    A = _system()
    A = (0.5 * (A + A.T)).tocsr()  # the form relies on A_ij = A_ji^T; the assembled matrix is symmetric up to f32
    H = ml.Hierarchy(A, N, smooth_prolongation=(0,), truncate=3)
    lam = 2.0 / (ml.spectral_omega(A, 0) * 1.1 * (1.0 + 1.0 / 30.0))
    Sp = ml.jacobi_smoother(A, (4.0 / 3.0) / lam)
    dev = _device_form_level_one(A, N, Sp)
    ref = H.stencil(1)
    assert H.width[1] == 7 and ref.shape == dev.shape
    assert np.abs(dev - ref).max() <= 1e-12 * np.abs(ref).max()


def test_truncated_level_one_keeps_the_gain():
    """Dropping level 1's ring at four coarse steps (rounding-level entries) changes no iteration count."""
    A = _system()
    b = np.random.default_rng(99).standard_normal(A.shape[0])
    _, k_full, _ = ml.flexible_pcg(A, b, ml.Hierarchy(A, N, smooth_prolongation=(0,)).vcycle, 1e-6, 1000)
    _, k_trunc, s = ml.flexible_pcg(A, b, ml.Hierarchy(A, N, smooth_prolongation=(0,), truncate=3).vcycle, 1e-6, 1000)
    assert s == "converged" and abs(k_trunc - k_full) <= 1, (k_trunc, k_full)
