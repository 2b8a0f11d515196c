"""The cluster tail of the V-cycle (tail3_kernel: the last three levels n17, n9, n5 in one 8-CTA cluster), restated
in f64 numpy on the CPU with the kernel's own decomposition: each of the eight ranks owns a contiguous slice of the
n17 rows (<= 37) and of the n9 rows (<= 11), computes only its own rows, and reads other ranks' rows of the vectors
that cross slices (t_17, z_9, t_9, e_9) from their slices, as the kernel does through distributed shared memory.
The restatement equals the recursive V-cycle (multilevel_ref.Hierarchy.vcycle) on those three levels, so the
slicing, the ownership map and the order of the five exchange steps lose no row and use no stale value."""
import numpy as np

from tests import multilevel_ref as ml
from tests import oracle_py

RANKS = 8
N3, N4, N5 = 17, 9, 5


def _system(seed=3):
    sc = oracle_py.Scene("sheet", N3, seed=seed, plane=True, projected=True)
    rp, ci = sc.pattern()
    x = sc.contact_state()
    h = 0.05
    x_hat = x + h * h * np.tile(sc.gravity, sc.V)
    _, vals = sc.assemble(x, x_hat, h, 0.0, curvature=False)
    return ml.bsr_matrix(rp, ci, vals)


def _stencil_rows(A, n):
    """[rows][25][3][3] blocks of an n x n grid operator with couplings at most two steps away, as 5 x 5 stencils
    (the device's coarse layout; zero outside the grid)."""
    A = A.tocsr()
    out = np.zeros((n * n, 25, 3, 3))
    for I in range(n * n):
        for o, J in _neighbours(n, I):
            out[I, o] = A[3 * I:3 * I + 3, 3 * J:3 * J + 3].toarray()
    return out


def _neighbours(n, I):
    X, Y = I % n, I // n
    for o in range(25):
        dx, dy = o % 5 - 2, o // 5 - 2
        x, y = X + dx, Y + dy
        if 0 <= x < n and 0 <= y < n:
            yield o, y * n + x


def _support(nc, nf, I):
    X, Y = I % nc, I // nc
    for s in range(9):
        ax, by = s % 3 - 1, s // 3 - 1
        fx, fy = 2 * X + ax, 2 * Y + by
        if 0 <= fx < nf and 0 <= fy < nf:
            yield (0.5 if ax else 1.0) * (0.5 if by else 1.0), fy * nf + fx


def _interpolate(e, nc, x, y):
    X0, Y0 = x >> 1, y >> 1
    w = (0.5 if x & 1 else 1.0) * (0.5 if y & 1 else 1.0)
    out = np.zeros(3)
    for b in range(2 if y & 1 else 1):
        for a in range(2 if x & 1 else 1):
            out += w * e[(Y0 + b) * nc + X0 + a]
    return out


def _slices(rows):
    per = (rows + RANKS - 1) // RANKS
    return per, [range(k * per, min(rows, (k + 1) * per)) for k in range(RANKS)]


def cluster_tail(H, r3, z3):
    """e_17 from r_17 and z_17 = S_17 r_17, computed rank by rank with the kernel's slices and exchange steps."""
    A3, A4 = _stencil_rows(H.A[0], N3), _stencil_rows(H.A[1], N4)
    S3, S4 = H.S[0], H.S[1]  # [rows][3][3]
    inv = H.coarse_inv
    per3, sl3 = _slices(N3 * N3)
    per4, sl4 = _slices(N4 * N4)
    r3, z3 = r3.reshape(-1, 3), z3.reshape(-1, 3)
    own3 = [np.zeros((per3, 3)) for _ in range(RANKS)]  # t_17 slices, later e_17
    r4s, z4s, t4s, e4s = ([np.zeros((per4, 3)) for _ in range(RANKS)] for _ in range(4))
    # t_17 = r_17 - A_17 z_17, own rows                                          | sync
    for k in range(RANKS):
        for i in sl3[k]:
            own3[k][i - k * per3] = r3[i] - sum(A3[i, o] @ z3[j] for o, j in _neighbours(N3, i))
    remote3 = lambda j: own3[j // per3][j % per3]
    # r_9 = P^T t_17, z_9 = S_9 r_9, own rows                                     | sync
    for k in range(RANKS):
        for I in sl4[k]:
            t = sum(w * remote3(j) for w, j in _support(N4, N3, I))
            r4s[k][I - k * per4], z4s[k][I - k * per4] = t, S4[I] @ t
    z4 = lambda J: z4s[J // per4][J % per4]
    # t_9 = r_9 - A_9 z_9, own rows                                              | sync
    for k in range(RANKS):
        for I in sl4[k]:
            t4s[k][I - k * per4] = r4s[k][I - k * per4] - sum(A4[I, o] @ z4(J) for o, J in _neighbours(N4, I))
    t4_all = np.array([t4s[J // per4][J % per4] for J in range(N4 * N4)])
    # every rank: r_5 = P^T t_9, e_5 = A_5^{-1} r_5; then e_9 on its own rows      | sync
    r5 = np.array([sum(w * t4_all[J] for w, J in _support(N5, N4, K)) for K in range(N5 * N5)])
    e5 = (inv @ r5.reshape(-1)).reshape(-1, 3)
    for k in range(RANKS):
        for I in sl4[k]:
            y = lambda J: z4(J) + _interpolate(e5, N5, J % N4, J // N4)
            d = r4s[k][I - k * per4] - sum(A4[I, o] @ y(J) for o, J in _neighbours(N4, I))
            e4s[k][I - k * per4] = y(I) + S4[I].T @ d
    e4_all = np.array([e4s[J // per4][J % per4] for J in range(N4 * N4)])  # | sync
    # e_17 = y_17 + S_17^T (r_17 - A_17 y_17), own rows
    e3 = np.zeros((N3 * N3, 3))
    for k in range(RANKS):
        for i in sl3[k]:
            y = lambda j: z3[j] + _interpolate(e4_all, N4, j % N3, j // N3)
            d = r3[i] - sum(A3[i, o] @ y(j) for o, j in _neighbours(N3, i))
            e3[i] = y(i) + S3[i].T @ d
    return e3.reshape(-1)


def test_slices_cover_every_row_once():
    for rows in (N3 * N3, N4 * N4):
        per, sl = _slices(rows)
        assert sorted(i for s in sl for i in s) == list(range(rows))
        assert all(len(s) <= per for s in sl)
    assert _slices(N3 * N3)[0] == 37 and _slices(N4 * N4)[0] == 11


def test_cluster_tail_equals_the_recursive_cycle():
    A = _system()
    H = ml.Hierarchy(A, N3)
    assert H.cols == [N3, N4, N5]
    r = np.random.default_rng(1).standard_normal(3 * N3 * N3)
    z = ml.block_apply(H.S[0], r)
    e = cluster_tail(H, r, z)
    ref = H.vcycle(r)
    assert np.linalg.norm(e - ref) <= 1e-12 * np.linalg.norm(ref), np.linalg.norm(e - ref) / np.linalg.norm(ref)
