"""f64 numpy restatement of the multilevel V-cycle preconditioner (drape_b200/csrc/mg.h, mg.cu), the checker of
the CUDA hierarchy and cycle. The preconditioner has no counterpart in the reference (its direction solver is
block-Jacobi PCG, engine/oracle/src/pcg.rs:37-281), so this restatement of the build's own algorithm is what the
GPU is compared against.

Hierarchy: n x n vertex grid, vertex = y * n + x, 3 unknowns per vertex; coarse grid (n - 1) / 2 + 1; bilinear
prolongation per component; Galerkin products P^T A P; omega * D^{-1} smoothing (pre S, post S^T); exact solve at
the coarsest level (n <= 5).
"""
import numpy as np
import scipy.sparse as sp

STENCIL = [(dx, dy) for dy in range(-2, 3) for dx in range(-2, 3)]  # offset o = (dy + 2) * 5 + dx + 2


def level_columns(n):
    cols = [n]
    while cols[-1] > 5 and (cols[-1] - 1) % 2 == 0:
        cols.append((cols[-1] - 1) // 2 + 1)
    return cols if cols[-1] <= 5 and len(cols) > 1 else [n]


def _weights_1d(n):
    """(fine index, coarse index, weight) triples of the 1D bilinear prolongation."""
    f = np.arange(n)
    even = f % 2 == 0
    fi = np.concatenate([f[even], f[~even], f[~even]])
    ci = np.concatenate([f[even] // 2, f[~even] // 2, f[~even] // 2 + 1])
    w = np.concatenate([np.ones(even.sum()), np.full((~even).sum(), 0.5), np.full((~even).sum(), 0.5)])
    return fi, ci, w


def prolongation(n):
    """P: (3 n^2) x (3 nc^2), bilinear per displacement component."""
    nc = (n - 1) // 2 + 1
    fi, ci, w = _weights_1d(n)
    fx, fy = np.meshgrid(np.arange(len(fi)), np.arange(len(fi)), indexing="xy")
    fx, fy = fx.ravel(), fy.ravel()
    rows = fi[fy] * n + fi[fx]
    cols = ci[fy] * nc + ci[fx]
    vals = w[fy] * w[fx]
    R = np.concatenate([3 * rows + c for c in range(3)])
    C = np.concatenate([3 * cols + c for c in range(3)])
    V = np.concatenate([vals] * 3)
    return sp.csr_matrix((V, (R, C)), shape=(3 * n * n, 3 * nc * nc))


def bsr_matrix(row_ptr, col_idx, blocks):
    """f64 CSR of the BSR(3x3) matrix with 9B row-major blocks."""
    R = len(row_ptr) - 1
    return sp.bsr_matrix((np.asarray(blocks, np.float64).reshape(-1, 3, 3), np.asarray(col_idx),
                          np.asarray(row_ptr)), shape=(3 * R, 3 * R)).tocsr()


def diagonal_blocks(A):
    R = A.shape[0] // 3
    D = np.zeros((R, 3, 3))
    C = A.tocoo()
    m = (C.row // 3) == (C.col // 3)
    D[C.row[m] // 3, C.row[m] % 3, C.col[m] % 3] = C.data[m]
    return D


def jacobi_smoother(A, omega):
    """[R, 3, 3] blocks omega * D^{-1} (zero where D is singular)."""
    D = diagonal_blocks(A)
    det = np.linalg.det(D)
    out = np.zeros_like(D)
    ok = np.isfinite(det) & (det != 0)
    out[ok] = omega * np.linalg.inv(D[ok])
    return out


POWER_STEPS = 10


def hash_unit(x):
    """The device's start-vector hash: uint32 index -> uniform [-1, 1)."""
    x = np.asarray(x, np.uint64) & 0xFFFFFFFF
    x ^= x >> 16
    x = (x * 0x7FEB352D) & 0xFFFFFFFF
    x ^= x >> 15
    x = (x * 0x846CA68B) & 0xFFFFFFFF
    x ^= x >> 16
    return (x & 0xFFFFFF).astype(np.float64) * (2.0 / 16777216.0) - 1.0


def spectral_omega(A, level):
    """omega = 2 / (1.1 lambda (1 + 1/30)), lambda = |D^{-1} A v| after POWER_STEPS power steps from the hashed
    start vector (the first step unnormalised, as on the device)."""
    R = A.shape[0] // 3
    Dinv = jacobi_smoother(A, 1.0)
    h = 3 * np.arange(R, dtype=np.uint64) + 7919 * level
    v = np.stack([hash_unit(h), hash_unit(h + 1), hash_unit(h + 2)], axis=1).reshape(-1)
    w = None
    for k in range(POWER_STEPS):
        if k > 0:
            v = w / np.linalg.norm(w)
        w = block_apply(Dinv, A @ v)
    lam = np.linalg.norm(w)
    return 2.0 / (1.1 * lam * (1.0 + 1.0 / 30.0))


def block_apply(S, r, transpose=False):
    r3 = r.reshape(-1, 3)
    return (np.einsum("kji,kj->ki" if transpose else "kij,kj->ki", S, r3)).reshape(-1)


def smoothed_prolongation(A, P, level, c=4.0 / 3.0):
    """(I - omega_P D^{-1} A) P with omega_P = c / lambda, lambda the spectral estimate of lambda_max(D^{-1} A) that
    spectral_omega uses (the prolongation smoothing of smoothed aggregation: Vanek, Mandel and Brezina, Computing
    56 (1996), with its omega_P = 4 / (3 lambda)). A candidate coarse space, checked on the host ahead of a device
    form."""
    lam = 2.0 / (spectral_omega(A, level) * 1.1 * (1.0 + 1.0 / 30.0))
    Dinv = jacobi_smoother(A, 1.0)
    R = A.shape[0] // 3
    Dm = sp.bsr_matrix((Dinv, np.arange(R), np.arange(R + 1)), shape=A.shape).tocsr()
    return (P - (c / lam) * (Dm @ (A @ P))).tocsr()


def chebyshev_interval(omega):
    """[lo, hi] of D^{-1} A that the spectral omega damps as degree-1 Chebyshev: omega = 2 / (lo + hi) with
    hi = 1.1 lambda and lo = hi / 30."""
    hi = 2.0 / (omega * (1.0 + 1.0 / 30.0))
    return hi / 30.0, hi


def chebyshev_apply(A, Dinv, r, lo, hi, degree):
    """z = p(D^{-1} A) D^{-1} r: `degree` steps of block-Jacobi preconditioned Chebyshev iteration for A z = r from
    z = 0 on the interval [lo, hi] (the three-term recurrence of Saad, Iterative Methods for Sparse Linear Systems,
    2nd ed., Algorithm 12.1). Degree 1 is omega D^{-1} r with omega = 2 / (lo + hi); each further degree costs one
    SpMV with A. A candidate fine smoother, checked here on the host ahead of a device kernel."""
    theta, delta = 0.5 * (hi + lo), 0.5 * (hi - lo)
    sigma = theta / delta
    rho = 1.0 / sigma
    d = block_apply(Dinv, r) / theta
    z = d.copy()
    res = r.copy()
    for _ in range(degree - 1):
        res = res - A @ d
        rho_next = 1.0 / (2.0 * sigma - rho)
        d = rho_next * rho * d + (2.0 * rho_next / delta) * block_apply(Dinv, res)
        rho = rho_next
        z = z + d
    return z


def truncate_stencil(A, n, radius):
    """A coarse operator on an n x n grid with every block coupling vertices more than `radius` grid steps apart
    (in either axis) dropped."""
    C = A.tocoo()
    i, j = C.row // 3, C.col // 3
    keep = (np.abs(i % n - j % n) <= radius) & (np.abs(i // n - j // n) <= radius)
    return sp.csr_matrix((C.data[keep], (C.row[keep], C.col[keep])), shape=A.shape)


class Hierarchy:
    """omega > 0: fixed damping on every level; omega = None: spectral_omega per level (the device default)."""

    def __init__(self, A, n, omega=None, fine_smoother=None, smooth_prolongation=(), truncate=None):
        """smooth_prolongation: levels whose prolongation is smoothed once (smoothed_prolongation), () for the
        bilinear one everywhere. truncate: the coarse operator below a smoothed prolongation keeps only the
        couplings within this many coarse steps (the device: smooth_prolongation=(0,), truncate=3, level 1 a 7 x 7
        stencil); None keeps the whole product."""
        self.cols = level_columns(n)
        if len(self.cols) < 2:
            raise ValueError("grid cannot be coarsened")
        self.A = [A.tocsr()]
        self.P = []
        self.width = [0]
        for l in range(len(self.cols) - 1):
            P = prolongation(self.cols[l])
            wide = l in smooth_prolongation
            if wide:
                P = smoothed_prolongation(self.A[-1], P, l)
            self.P.append(P)
            C = (P.T @ self.A[-1] @ P).tocsr()
            if wide and truncate is not None:
                C = truncate_stencil(C, self.cols[l + 1], truncate)
            self.A.append(C)
            self.width.append(2 * truncate + 1 if wide and truncate is not None else 5)
        self.omega = [omega if omega else spectral_omega(Al, l) for l, Al in enumerate(self.A[:-1])]
        self.S = [jacobi_smoother(Al, w) for Al, w in zip(self.A[:-1], self.omega)]
        if fine_smoother is not None:
            self.S[0] = fine_smoother
        self.coarse_inv = np.linalg.inv(self.A[-1].toarray())

    def vcycle(self, r, level=0):
        if level == len(self.A) - 1:
            return self.coarse_inv @ r
        A, S, P = self.A[level], self.S[level], self.P[level]
        z = block_apply(S, r)
        y = z + P @ self.vcycle(P.T @ (r - A @ z), level + 1)
        return y + block_apply(S, r - A @ y, transpose=True)

    def stencil(self, level):
        """Level operator as the GPU's [w^2 * 9][rows] stencil array (w = self.width[level])."""
        n = self.cols[level]
        A = self.A[level]
        rows = n * n
        w = self.width[level]
        h = w // 2
        offsets = [(dx, dy) for dy in range(-h, h + 1) for dx in range(-h, h + 1)]
        out = np.zeros((w * w * 9, rows))
        Ad = A.tocsr()
        for o, (dx, dy) in enumerate(offsets):
            X, Y = np.meshgrid(np.arange(n), np.arange(n), indexing="xy")
            X, Y = X.ravel(), Y.ravel()
            ok = (X + dx >= 0) & (X + dx < n) & (Y + dy >= 0) & (Y + dy < n)
            I = (Y * n + X)[ok]
            J = ((Y + dy) * n + X + dx)[ok]
            for e in range(9):
                a, b = divmod(e, 3)
                out[o * 9 + e, I] = np.asarray(Ad[3 * I + a, 3 * J + b]).ravel()
        return out


def flexible_pcg(A, b, M, tol, maxit):
    """Flexible CG with the Polak-Ribiere beta (the GPU's recurrence), f64."""
    x = np.zeros_like(b)
    r = b.copy()
    rr0 = r @ r
    z = M(r)
    p = z.copy()
    rz = z @ r
    r_prev = None
    for k in range(maxit):
        if k > 0:
            z = M(r)
            beta = (z @ r - z @ r_prev) / rz
            rz = z @ r
            p = z + beta * p
        q = A @ p
        pq = p @ q
        if not pq > 0:
            return x, k, "breakdown"
        alpha = rz / pq
        x = x + alpha * p
        r_prev = r
        r = r - alpha * q
        if r @ r <= tol * tol * rr0:
            return x, k + 1, "converged"
    return x, maxit, "limit"
