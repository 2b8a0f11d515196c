"""The single-reduction block-Jacobi PCG of pcg_kernel (Chronopoulos-Gear form), restated in f32 numpy on the CPU
next to the reference's two-reduction iteration (pcg.rs:271-296), on the reference's E1 tension and dynamic
systems: the form the kernel uses (u = M r recomputed from r every iteration, the SpMV applied to u formed one
step from the previous iteration's published M r, M w and M s, and p.A p expanded over five dot products) takes
the same iteration counts as the two-reduction one; carrying u as a recurrence instead stagnates above rtol 1e-7,
which is why the kernel does not."""
import numpy as np
import pytest

from tests import multilevel_ref as ml
from tests import oracle_py

F = np.float32


def _system(kind, n):
    rp, ci, vals, rhs = oracle_py.linear_case(kind, n)
    A = ml.bsr_matrix(rp, ci, vals.astype(F).astype(np.float64)).astype(F).tocsr()
    Dinv = ml.jacobi_smoother(A.astype(np.float64), 1.0).astype(F)
    return A, Dinv, rhs.astype(F)


def _M(Dinv, v):
    return ml.block_apply(Dinv, v).astype(F)


def two_reduction(A, Dinv, b, tol, maxit):
    x = np.zeros_like(b)
    r = b.copy()
    z = _M(Dinv, r)
    p = z.copy()
    rz, rr0 = F(r @ z), F(r @ r)
    for it in range(1, maxit + 1):
        q = (A @ p).astype(F)
        a = F(rz / F(p @ q))
        x += a * p
        r -= a * q
        z = _M(Dinv, r)
        rz_new, rr = F(r @ z), F(r @ r)
        if rr <= tol * tol * rr0:
            return it
        p = z + F(rz_new / rz) * p
        rz = rz_new
    return None


def single_reduction(A, Dinv, b, tol, maxit, recurrence=False):
    """The kernel's iteration: one phase and one reduction (gamma, delta, rho, u.s + p.w, p.s) per iteration."""
    r = b.copy()
    x = np.zeros_like(b)
    u = _M(Dinv, r)
    p, s, w = np.zeros_like(b), np.zeros_like(b), np.zeros_like(b)
    pub_u, pub_mw, pub_ms = u.copy(), np.zeros_like(b), np.zeros_like(b)
    rr0 = F(r @ r)
    alpha = beta = gamma = F(0)
    for k in range(maxit + 1):
        if k > 0:
            s = w + beta * s
            p = u + beta * p
            x += alpha * p
            r -= alpha * s
            ut = pub_u - alpha * (pub_mw + beta * pub_ms)  # what a gathering CTA forms
            u = ut if recurrence else _M(Dinv, r)          # what the owner keeps
        else:
            ut = pub_u
        w = (A @ ut).astype(F)
        g, d, rr = F(r @ u), F(w @ u), F(r @ r)
        e12, e3 = F(u @ s) + F(p @ w), F(p @ s)
        pub_u, pub_mw, pub_ms = u.copy(), _M(Dinv, w), _M(Dinv, s)
        if k > 0 and rr <= tol * tol * rr0:
            return k
        beta = F(0) if k == 0 else F(g / gamma)
        pq = d + beta * e12 + beta * beta * e3
        if not pq > 0:
            return None
        alpha, gamma = F(g / pq), g
    return None


@pytest.mark.parametrize("kind", ["tension", "dynamic"])
def test_single_reduction_takes_the_two_reduction_iterations(kind):
    A, Dinv, b = _system(kind, 33)
    k2 = two_reduction(A, Dinv, b, 1e-7, 3000)
    k1 = single_reduction(A, Dinv, b, 1e-7, 3000)
    assert k2 is not None and k1 is not None
    assert abs(k1 - k2) <= 0.02 * k2 + 1, (k1, k2)


def test_carrying_u_as_a_recurrence_stagnates():
    A, Dinv, b = _system("tension", 33)
    assert single_reduction(A, Dinv, b, 1e-7, 1500, recurrence=True) is None
    assert single_reduction(A, Dinv, b, 1e-7, 1500) is not None
