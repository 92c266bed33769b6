"""The quantics inputs: the oracle's Heston generator pinned to the reference's own checks, and the
product's builders (carry-automaton route) against the oracle (dense TT-SVD route).

The oracle pins follow ``test/QTTS/Models/Heston/test_heston.jl``: the generator against the dense
one-sided-stencil matrix and the forward adjoint against its transpose (< 1e-11), mass conservation
of the forward operator, the degenerate v = 0 rows, the manufactured affine solution converging at
second order, and five BUG steps against the dense exponential (< 1e-5).
"""

import numpy as np
import scipy.linalg as sl

from oracle import qtt as Q
from oracle import step as OS

HP = Q.HestonParams(0.03, 0.01, 2.0, 0.09, 0.4, -0.7)
HP_FIELDS = (HP.r, HP.q, HP.kappa, HP.theta, HP.sigma, HP.rho)


def heston_grid(nx, ny):
    return Q.qtt_grid(nx, ny, x=(-1.0, 1.0), y=(0.0, 0.5), periodic_x=False, periodic_y=False)


def relerr(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def test_grid_and_separable_field():
    g = heston_grid(3, 4)
    assert g.length == 7 and np.isclose(g.dx, 2 / 7) and np.isclose(g.dy, 0.5 / 15)
    cores = Q.qtt_separable(g, lambda x: np.exp(0.5 * x), lambda v: np.exp(-v))
    assert [c.shape[2] for c in cores[:-1]] == [1] * 6  # exponentials are rank 1 in QTT
    psi = Q.qtt_mps(cores)
    xs, vs = Q.coords(g)
    exact = np.array([np.exp(0.5 * x - v) for v in vs for x in xs])  # x fastest
    assert relerr(Q.qtt_dense(psi), exact) < 1e-13


def test_generator_adjoint_mass_and_degenerate_rows():
    g = heston_grid(3, 3)
    D = Q.heston_dense(g, HP)
    M = Q.mpo_dense(Q.heston_cores(g, HP))
    assert relerr(M, D) < 1e-11
    F = Q.mpo_dense(Q.heston_cores(g, HP, adjoint=True))
    assert relerr(F, (D + HP.r * np.eye(64)).T) < 1e-11
    assert np.linalg.norm(np.ones(64) @ F) < 1e-9 * np.linalg.norm(F)
    flat = Q.HestonParams(HP.r, HP.q, HP.kappa, HP.theta, 0.0, 0.0)
    Md = Q.mpo_dense(Q.heston_cores(g, flat))
    assert relerr(M[:8], Md[:8]) < 1e-11  # v = 0: no diffusion or mixed term


def test_manufactured_affine_solution_second_order():
    a, b, p = 0.5, -1.0, HP

    def lam(v):
        return ((a * a - a) * v / 2 + p.rho * p.sigma * a * b * v + p.sigma ** 2 * b * b * v / 2
                + (p.r - p.q) * a + p.kappa * (p.theta - v) * b - p.r)

    errs = []
    for nbits in (4, 5):
        g = heston_grid(nbits, nbits)
        xs, vs = Q.coords(g)
        field = Q.qtt_dense(Q.qtt_mps(Q.qtt_separable(g, lambda x: np.exp(a * x),
                                                      lambda v: np.exp(b * v))))
        applied = Q.mpo_dense(Q.heston_cores(g, p)) @ field
        exact = np.array([lam(v) * np.exp(a * x + b * v) for v in vs for x in xs])
        errs.append(np.max(np.abs(applied - exact)) / np.max(np.abs(exact)))
    assert errs[1] < 0.35 * errs[0]
    assert errs[1] < 1e-2


def test_bug_step_against_dense_exponential():
    g = heston_grid(4, 4)
    init = Q.qtt_separable(g, lambda x: np.exp(0.5 * x), lambda v: np.exp(-2 * v) * (1 + v))
    exact = sl.expm(0.1 * Q.heston_dense(g, HP)) @ Q.qtt_dense(Q.qtt_mps(init))
    mpo = Q.heston_mpo(g, HP)
    errors = []
    for tol_basis in (1e-3, 1e-8):
        psi = Q.qtt_mps(init, center=1)
        rng = np.random.default_rng(0)
        for _ in range(5):
            OS.cbe_bug_step(psi, mpo, 0.02, tol_basis=tol_basis, tol_trunc=1e-12, maxdim=64,
                            hermitian=False, rng=rng)
        errors.append(relerr(Q.qtt_dense(psi), exact))
    assert errors[1] <= max(errors[0], 1e-10)
    assert errors[1] < 1e-5


def _op_dot(A, B):
    """<A, B> (Frobenius) of two operator chains, core by core."""
    E = np.ones((1, 1), dtype=np.complex128)
    for a, b in zip(A, B):
        E = np.einsum("xy,xoir,yois->rs", E, a.conj(), b)
    return E[0, 0]


def test_product_builders_match_oracle():
    from bondupdategalerkin_b200 import qtt as P

    dom = dict(x=(-1.0, 1.0), y=(0.0, 0.5), periodic_x=False, periodic_y=False)
    g, pg = heston_grid(5, 5), P.qtt_grid(5, 5, **dom)
    for adjoint in (False, True):
        D = Q.heston_dense(g, HP, adjoint=adjoint)
        pc = P.heston_cores(pg, P.HestonParams(*HP_FIELDS), adjoint=adjoint)
        assert relerr(Q.mpo_dense(pc), D) < 1e-11
    for order in (1, 2):
        assert relerr(Q.mpo_dense(P.op_derivative(5, 0.1, order)),
                      Q.derivative_dense(32, 0.1, order)) < 1e-12
    # full size (10 + 10 bits): || A_product - A_oracle ||_F from <A,A> + <B,B> - 2 Re <A,B>; the
    # identity cancels to ~sqrt(eps) of the norm in float64, which bounds what it can resolve
    g10, pg10 = heston_grid(10, 10), P.qtt_grid(10, 10, **dom)
    A = Q.heston_cores(g10, HP)
    B = P.heston_cores(pg10, P.HestonParams(*HP_FIELDS))
    aa, bb, ab = _op_dot(A, A).real, _op_dot(B, B).real, _op_dot(A, B).real
    assert np.sqrt(max(aa + bb - 2 * ab, 0.0)) <= 1e-6 * np.sqrt(aa)
    assert [c.shape[3] for c in A[:-1]] == [c.shape[3] for c in B[:-1]]
    # separable fields: the same TT up to the core gauge
    fx, fv = (lambda x: np.exp(0.5 * x)), (lambda v: np.exp(-v))
    ta, tb = Q.qtt_separable(g10, fx, fv), P.qtt_separable(pg10, fx, fv)
    assert [c.shape for c in ta] == [c.shape for c in tb]
