"""Krylov solvers of the CPU oracle: the root ``expv`` and the local enrichment recurrences.

TEST INFRASTRUCTURE (see ``oracle/blocks.py``). Restates:

* ``_shift``, ``_tridiag_eigen``, ``_coeffs_from_eigen`` (``src/BUG/Core/LocalSolvers/krylov.jl:44-117``),
  ``lanczos_expv`` (``krylov.jl:128-263``), ``arnoldi_expv`` (``krylov.jl:343-442``), ``_combine``
  (``:305-311``), ``_cgs2!`` (``:321-332``), ``_apply_scale`` (``:296-302``);
* ``_tail``, ``_tail_sup``, ``_pick_tau``, ``_hess_coeffs`` (``root_methods.jl:87-141``);
* ``_kry_weight``, ``_residual_integral`` (``src/BUG/Core/RankAdaptation/krylov_enrichment.jl:58-120``);
* ``_lanczos_chain`` (``krylov_lanczos.jl:18-71``), ``_arnoldi_chain`` (``krylov_arnoldi.jl:13-58``),
  ``_krylov_basis`` / ``_krylov_stop`` (``krylov_recurrence.jl:27-72``).

Vectors are block tensors (``oracle.blocks.BT``) or plain numpy vectors; the module only needs
``inner``, ``norm``, ``add`` and ``scale`` from ``ops``.
"""

from __future__ import annotations

import math

import numpy as np
import scipy.linalg

EXPV_SAFE_EXPONENT = 60.0
EXPV_SHIFT_TRIGGER = 30.0
EXPV_MAX_NORM = 1e150
TAIL_NODES = 8
KRY_BREAKDOWN = 1e-13
KRY_MAXDEPTH = 64
ROOT_MAXITER = 30
KRY_SKEW_TOL = 1e-12
RESIDUAL_MAX_PANELS = 4096


class VecOps:
    """Vector operations for block tensors."""

    def __init__(self):
        from . import blocks as B

        self.B = B

    def inner(self, a, b):
        return self.B.inner(a, b)

    def norm(self, a):
        return self.B.norm(a)

    def lin(self, terms):
        """``sum c_i v_i`` evaluated left to right."""
        out = None
        for c, v in terms:
            out = self.B.scale(v, c) if out is None else self.B.add(out, v, 1.0, c)
        return out


class NumpyOps:
    def inner(self, a, b):
        return complex(np.vdot(a, b))

    def norm(self, a):
        return float(np.linalg.norm(a))

    def lin(self, terms):
        out = None
        for c, v in terms:
            out = c * v if out is None else out + c * v
        return out


def shift(vals, tau) -> float:
    if len(vals) == 0:
        return 0.0
    ex = [(tau * complex(v)).real for v in vals]
    top = int(np.argmax(ex))
    return float(np.real(vals[top])) if ex[top] > EXPV_SHIFT_TRIGGER else 0.0


def tridiag_eigen(alpha, beta):
    alpha = np.asarray(alpha, dtype=np.float64)
    beta = np.asarray(beta, dtype=np.float64)
    if not (np.all(np.isfinite(alpha)) and np.all(np.isfinite(beta))):
        raise ValueError("Lanczos tridiagonal has non-finite entries: the input vector or the operator is not finite")
    n = len(alpha)
    T = np.diag(alpha)
    if n > 1:
        T += np.diag(beta, 1) + np.diag(beta, -1)
    return np.linalg.eigh(T)


def coeffs_from_eigen(vals, vecs, tau):
    sigma = shift(vals, tau)
    w = np.exp(tau * (vals.astype(np.complex128) - sigma)) * vecs[0, :].astype(np.complex128)
    return vecs.astype(np.complex128) @ w, tau * sigma


def hess_coeffs(Hm, tau):
    if Hm.size == 0:
        return np.zeros(0, dtype=np.complex128), 0j
    sigma = shift(np.linalg.eigvals(Hm), tau)
    P = scipy.linalg.expm(tau * (Hm - sigma * np.eye(Hm.shape[0])))
    return P[:, 0].copy(), tau * sigma


# ── implicit roots (root_methods.jl:12-75, 143-168) ─────────────────────────────────────────────
# The stability functions R(z) = N(z) / D(z) of one implicit Runge-Kutta step (coefficients constant
# term first): the trapezoid rule and Radau IIA with two and three stages, the (k, k+1) Pade
# approximants of exp(z).
ROOT_PADE = {
    "trapezoid": ([1.0, 1 / 2], [1.0, -1 / 2]),
    "radau2": ([1.0, 1 / 3], [1.0, -2 / 3, 1 / 6]),
    "radau3": ([1.0, 2 / 5, 1 / 20], [1.0, -3 / 5, 3 / 20, -1 / 60]),
}
ROOT_METHODS = ("exp",) + tuple(ROOT_PADE) + ("radau2_gmres",)


def root_stability(method, z):
    """``root_stability``: ``R(z)`` (``exp(z)`` for ``"exp"``)."""
    z = complex(z)
    if method == "exp":
        return np.exp(z)
    num, den = ROOT_PADE[method]
    return np.polyval(num[::-1], z) / np.polyval(den[::-1], z)


def rational_shift(vals, tau, shift=True):
    """``_rational_shift``: the Ritz value maximising ``Re(tau lambda)`` (none in real time)."""
    if not shift or len(vals) == 0 or tau.real == 0:
        return 0j
    return complex(vals[int(np.argmax([(tau * complex(v)).real for v in vals]))])


def rational_coeffs(vals, vecs, tau, method, shift=True):
    """``_rational_coeffs``: ``R(tau (T - sigma)) e_1`` on the tridiagonal's eigenpairs, no scale."""
    sigma = rational_shift(vals, tau, shift)
    w = np.array([root_stability(method, tau * (complex(v) - sigma)) for v in vals])
    return vecs.astype(np.complex128) @ (w * vecs[0, :].astype(np.complex128)), 0j


def hess_rational(Hm, tau, method, shift=True):
    """``_hess_rational``: ``R(tau (H - sigma)) e_1`` on the Arnoldi Hessenberg, no scale."""
    if Hm.size == 0:
        return np.zeros(0, dtype=np.complex128), 0j
    sigma = rational_shift(np.linalg.eigvals(Hm), tau, shift)
    M = tau * (Hm - sigma * np.eye(Hm.shape[0]))
    num, den = ROOT_PADE[method]

    def poly(c):
        out = c[-1] * np.eye(M.shape[0], dtype=np.complex128)
        for k in range(len(c) - 2, -1, -1):
            out = out @ M + c[k] * np.eye(M.shape[0])
        return out

    e1 = np.zeros(M.shape[0], dtype=np.complex128)
    e1[0] = 1.0
    return np.linalg.solve(poly(den), poly(num) @ e1), 0j


def tail(coeff, betak):
    return 0.0 if len(coeff) == 0 else betak * abs(coeff[-1])


def tail_sup(evalcoeff, step, betak, above=math.inf):
    t = tail(evalcoeff(step)[0], betak)
    if step.real != 0:
        return t
    for node in range(1, TAIL_NODES):
        if t >= above:
            return t
        t = max(t, tail(evalcoeff(step * (node / TAIL_NODES))[0], betak))
    return t


def pick_tau(evalcoeff, tau_rem, betak, conv_tol):
    def accepted(trial):
        tl = tail_sup(evalcoeff, trial, betak, above=conv_tol if conv_tol > 0 else math.inf)
        return math.isfinite(tl) and (conv_tol <= 0 or tl <= conv_tol)

    if accepted(tau_rem):
        return tau_rem
    lo, hi = 0.0, 1.0
    for _ in range(40):
        mid = 0.5 * (lo + hi)
        if accepted(mid * tau_rem):
            lo = mid
        else:
            hi = mid
    return max(lo, 1e-6) * tau_rem


def combine(ops, coeff, basis, beta0):
    return ops.lin([(coeff[c] * beta0, basis[c]) for c in range(len(coeff))])


def apply_scale(ops, cur, logscale):
    sc = np.exp(logscale)
    if not (math.isfinite(abs(sc)) and sc != 0):
        return cur
    n = ops.norm(cur)
    if math.isfinite(n) and n > 0 and abs(sc) * n > EXPV_MAX_NORM:
        return cur
    if sc == 1:
        return cur
    return ops.lin([(sc, cur)])


def lanczos_expv(ops, apply, tau, vector, tol=1e-13, maxiter=60, reorth=False, conv_tol=0.0,
                 substeps=1, root_method="exp", rational_shift=True):
    """``exp(tau*A) vector`` for Hermitian ``A`` (``krylov.jl:128-263``); with an implicit
    ``root_method`` its stability function instead, in one stage. Returns ``(result, report)``
    with ``report = (iterations, substeps, err)``."""
    if root_method not in ROOT_METHODS:
        raise NotImplementedError(f"root_method {root_method!r}: {ROOT_METHODS} are built")
    if root_method == "radau2_gmres":
        return radau2_gmres_expv(ops, apply, tau, vector, tol=tol, maxiter=maxiter,
                                 conv_tol=conv_tol, rational_shift_on=rational_shift)
    if root_method != "exp":
        substeps = 1

    def coeffs(vals, vecs, s):
        if root_method == "exp":
            return coeffs_from_eigen(vals, vecs, s)
        return rational_coeffs(vals, vecs, s, root_method, rational_shift)

    tau = complex(tau)
    beta0 = ops.norm(vector)
    if beta0 == 0:
        return vector, (0, 0, 0.0)
    cur = vector
    tau_rem = tau
    logscale = 0j
    total = nsub = 0
    err = 0.0
    while True:
        nsub += 1
        cur_norm = ops.norm(cur)
        if cur_norm == 0:
            break
        v = ops.lin([(1.0 / cur_norm, cur)])
        basis = [v]
        alpha, betas = [], []
        residual = apply(v)
        total += 1
        a = ops.inner(v, residual).real
        alpha.append(a)
        residual = ops.lin([(1.0, residual), (-a, v)])
        for _ in range(2, maxiter + 1):
            off = ops.norm(residual)
            if off < tol:
                break
            if conv_tol > 0:
                vals, vecs = tridiag_eigen(alpha, betas)
                tt = tail_sup(lambda s: coeffs(vals, vecs, s), tau_rem, off, above=conv_tol)
                if tt < conv_tol:
                    break
            betas.append(off)
            v = ops.lin([(1.0 / off, residual)])
            basis.append(v)
            residual = apply(v)
            total += 1
            a = ops.inner(v, residual).real
            alpha.append(a)
            residual = ops.lin([(1.0, residual), (-a, v), (-off, basis[-2])])
            if reorth:
                for _p in range(2):
                    corr = [(ops.inner(prev, residual), prev) for prev in basis]
                    residual = ops.lin([(1.0, residual)] + [(-c, p) for c, p in corr])
        vals, vecs = tridiag_eigen(alpha, betas)
        evalcoeff = lambda s: coeffs(vals, vecs, complex(s))
        betak = ops.norm(residual)
        if substeps == 1:
            tau_s = tau_rem
        elif substeps > 1:
            tau_s = tau_rem / (substeps - nsub + 1)
        else:
            tau_s = pick_tau(evalcoeff, tau_rem, betak, conv_tol)
        coeff, ls = evalcoeff(tau_s)
        err += tail_sup(evalcoeff, tau_s, betak) * cur_norm / beta0
        cur = combine(ops, coeff, basis, cur_norm)
        logscale += ls
        tau_rem -= tau_s
        if substeps == 1 or abs(tau_rem) <= 1e-14 * max(abs(tau), 1.0):
            break
        if nsub >= 10_000:
            raise RuntimeError(f"expv: substep search failed to advance (tau_rem = {tau_rem})")
    return apply_scale(ops, cur, logscale), (total, nsub, err)


def cgs2(ops, H, column, basis, vector):
    for _p in range(2):
        corr = []
        for row, b in enumerate(basis):
            ov = ops.inner(b, vector)
            H[row, column] += ov
            corr.append((ov, b))
        vector = ops.lin([(1.0, vector)] + [(-c, b) for c, b in corr])
    return vector


def arnoldi_expv(ops, apply, tau, vector, tol=1e-13, maxiter=60, conv_tol=0.0, substeps=1,
                 root_method="exp", rational_shift=True):
    """``exp(tau*A) vector`` for any ``A`` by Arnoldi with CGS2 (``krylov.jl:343-442``); with an
    implicit ``root_method`` its stability function instead, in one stage."""
    if root_method not in ROOT_METHODS:
        raise NotImplementedError(f"root_method {root_method!r}: {ROOT_METHODS} are built")
    if root_method == "radau2_gmres":
        return radau2_gmres_expv(ops, apply, tau, vector, tol=tol, maxiter=maxiter,
                                 conv_tol=conv_tol, rational_shift_on=rational_shift)
    if root_method != "exp":
        substeps = 1

    def hcoeffs(Hm, s):
        if root_method == "exp":
            return hess_coeffs(Hm, s)
        return hess_rational(Hm, s, root_method, rational_shift)

    tau = complex(tau)
    beta0 = ops.norm(vector)
    if beta0 == 0:
        return vector, (0, 0, 0.0)
    cur = vector
    tau_rem = tau
    logscale = 0j
    total = nsub = 0
    err = 0.0
    while True:
        nsub += 1
        cur_norm = ops.norm(cur)
        if cur_norm == 0:
            break
        basis = [ops.lin([(1.0 / cur_norm, cur)])]
        H = np.zeros((maxiter + 1, maxiter), dtype=np.complex128)
        dim = 0
        betak = 0.0
        for k in range(maxiter):
            residual = cgs2(ops, H, k, basis, apply(basis[k]))
            total += 1
            dim = k + 1
            rn = ops.norm(residual)
            betak = rn
            if rn < tol:
                break
            if conv_tol > 0:
                lead = H[:dim, :dim].copy()
                tt = tail_sup(lambda s: hcoeffs(lead, s), tau_rem, rn, above=conv_tol)
                if tt < conv_tol:
                    break
            H[k + 1, k] = rn
            if k + 1 == maxiter:
                break
            basis.append(ops.lin([(1.0 / rn, residual)]))
        Hm = H[:dim, :dim].copy()
        evalcoeff = lambda s: hcoeffs(Hm, complex(s))
        if substeps == 1:
            tau_s = tau_rem
        elif substeps > 1:
            tau_s = tau_rem / (substeps - nsub + 1)
        else:
            tau_s = pick_tau(evalcoeff, tau_rem, betak, conv_tol)
        coeff, ls = evalcoeff(tau_s)
        err += tail_sup(evalcoeff, tau_s, betak) * cur_norm / beta0
        cur = combine(ops, coeff, basis[:dim], cur_norm)
        logscale += ls
        tau_rem -= tau_s
        if substeps == 1 or abs(tau_rem) <= 1e-14 * max(abs(tau), 1.0):
            break
        if nsub >= 10_000:
            raise RuntimeError(f"expv: substep search failed to advance (tau_rem = {tau_rem})")
    return apply_scale(ops, cur, logscale), (total, nsub, err)


# ── radau2_gmres: Radau IIA(2) coupled stages by matrix-free shifted GMRES (root_methods.jl:170-345)
RADAU2_A = np.array([[5 / 12, -1 / 12], [3 / 4, 1 / 4]])
RADAU_MAXCYCLE = 4  # _RADAU_MAXCYCLE


def _radau2_eig():
    lam, P = np.linalg.eig(RADAU2_A.astype(np.complex128))
    return lam, P, np.linalg.inv(P)


def shifted_gmres(ops, apply, rhs, tau, zs, ds, Wt, sigma, target, maxiter, tol):
    """``_shifted_gmres``: one GMRES cycle for ``(I - z_k (B - sigma)) Z_k = d_k rhs`` on one Arnoldi
    basis of ``B``; stops when the stage residual ``|sum_k Wt[:, k] g_k|`` reaches ``target``, at
    breakdown or at ``maxiter``. ``sigma = None`` takes the shift from the current Ritz values."""
    beta = ops.norm(rhs)
    basis = [ops.lin([(1.0 / beta, rhs)])]
    H = np.zeros((maxiter + 1, maxiter), dtype=np.complex128)
    ys, res, sig, nmv = [], math.inf, 0j, 0
    for k in range(1, maxiter + 1):
        nv = cgs2(ops, H, k - 1, basis, apply(basis[k - 1]))
        nmv += 1
        nn = ops.norm(nv)
        H[k, k - 1] = nn
        Hb = H[:k + 1, :k]
        Ib = np.eye(k + 1, k, dtype=np.complex128)
        sig = rational_shift(np.linalg.eigvals(H[:k, :k]), tau) if sigma is None else sigma
        be1 = np.zeros(k + 1, dtype=np.complex128)
        be1[0] = beta
        SR = np.zeros((k + 1, len(zs)), dtype=np.complex128)
        ys = []
        for i, z in enumerate(zs):
            M = Ib - z * (Hb - sig * Ib)
            c = np.linalg.lstsq(M, ds[i] * be1, rcond=None)[0]
            ys.append(c)
            SR[:, i] = ds[i] * be1 - M @ c
        res = float(np.linalg.norm(SR @ Wt.T))
        if nn < tol or res <= target or k == maxiter:
            break
        basis.append(ops.lin([(1.0 / nn, nv)]))
    return [combine(ops, c, basis[:len(c)], 1.0) for c in ys], res, nmv, sig


def radau2_gmres_expv(ops, apply, tau, vector, tol=1e-13, maxiter=60, conv_tol=0.0,
                      rational_shift_on=True):
    """``radau2_gmres_expv``: one Radau IIA(2) step of ``dx/dt = B x`` over ``tau``, the coupled
    stages decoupled by the eigenvectors of the Butcher matrix and solved on one Krylov basis,
    restarted on the true stage residual at most ``RADAU_MAXCYCLE`` times. Returns ``(Y_2,
    (applications, 1, relative stage residual))``."""
    tau = complex(tau)
    beta0 = ops.norm(vector)
    if beta0 == 0:
        return vector, (0, 0, 0.0)
    lam, P, Pinv = _radau2_eig()
    zs = tau * lam
    target = conv_tol * beta0 if conv_tol > 0 else 0.0
    Zs, _, nmv, sigma = shifted_gmres(ops, apply, vector, tau, zs, Pinv @ np.ones(2), P,
                                      None if rational_shift_on else 0j, target, maxiter, tol)

    def stage(Z, i):
        return ops.lin([(P[i, 0], Z[0]), (P[i, 1], Z[1])])

    Y = [stage(Zs, 0), stage(Zs, 1)]

    def residual(Y):
        nonlocal nmv
        BY = []
        for y in Y:
            img = apply(y)
            BY.append(img if sigma == 0 else ops.lin([(1.0, img), (-sigma, y)]))
        nmv += 2
        R = [ops.lin([(1.0, vector), (-1.0, Y[i]), (tau * RADAU2_A[i, 0], BY[0]),
                      (tau * RADAU2_A[i, 1], BY[1])]) for i in range(2)]
        return R, math.sqrt(ops.norm(R[0]) ** 2 + ops.norm(R[1]) ** 2)

    R, res = residual(Y)
    cycles = 1
    while target > 0 and res > target and cycles < RADAU_MAXCYCLE:
        cycles += 1
        dZ = []
        for i in range(2):
            rho = ops.lin([(Pinv[i, 0], R[0]), (Pinv[i, 1], R[1])])
            if ops.norm(rho) == 0:
                dZ.append(rho)
                continue
            Zk, _, m, _ = shifted_gmres(ops, apply, rho, tau, zs[i:i + 1], np.ones(1, dtype=np.complex128),
                                        P[:, i:i + 1], sigma, target / math.sqrt(2), maxiter, tol)
            nmv += m
            dZ.append(Zk[0])
        Y = [ops.lin([(1.0, Y[i]), (1.0, stage(dZ, i))]) for i in range(2)]
        R, res = residual(Y)
    return Y[1], (nmv, 1, res / beta0)


def expv(ops, apply, tau, vector, hermitian=True, **kw):
    """``expv`` dispatcher (``root_methods.jl:359-402``): ``root_method`` ``"exp"``, one of the
    implicit roots ``"trapezoid"``, ``"radau2"``, ``"radau3"``, or ``"radau2_gmres"``."""
    if kw.get("root_method") == "radau2_gmres":
        return radau2_gmres_expv(ops, apply, tau, vector, tol=kw.get("tol", 1e-13),
                                 maxiter=kw.get("maxiter", 60), conv_tol=kw.get("conv_tol", 0.0),
                                 rational_shift_on=kw.get("rational_shift", True))
    if hermitian:
        return lanczos_expv(ops, apply, tau, vector, **kw)
    kw.pop("reorth", None)
    return arnoldi_expv(ops, apply, tau, vector, **kw)


# ── local Krylov weights and chains ──────────────────────────────────────────────────────────


def residual_integral(defect_norm, generator, tau, state_seed=True):
    """``|tau| int_0^1 defect_norm(exp(s M) e_1) ds`` by composite Simpson in log space
    (``krylov_enrichment.jl:89-120``)."""
    g = np.asarray(generator, dtype=np.complex128)
    n = g.shape[0]
    unitary = np.linalg.norm(g + g.conj().T) <= KRY_SKEW_TOL * np.linalg.norm(g)
    sigma = 0.0 if unitary else float(np.max(np.linalg.eigvals(g).real))
    shifted = g - sigma * np.eye(n)
    intervals = 2 * min(max(math.ceil(2 * np.linalg.norm(shifted, 1)), 8), RESIDUAL_MAX_PANELS)
    spacing = 1.0 / intervals
    prop = scipy.linalg.expm(spacing * shifted)
    col = np.zeros(n, dtype=np.complex128)
    col[0] = 1
    logs = np.empty(intervals + 1)
    for node in range(intervals + 1):
        if node > 0:
            col = prop @ col
        w = 1.0 if node in (0, intervals) else (4.0 if node % 2 == 1 else 2.0)
        mag = defect_norm(col)
        logs[node] = -math.inf if mag == 0 else math.log(w * spacing / 3 * mag) + node * spacing * sigma
    peak = float(np.max(logs))
    if peak == -math.inf:
        return 0.0
    lw = math.log(abs(tau)) + peak + math.log(float(np.sum(np.exp(logs - peak))))
    if unitary or not state_seed:
        return math.exp(lw)
    return math.exp(lw - sigma - math.log(max(np.linalg.norm(col), np.finfo(float).tiny)))


def kry_weight(Hm, k, tau, state_seed=True):
    """Weight of ``v_{k+1}`` in ``exp(tau H) v_1`` (``krylov_enrichment.jl:58-73``); ``k`` 1-based."""
    beta = abs(Hm[k, k - 1])
    if beta == 0:
        return 0.0
    return beta * residual_integral(lambda c: abs(c[k - 1]), tau * Hm[:k, :k], tau, state_seed)


def krylov_stop(weight, allowance, step, fixed_depth):
    if fixed_depth > 0:
        return step >= fixed_depth, step >= fixed_depth and weight <= allowance
    return weight <= allowance, weight <= allowance


def lanczos_chain(ops, unit_seed, applyH, tau, allowance, score, maxdepth=KRY_MAXDEPTH, amp=1.0,
                  state_seed=True, fixed_depth=0):
    vs, weights = [unit_seed], [amp]
    Hm = np.zeros((maxdepth + 1, maxdepth + 1), dtype=np.complex128)
    closed = capped = False
    n_h1 = 0
    prev_beta = 0.0
    for step in range(1, maxdepth + 1):
        image = applyH(vs[step - 1])
        n_h1 += 1
        if step > 1:
            image = ops.lin([(1.0, image), (-prev_beta, vs[step - 2])])
        alpha = ops.inner(vs[step - 1], image)
        if not abs(alpha.imag) <= 1e-9 * max(abs(alpha), 1.0):
            raise ValueError(f"Lanczos needs a Hermitian one-site generator (imag alpha = {alpha})")
        Hm[step - 1, step - 1] = alpha.real
        image = ops.lin([(1.0, image), (-alpha.real, vs[step - 1])])
        if step >= 20 and step % 2 == 0:
            corr = [(ops.inner(b, image), b) for b in vs]
            image = ops.lin([(1.0, image)] + [(-c, b) for c, b in corr])
        beta = ops.norm(image)
        if beta <= KRY_BREAKDOWN:
            closed = True
            break
        Hm[step, step - 1] = beta
        Hm[step - 1, step] = beta
        nv = ops.lin([(1.0 / beta, image)])
        vs.append(nv)
        w = amp * kry_weight(Hm, step, tau, state_seed)
        weights.append(w)
        if not score(nv, w, step == 1):
            capped = True
            break
        stop, closed = krylov_stop(w, allowance, step, fixed_depth)
        if stop:
            break
        prev_beta = beta
    if not closed:
        capped = True
    return dict(basis=vs, weights=weights, n_h1=n_h1, closed=closed, capped=capped)


def arnoldi_chain(ops, unit_seed, applyH, tau, allowance, score, maxdepth=KRY_MAXDEPTH, amp=1.0,
                  state_seed=True, fixed_depth=0):
    nh = 0
    capped = closed = False
    vs, ws = [unit_seed], [amp]
    Hm = np.zeros((maxdepth + 1, maxdepth + 1), dtype=np.complex128)
    for step in range(1, maxdepth + 1):
        image = applyH(vs[-1])
        nh += 1
        for _p in range(2):
            corr = []
            for row, b in enumerate(vs):
                ov = ops.inner(b, image)
                Hm[row, step - 1] += ov
                corr.append((ov, b))
            image = ops.lin([(1.0, image)] + [(-c, b) for c, b in corr])
        rn = ops.norm(image)
        if rn <= KRY_BREAKDOWN:
            closed = True
            break
        Hm[step, step - 1] = rn
        nv = ops.lin([(1.0 / rn, image)])
        vs.append(nv)
        w = amp * kry_weight(Hm, step, tau, state_seed)
        ws.append(w)
        if not score(nv, w, step == 1):
            capped = True
            break
        stop, closed = krylov_stop(w, allowance, step, fixed_depth)
        if stop:
            break
    if not closed:
        capped = True
    return dict(basis=vs, weights=ws, n_h1=nh, closed=closed, capped=capped)


def krylov_basis(ops, seed, applyH, tau, allowance, score, maxdepth=KRY_MAXDEPTH, amp=1.0,
                 state_seed=True, recurrence="arnoldi", fixed_depth=0):
    if recurrence not in ("lanczos", "arnoldi"):
        raise ValueError(f"unknown local Krylov recurrence: {recurrence}")
    sn = ops.norm(seed)
    if not sn > 0:
        return dict(basis=[], weights=[], n_h1=0, closed=True, capped=False)
    teff = 1.0 + 0j if tau == 0 else complex(tau)
    unit = ops.lin([(1.0 / sn, seed)])
    chain = lanczos_chain if recurrence == "lanczos" else arnoldi_chain
    return chain(ops, unit, applyH, teff, allowance, score, maxdepth=maxdepth, amp=amp,
                 state_seed=state_seed, fixed_depth=fixed_depth)
