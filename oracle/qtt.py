"""Quantics (QTT) inputs of the CPU oracle: the grid, separable fields and the Heston generator.

TEST INFRASTRUCTURE (see ``oracle/blocks.py``): only ``tests/``, the smoke check and the bench's CPU
baseline use this module, as the checker. Restates, under the ``:none`` symmetry:

* ``qtt_grid`` (``src/QTTS/Tooling/grid.jl:152-168``) with its default ordering, GROUPED and least
  significant bit first (``grid.jl:1-12``, ``_qtt_site_map`` ``grid.jl:58-73``): site ``k + 1``
  holds bit ``k`` of the x index, site ``nx + k + 1`` bit ``k`` of the y index, so the site
  configuration ``c = sum_s 2^(s-1) b_s`` IS the grid index ``ix + 2^nx iy``;
* ``tt_from_dense`` / ``tt_from_samples`` with the ``_qtt_rank`` rule (``src/QTTS/Tooling/
  cores.jl:18-28,52-90``), ``qtt_separable`` and the grouped ``qtt_embed`` (``cores.jl:175-227,
  265-270``: on the grouped ordering the two chains are concatenated);
* ``qtt_mps`` (``src/QTTS/Tooling/state_adapter.jl:72-82``): the cores as one dense block each,
  gauged to the centre by exact SVD moves;
* ``heston_op`` (``src/QTTS/Models/Heston/heston.jl:36-61``) with the ``:onesided`` stencils of
  ``qtt_derivative`` (``src/QTTS/Tooling/derivatives.jl:40-83``; row by row as the reference's
  dense test helper ``_ref_d``, ``test/common/qtt_fixtures.jl:37-70``), and ``qtt_to_mpo``
  (``state_adapter.jl:96-109``: the solver MPO stores ``(w_l, in, out, w_r)``, the ket contracting
  ``in``).

The oracle's route to the MPO is its own: every one-dimensional factor is formed as a dense
``2^n x 2^n`` matrix and TT-SVD'd into operator cores, the three x-factor groups of the generator
are summed as a direct sum and the sum is compressed. The reference assembles the same operator
from carry-automaton shifts (``derivatives.jl:21-36``); both are exact up to the 1e-14 compression,
and ``tests/test_qtt_oracle.py`` pins this one to the dense generator as ``test/QTTS/Models/Heston/
test_heston.jl:14-54`` does.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .blocks import BT, Leg
from .models import MPO, MPS
from .step import canonical


@dataclass(frozen=True)
class Grid:
    """``x_i = x0 + i dx`` (``i < 2^nx``), ``y_j = y0 + j dy`` (``j < 2^ny``), grouped LSB-first."""

    nx: int
    ny: int
    x0: float
    dx: float
    y0: float
    dy: float
    periodic_x: bool
    periodic_y: bool

    @property
    def length(self) -> int:
        return self.nx + self.ny


def qtt_grid(nx, ny, x=(-1.0, 1.0), y=(-1.0, 1.0), periodic_x=True, periodic_y=True,
             order="grouped", endian="lsb_first") -> Grid:
    """``grid.jl:152-168``: spacing ``(b - a) / 2^n`` (periodic) or ``/(2^n - 1)`` (end points)."""
    if nx < 1 or ny < 1:
        raise ValueError("qtt_grid needs at least one bit per coordinate")
    if not (x[1] > x[0] and y[1] > y[0]):
        raise ValueError(f"empty domain {x} x {y}")
    if order not in ("grouped", "interleaved"):  # QTTOrdering, grid.jl:43-46
        raise ValueError(f"order must be :grouped or :interleaved, got :{order}")
    if endian not in ("lsb_first", "msb_first"):
        raise ValueError(f"endian must be :lsb_first or :msb_first, got :{endian}")
    if (order, endian) != ("grouped", "lsb_first"):
        raise NotImplementedError("only the default ordering (grouped, least significant bit first) "
                                  "is built; the others are the reference's diagnostics")
    dx = (x[1] - x[0]) / (2 ** nx if periodic_x else 2 ** nx - 1)
    dy = (y[1] - y[0]) / (2 ** ny if periodic_y else 2 ** ny - 1)
    return Grid(nx, ny, float(x[0]), dx, float(y[0]), dy, periodic_x, periodic_y)


def coords(g: Grid):
    return g.x0 + g.dx * np.arange(2 ** g.nx), g.y0 + g.dy * np.arange(2 ** g.ny)


def cell(g: Grid) -> float:
    return g.dx * g.dy


# ── TT-SVD ────────────────────────────────────────────────────────────────────────────────────

def _rank(S, delta, maxdim):
    """``_qtt_rank`` (``cores.jl:18-28``): the smallest rank whose discarded tail is <= delta."""
    r = len(S)
    tail = 0.0
    while r > 1 and tail + S[r - 1] ** 2 <= delta ** 2:
        tail += S[r - 1] ** 2
        r -= 1
    return max(min(r, maxdim), 1)


def _tt_svd(A, local, tol, maxdim):
    """TT-SVD of ``A`` whose axes are the sites in order, each of size ``local``."""
    L = A.ndim
    nrm = np.linalg.norm(A)
    delta = tol * nrm / np.sqrt(max(L - 1, 1))
    cores = []
    M = A.reshape(local, -1)
    chi = 1
    for _ in range(L - 1):
        M = M.reshape(chi * local, -1)
        U, S, Vh = np.linalg.svd(M, full_matrices=False)
        r = _rank(S, delta, maxdim)
        cores.append(U[:, :r].reshape(chi, local, r))
        M = S[:r, None] * Vh[:r]
        chi = r
    cores.append(M.reshape(chi, local, 1))
    return cores


def tt_from_samples(vals, tol=1e-14, maxdim=1 << 30):
    """The 1D quantics TT of ``vals[i] = f(x_i)``, logical order (bit 0 on the first site)
    (``tt_from_samples``, ``cores.jl:86-90``)."""
    vals = np.asarray(vals)
    n = int(round(np.log2(len(vals))))
    if 2 ** n != len(vals):
        raise ValueError(f"need 2^n samples, got {len(vals)}")
    # axis k of the array is bit k: i = sum_k 2^k b_k (Fortran-order reshape)
    A = np.asarray(vals, dtype=np.complex128).reshape((2,) * n, order="F")
    return _tt_svd(A, 2, tol, maxdim)


def op_from_dense(M, tol=1e-14, maxdim=1 << 30):
    """Operator cores ``(w_l, out, in, w_r)`` of a dense ``2^n x 2^n`` matrix ``M[out, in]``, bit
    ``k`` of both indices on site ``k + 1`` (the logical order of ``cores.jl:1-12``)."""
    M = np.asarray(M, dtype=np.complex128)
    n = int(round(np.log2(M.shape[0])))
    # T[o_{n-1} .. o_0, i_{n-1} .. i_0] (C order puts the most significant bit first)
    T = M.reshape((2,) * (2 * n))
    perm = []
    for k in range(n):
        perm += [n - 1 - k, 2 * n - 1 - k]  # site k: (o_k, i_k)
    T = T.transpose(perm).reshape((4,) * n)
    cores = _tt_svd(T, 4, tol, maxdim)
    return [c.reshape(c.shape[0], 2, 2, c.shape[2]) for c in cores]


def op_compress(cores, tol=1e-14):
    """Left QR sweep, then right-to-left SVD truncation at relative Frobenius ``tol / sqrt(L-1)``
    (``tt_compress``, ``cores.jl:92-128``, on operator cores read with d = 4)."""
    C = [c.reshape(c.shape[0], 4, c.shape[3]).astype(np.complex128) for c in cores]
    L = len(C)
    for k in range(L - 1):
        chi, d, r = C[k].shape
        Q, R = np.linalg.qr(C[k].reshape(chi * d, r))
        C[k] = Q.reshape(chi, d, Q.shape[1])
        C[k + 1] = np.tensordot(R, C[k + 1], axes=(1, 0))
    nrm = np.linalg.norm(C[-1])
    delta = tol * nrm / np.sqrt(max(L - 1, 1))
    for k in range(L - 1, 0, -1):
        chi, d, r = C[k].shape
        U, S, Vh = np.linalg.svd(C[k].reshape(chi, d * r), full_matrices=False)
        rr = _rank(S, delta, 1 << 30)
        C[k] = Vh[:rr].reshape(rr, d, r)
        C[k - 1] = np.tensordot(C[k - 1], U[:, :rr] * S[:rr], axes=(2, 0))
    return [c.reshape(c.shape[0], 2, 2, c.shape[2]) for c in C]


def op_direct_sum(chains):
    """``sum_t chain_t`` as one chain: block-diagonal inner cores, boundary cores concatenated."""
    L = len(chains[0])
    out = []
    for s in range(L):
        parts = [ch[s] for ch in chains]
        wl = 1 if s == 0 else sum(p.shape[0] for p in parts)
        wr = 1 if s == L - 1 else sum(p.shape[3] for p in parts)
        c = np.zeros((wl, 2, 2, wr), dtype=np.complex128)
        ol = orr = 0
        for p in parts:
            a, b = p.shape[0], p.shape[3]
            li = slice(0, 1) if s == 0 else slice(ol, ol + a)
            ri = slice(0, 1) if s == L - 1 else slice(orr, orr + b)
            c[li, :, :, ri] += p
            if s != 0:
                ol += a
            if s != L - 1:
                orr += b
        out.append(c)
    return out


# ── fields and states ────────────────────────────────────────────────────────────────────────

def qtt_separable(g: Grid, fx, fy, tol=1e-14):
    """``fx(x) fy(y)`` from two 1D TT-SVDs, concatenated on the grouped ordering
    (``cores.jl:265-270``)."""
    xs, ys = coords(g)
    tx = tt_from_samples(np.array([fx(x) for x in xs]), tol)
    ty = tt_from_samples(np.array([fy(y) for y in ys]), tol)
    return tx + ty


def qtt_mps(cores, center=1) -> MPS:
    """``state_adapter.jl:72-82``: one dense block per site (``:none``), centre at L, then exact SVD
    moves to site 1 and on to ``center``."""
    L = len(cores)
    ts = []
    for c in cores:
        legs = [Leg(-1, {0: c.shape[0]}), Leg(-1, {0: 2}), Leg(+1, {0: c.shape[2]})]
        ts.append(BT(legs, {(0, 0, 0): np.asarray(c, dtype=np.complex128)}))
    psi = MPS(ts, L)
    canonical(psi, 1)
    canonical(psi, center)
    return psi


def qtt_dense(psi: MPS) -> np.ndarray:
    """Amplitudes at ``c = sum_s 2^(s-1) b_s`` (site 1 fastest: the grid index ``ix + 2^nx iy``).
    Small sizes only."""
    v = None
    for i in range(1, len(psi) + 1):
        t = psi[i]
        blk = t.blocks.get((0, 0, 0))
        if blk is None:
            blk = np.zeros(tuple(l.sectors[0] for l in t.legs), dtype=np.complex128)
        if v is None:
            v = blk[0]  # (2, chi_r); index = b_1
        else:
            # v[c_prev, chi] x blk[chi, b, chi_r] -> new index c_prev + 2^(i-1) b (b slower)
            v = np.einsum("ca,abr->bcr", v, blk).reshape(-1, blk.shape[2])
    return v[:, 0]


# ── one-dimensional operators and the Heston generator ─────────────────────────────────────

def derivative_dense(N, h, order, bc="onesided"):
    """The ``N x N`` central difference of ``order`` 1 or 2 with boundary ``bc``, the first and
    last rows replaced by second-order one-sided stencils under ``onesided``
    (``derivatives.jl:40-83``, row by row as ``_ref_d``, ``qtt_fixtures.jl:37-70``)."""
    D = np.zeros((N, N))
    stencil = ((1, 1 / (2 * h)), (-1, -1 / (2 * h))) if order == 1 else \
        ((1, 1 / h ** 2), (0, -2 / h ** 2), (-1, 1 / h ** 2))
    for row in range(N):
        for off, w in stencil:
            col = row + off
            if bc == "periodic":
                col %= N
            elif not 0 <= col < N:
                continue
            D[row, col] += w
    if bc == "onesided":
        D[0, :] = 0.0
        D[-1, :] = 0.0
        if order == 1:
            D[0, :3] = np.array([-3, 4, -1]) / (2 * h)
            D[-1, -3:] = np.array([1, -4, 3]) / (2 * h)
        else:
            D[0, :4] = np.array([2, -5, 4, -1]) / h ** 2
            D[-1, -4:] = np.array([-1, 4, -5, 2]) / h ** 2
    return D


@dataclass(frozen=True)
class HestonParams:
    """``heston.jl:16-23``: rate, dividend yield, mean reversion, long-run variance, vol of vol,
    correlation."""

    r: float
    q: float
    kappa: float
    theta: float
    sigma: float
    rho: float


def heston_factors(g: Grid, p: HestonParams, adjoint=False):
    """The generator ``A_H`` as ``sum_t Ax_t (x) Av_t`` with the three x factors ``D_xx, D_x, I``
    (``heston.jl:36-61`` regrouped by x factor); with ``adjoint`` the factors of the forward
    operator ``A_H'`` (transpose, no discount)."""
    if g.periodic_x or g.periodic_y:
        raise ValueError("heston_op: build the grid with periodic_x = periodic_y = false")
    if abs(g.y0) >= 1e-14:
        raise ValueError("heston_op: the variance grid must start at v = 0")
    Nx, Nv = 2 ** g.nx, 2 ** g.ny
    _, vs = coords(g)
    D1x, D2x = derivative_dense(Nx, g.dx, 1), derivative_dense(Nx, g.dx, 2)
    D1v, D2v = derivative_dense(Nv, g.dy, 1), derivative_dense(Nv, g.dy, 2)
    V = np.diag(vs)
    Iv, Ix = np.eye(Nv), np.eye(Nx)
    disc = 0.0 if adjoint else p.r
    terms = [
        (D2x, 0.5 * V),
        (D1x, p.rho * p.sigma * (V @ D1v) + (p.r - p.q) * Iv - 0.5 * V),
        (Ix, 0.5 * p.sigma ** 2 * (V @ D2v) + p.kappa * p.theta * D1v - p.kappa * (V @ D1v)
         - disc * Iv),
    ]
    if adjoint:
        terms = [(ax.T.copy(), av.T.copy()) for ax, av in terms]
    return terms


def heston_dense(g: Grid, p: HestonParams, adjoint=False) -> np.ndarray:
    """The dense generator on the grid index ``ix + 2^nx iy`` (x fastest): ``kron(Av, Ax)``
    summed (``test_heston.jl:14-27``). Small grids only."""
    return sum(np.kron(av, ax) for ax, av in heston_factors(g, p, adjoint))


def heston_cores(g: Grid, p: HestonParams, adjoint=False, tol=1e-14):
    """Operator cores ``(w_l, out, in, w_r)`` of the generator on the grid's ``nx + ny`` sites."""
    chains = [op_from_dense(ax, tol) + op_from_dense(av, tol)
              for ax, av in heston_factors(g, p, adjoint)]
    return op_compress(op_direct_sum(chains), tol)


def cores_to_mpo(cores) -> MPO:
    """``qtt_to_mpo`` (``state_adapter.jl:96-109``): the solver MPO stores ``(w_l, in, out, w_r)``
    with arrows ``(w_l:-1, s_in:+1, s_out:-1, w_r:+1)``, one dense block under ``:none``."""
    ts = []
    for c in cores:
        W = np.ascontiguousarray(np.asarray(c, dtype=np.complex128).transpose(0, 2, 1, 3))
        legs = [Leg(-1, {0: W.shape[0]}), Leg(+1, {0: 2}), Leg(-1, {0: 2}), Leg(+1, {0: W.shape[3]})]
        ts.append(BT(legs, {(0, 0, 0, 0): W}))
    return MPO(ts)


def heston_mpo(g: Grid, p: HestonParams, adjoint=False) -> MPO:
    """``heston_mpo`` (``heston.jl:69``)."""
    return cores_to_mpo(heston_cores(g, p, adjoint))


def mpo_dense(cores) -> np.ndarray:
    """``M[out, in]`` of operator cores on the site-1-fastest index. Small sizes only."""
    M = None
    for c in cores:
        if M is None:
            M = c[0]  # (out, in, w_r)
        else:
            # (O, I, w) x (w, o, i, r) -> (o O, i I, r), the new bit slower
            M = np.einsum("OIw,woir->oOiIr", M, c)
            M = M.reshape(M.shape[0] * M.shape[1], M.shape[2] * M.shape[3], M.shape[4])
    return M[:, :, 0]


# ── the QTT BUG step of a linear flow (src/QTTS/Tooling/nonlinear_step.jl) ───────────────────

QTT_KRYLOV_MARGIN = 0.5       # _QTT_KRYLOV_MARGIN, nonlinear_step.jl:8
QTT_RATIONAL_MAXITER = 200    # _QTT_RATIONAL_MAXITER, nonlinear_step.jl:17
QTT_TOL_FLOOR = 1e-14         # _QTT_TOL_FLOOR, nonlinear_step.jl:23


def qtt_step_tolerance(tol, h, order, scaling="order", h_ref=0.1):
    """``qtt_step_tolerance`` (``nonlinear_step.jl:25-47``): ``tol (|h| / h_ref)^(order + 1)``
    (never looser than ``tol``), floored at 1e-14 unless ``tol`` is already below it; ``fixed``
    returns ``tol``."""
    if scaling not in ("order", "fixed"):
        raise ValueError(f"tol_scaling must be :order or :fixed, got :{scaling}")
    if not h_ref > 0:
        raise ValueError(f"tol_h_ref must be positive, got {h_ref}")
    if scaling == "fixed" or tol == 0:
        return float(tol)
    factor = min(1.0, (abs(float(h)) / float(h_ref)) ** (order + 1))
    return max(float(tol) * factor, min(float(tol), QTT_TOL_FLOOR))


def qtt_root_for_order(order):
    """``qtt_root_for_order`` (``stage_solvers.jl:161-165``): 2 trapezoid, 3 Radau IIA (2 stages),
    4 Radau IIA (3 stages)."""
    roots = {2: "trapezoid", 3: "radau2", 4: "radau3"}
    if order not in roots:
        raise ValueError(f"nonlinear BUG orders are 2, 3, 4; got {order}")
    return roots[order]


def qtt_bug_step(psi, mpo, t, h, *, pref=1.0, order=2, root=None, tol_stage=1e-10, tol_basis=1e-6,
                 tol_trunc=1e-8, maxdim=128, stage_solver="auto", tol_scaling="order",
                 tol_h_ref=0.1, tol_krylov=None, rng=None, **kwargs):
    """``qtt_bug_step!`` (``nonlinear_step.jl:102-371``) for a linear flow ``F = pref H psi``
    (``LinearFlow``, ``flows.jl:20-31``, with ``H`` the operator of ``mpo``): ``stage_solver =
    :auto`` is ``:krylov_rational`` there, i.e. ``cbe_bug_step!`` at ``order`` with the rational root
    ``root`` (trapezoid / Radau IIA stability function on the Arnoldi basis of the Galerkin operator)
    applied unshifted, capped at 200 Arnoldi vectors, then compressed (``nonlinear_step.jl:238-250,
    327-371``). The tolerances are per-step ``qtt_step_tolerance`` values. The Newton-GMRES stage path
    of nonlinear flows is not restated. Returns the step report (``converged``: the root's Krylov
    error within the stage tolerance)."""
    if stage_solver not in ("auto", "krylov_rational", "newton_gmres"):
        raise ValueError("stage_solver must be :auto, :newton_gmres or :krylov_rational, "
                         f"got :{stage_solver}")
    if stage_solver == "newton_gmres":
        raise NotImplementedError("stage_solver = :newton_gmres (the nonlinear stage equations)")
    root = qtt_root_for_order(order) if root is None else root
    st = lambda tol: qtt_step_tolerance(tol, h, order, scaling=tol_scaling, h_ref=tol_h_ref)  # noqa: E731
    tol_step = dict(basis=st(tol_basis), trunc=st(tol_trunc), stage=st(tol_stage),
                    scaling=tol_scaling, h_ref=float(tol_h_ref))
    tol_kry = st(QTT_KRYLOV_MARGIN * tol_basis if tol_krylov is None else tol_krylov)
    from oracle import step as S

    info = S.cbe_bug_step(psi, mpo, complex(pref * h), order=order, tol_basis=tol_step["basis"],
                          tol_trunc=tol_step["trunc"], maxdim=maxdim, hermitian=False, eshift=0.0,
                          tol_krylov=tol_kry, root_method=root, tol_root=tol_step["stage"],
                          root_shift=False, root_maxiter=QTT_RATIONAL_MAXITER, truncate=True,
                          rng=rng, **kwargs)
    err = info["ledger"].expv_err
    return dict(solver="krylov_rational", root=root, order=order, converged=err <= tol_step["stage"],
                residual=err, krylov=info["ledger"].expv_iters, discarded=info["discarded"],
                chi=max(psi.bond_dims()), rank_capped=max(psi.bond_dims()) >= maxdim,
                tol_step=tol_step, bond_dims=info["bond_dims"], status=info["status"], info=info)
