"""Quantics (QTT) inputs on device: grids, separable fields and the Heston generator.

Host-side builders of the ``:none``-symmetry workloads (the Heston PDE on a quantics grid). Cores
are formed with numpy once, on the host, and uploaded; the BUG step then runs on device. Follows
the reference's conventions:

* ``qtt_grid`` (``src/QTTS/Tooling/grid.jl:152-168``), the default GROUPED ordering with the least
  significant bit first (``grid.jl:1-12``): site ``k + 1`` holds bit ``k`` of the x index and site
  ``nx + k + 1`` bit ``k`` of the y index;
* fields: ``tt_from_samples`` (TT-SVD with the ``_qtt_rank`` rule, ``src/QTTS/Tooling/
  cores.jl:18-28,52-90``) and ``qtt_separable`` (``cores.jl:265-270``); ``qtt_mps``
  (``src/QTTS/Tooling/state_adapter.jl:72-82``);
* operators: cores ``(w_l, out, in, w_r)``; the shift ``(S psi)_i = psi_{i+1}`` as a binary carry
  automaton with the carry on the bond (``src/QTTS/Tooling/derivatives.jl:21-36``), central
  differences as sums of shifts, the ``:onesided`` boundary rows as rank-1 corrections
  (``derivatives.jl:40-83``), coordinate diagonals of rank 2, products and sums of chains and
  their compression (``src/QTTS/Tooling/mpo_algebra.jl``, ``cores.jl:92-128``);
* ``heston_op`` / ``heston_mpo`` (``src/QTTS/Models/Heston/heston.jl:36-69``) and ``qtt_to_mpo``
  (``state_adapter.jl:96-109``): the solver MPO stores ``(w_l, in, out, w_r)``.

Nothing here forms an object of size ``2^n``: every operator is assembled core by core.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .models import MPO, MPS
from .tensor import Leg, from_blocks


@dataclass(frozen=True)
class Grid:
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
    """The grid on ``x[0] <= x < x[1]`` (periodic) or ``x[0] <= x <= x[1]`` (end points on the
    grid), likewise in y."""
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


@dataclass(frozen=True)
class HestonParams:
    """Rate, dividend yield, mean reversion, long-run variance, vol of vol, correlation."""

    r: float
    q: float
    kappa: float
    theta: float
    sigma: float
    rho: float

    def feller(self) -> bool:
        return 2 * self.kappa * self.theta >= self.sigma ** 2


# ── fields ──────────────────────────────────────────────────────────────────────────────────

def _tail_rank(S, delta):
    r = len(S)
    tail = 0.0
    while r > 1 and tail + S[r - 1] ** 2 <= delta ** 2:
        tail += S[r - 1] ** 2
        r -= 1
    return r


def tt_from_samples(vals, tol=1e-14):
    """1D quantics TT of ``vals[i] = f(x_i)``: cores ``(chi_l, 2, chi_r)``, bit 0 first."""
    vals = np.asarray(vals, dtype=np.complex128)
    n = int(round(np.log2(len(vals))))
    if 2 ** n != len(vals):
        raise ValueError(f"need 2^n samples, got {len(vals)}")
    # row index = bit 0, the remaining bits along the columns
    M = vals.reshape((2,) * n, order="F").reshape(2, -1)
    delta = tol * np.linalg.norm(vals) / np.sqrt(max(n - 1, 1))
    cores, chi = [], 1
    for _ in range(n - 1):
        M = M.reshape(chi * 2, -1)
        U, S, Vh = np.linalg.svd(M, full_matrices=False)
        r = _tail_rank(S, delta)
        cores.append(U[:, :r].reshape(chi, 2, r))
        M = S[:r, None] * Vh[:r]
        chi = r
    cores.append(M.reshape(chi, 2, 1))
    return cores


def qtt_separable(g: Grid, fx, fy, tol=1e-14):
    """``fx(x) fy(y)``: two 1D TTs placed on the grouped ordering (x sites, then y sites)."""
    xs, ys = coords(g)
    return tt_from_samples([fx(x) for x in xs], tol) + tt_from_samples([fy(y) for y in ys], tol)


def qtt_mps(cores, center=1) -> MPS:
    """The device state of TT ``cores``: one dense block per site, uploaded, then gauged to site 1
    and on to ``center`` by exact SVD moves on device."""
    from .models import canonical

    ts = []
    for c in cores:
        c = np.asarray(c, dtype=np.complex128)
        legs = [Leg(-1, {0: c.shape[0]}), Leg(-1, {0: 2}), Leg(+1, {0: c.shape[2]})]
        ts.append(from_blocks(legs, {(0, 0, 0): c}))
    psi = MPS(ts, len(ts))
    canonical(psi, 1)
    canonical(psi, center)
    return psi


# ── operator chains: cores (w_l, out, in, w_r) ───────────────────────────────────────────────

def op_identity(n):
    return [np.eye(2, dtype=np.complex128).reshape(1, 2, 2, 1) for _ in range(n)]


def op_shift(n, periodic=False):
    """``(S psi)_i = psi_{i+1}``: bit k of the input is bit k of the output plus the carry from
    bit k-1; the +1 enters at bit 0 and the carry out of the top bit wraps (periodic) or is lost."""
    core = np.zeros((2, 2, 2, 2), dtype=np.complex128)  # [carry_in, out, in, carry_out]
    for cin in range(2):
        for o in range(2):
            s = o + cin
            core[cin, o, s % 2, s // 2] = 1.0
    cores = [core.copy() for _ in range(n)]
    cores[0] = cores[0][1:2]
    cores[-1] = cores[-1].sum(axis=3, keepdims=True) if periodic else cores[-1][:, :, :, 0:1]
    return cores


QTT_BCS = ("periodic", "dirichlet0", "onesided")  # derivatives.jl:15


def qtt_shift(n, bc="periodic"):
    """``qtt_shift(n; bc = :periodic)`` (``derivatives.jl:23-40``): ``(S psi)_i = psi_{i+1}`` on
    ``n`` bits; ``periodic`` wraps ``2^n - 1`` onto 0, any other boundary leaves the last row zero.
    The backward shift is ``op_transpose(qtt_shift(n, bc))``."""
    if n < 1:
        raise ValueError("qtt_shift needs n >= 1")
    return op_shift(n, periodic=bc == "periodic")


def qtt_derivative(n, h, order=1, bc="periodic"):
    """``qtt_derivative(n, h; order = 1, bc = :periodic)`` (``derivatives.jl:53-83``): the
    second-order central difference of ``order`` 1 or 2 with boundary ``bc`` (one of ``QTT_BCS``);
    ``onesided`` needs at least four points."""
    if bc not in QTT_BCS:
        raise ValueError(f"bc must be one of {QTT_BCS}, got :{bc}")
    if order not in (1, 2):
        raise ValueError(f"order must be 1 or 2, got {order}")
    return op_derivative(n, h, order=order, bc=bc)


def op_transpose(ch):
    return [c.transpose(0, 2, 1, 3).copy() for c in ch]


def op_scale(ch, a):
    out = [c.copy() for c in ch]
    out[0] = out[0] * a
    return out


def op_sum(chains):
    """Direct sum: block-diagonal inner cores, boundary cores concatenated along the bond."""
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


def op_compress(ch, tol=1e-14):
    """Left QR sweep, right-to-left SVD sweep keeping each bond's smallest rank whose tail fits
    ``tol * |chain| / sqrt(L - 1)`` (cores read as d = 4)."""
    C = [c.reshape(c.shape[0], 4, c.shape[3]).astype(np.complex128) for c in ch]
    L = len(C)
    if L == 1:
        return [c.reshape(c.shape[0], 2, 2, c.shape[2]) for c in C]
    for k in range(L - 1):
        chi, d, r = C[k].shape
        Q, R = np.linalg.qr(C[k].reshape(chi * d, r))
        C[k] = Q.reshape(chi, d, Q.shape[1])
        C[k + 1] = np.tensordot(R, C[k + 1], axes=(1, 0))
    delta = tol * np.linalg.norm(C[-1]) / np.sqrt(L - 1)
    for k in range(L - 1, 0, -1):
        chi, d, r = C[k].shape
        U, S, Vh = np.linalg.svd(C[k].reshape(chi, d * r), full_matrices=False)
        rr = _tail_rank(S, delta)
        C[k] = Vh[:rr].reshape(rr, d, r)
        C[k - 1] = np.tensordot(C[k - 1], U[:, :rr] * S[:rr], axes=(2, 0))
    return [c.reshape(c.shape[0], 2, 2, c.shape[2]) for c in C]


def op_lincomb(terms, tol=1e-14):
    return op_compress(op_sum([op_scale(ch, a) for a, ch in terms]), tol)


def op_compose(A, B, tol=1e-14):
    """``A B`` (apply B first): bonds multiply, the inner index is summed."""
    out = []
    for a, b in zip(A, B):
        c = np.einsum("aomr,bmis->aboirs", a, b)
        out.append(c.reshape(a.shape[0] * b.shape[0], 2, 2, a.shape[3] * b.shape[3]))
    return op_compress(out, tol)


def op_ket_bra(n, row, col):
    """``|row><col|`` on n bits (rank 1)."""
    out = []
    for k in range(n):
        c = np.zeros((1, 2, 2, 1), dtype=np.complex128)
        c[0, (row >> k) & 1, (col >> k) & 1, 0] = 1.0
        out.append(c)
    return out


def op_coord_diag(n, x0, dx):
    """``diag(x0 + dx i)``: rank 2, the bond carries (1, partial sum)."""
    out = []
    for k in range(n):
        c = np.zeros((2, 2, 2, 2), dtype=np.complex128)
        for b in range(2):
            c[0, b, b, 0] = 1.0
            c[0, b, b, 1] = dx * (2 ** k) * b
            c[1, b, b, 1] = 1.0
        out.append(c)
    out[0] = out[0][0:1].copy()
    out[0][0, :, :, 1] += x0 * np.eye(2)
    out[-1] = out[-1][:, :, :, 1:2].copy()
    return out


_ONESIDED = {1: ([-3.0, 4.0, -1.0], [1.0, -4.0, 3.0]),
             2: ([2.0, -5.0, 4.0, -1.0], [-1.0, 4.0, -5.0, 2.0])}


def op_derivative(n, h, order=1, bc="onesided"):
    """Second-order differences on ``2^n`` points of spacing h: the central ``(S+ - S-)/2h`` or
    ``(S+ - 2I + S-)/h^2``. ``dirichlet0`` drops what leaves the box; ``onesided`` adds rank-1
    corrections turning the first and last rows into the one-sided second-order stencils."""
    if bc not in ("periodic", "dirichlet0", "onesided"):
        raise ValueError(f"bad boundary condition {bc!r}")
    fwd = op_shift(n, periodic=bc == "periodic")
    bwd = op_transpose(fwd)
    if order == 1:
        central = op_lincomb([(1 / (2 * h), fwd), (-1 / (2 * h), bwd)])
        crow = {1: 1 / (2 * h), -1: -1 / (2 * h)}
        scale = 1 / (2 * h)
    elif order == 2:
        central = op_lincomb([(1 / h ** 2, fwd), (-2 / h ** 2, op_identity(n)), (1 / h ** 2, bwd)])
        crow = {1: 1 / h ** 2, 0: -2 / h ** 2, -1: 1 / h ** 2}
        scale = 1 / h ** 2
    else:
        raise ValueError(f"order must be 1 or 2, got {order}")
    if bc != "onesided":
        return central
    N = 2 ** n
    if N < 4:
        raise ValueError(":onesided stencils need at least 4 points")
    first, last = _ONESIDED[order]
    patch = {}
    for j, w in enumerate(first):            # row 0: the one-sided stencil minus the central row
        patch[(0, j)] = patch.get((0, j), 0.0) + w * scale
    for off, w in crow.items():
        if 0 <= off < N:
            patch[(0, off)] = patch.get((0, off), 0.0) - w
    for j, w in enumerate(last):             # row N-1
        col = N - len(last) + j
        patch[(N - 1, col)] = patch.get((N - 1, col), 0.0) + w * scale
    for off, w in crow.items():
        col = N - 1 + off
        if 0 <= col < N:
            patch[(N - 1, col)] = patch.get((N - 1, col), 0.0) - w
    terms = [(1.0, central)] + [(v, op_ket_bra(n, r, c)) for (r, c), v in sorted(patch.items())
                                if v != 0.0]
    return op_lincomb(terms)


def heston_cores(g: Grid, p: HestonParams, adjoint=False, tol=1e-14):
    """``A_H = v/2 d_xx + rho sigma v d_xv + sigma^2 v/2 d_vv + (r - q - v/2) d_x
    + kappa (theta - v) d_v - r`` as operator cores on the grid's sites (``heston.jl:36-61``);
    ``adjoint``: the forward-density operator (transpose, no discount)."""
    if g.periodic_x or g.periodic_y:
        raise ValueError("heston_op: build the grid with periodic_x = periodic_y = false")
    if abs(g.y0) >= 1e-14:
        raise ValueError("heston_op: the variance grid must start at v = 0")
    d1x, d2x = op_derivative(g.nx, g.dx, 1), op_derivative(g.nx, g.dx, 2)
    d1v, d2v = op_derivative(g.ny, g.dy, 1), op_derivative(g.ny, g.dy, 2)
    var = op_coord_diag(g.ny, g.y0, g.dy)
    var_d1v, var_d2v = op_compose(var, d1v), op_compose(var, d2v)
    ix, iv = op_identity(g.nx), op_identity(g.ny)
    terms = [
        (0.5, d2x, var),
        (p.rho * p.sigma, d1x, var_d1v),
        (0.5 * p.sigma ** 2, ix, var_d2v),
        (p.r - p.q, d1x, iv),
        (-0.5, d1x, var),
        (p.kappa * p.theta, ix, d1v),
        (-p.kappa, ix, var_d1v),
    ]
    if not adjoint:
        terms.append((-p.r, ix, iv))
    chain = op_lincomb([(a, ax + av) for a, ax, av in terms], tol)
    return op_transpose(chain) if adjoint else chain


def cores_to_mpo(cores) -> MPO:
    """The solver MPO of operator cores: stored as ``(w_l, in, out, w_r)`` with arrows
    ``(w_l:-1, s_in:+1, s_out:-1, w_r:+1)``, one dense block per site."""
    ts = []
    for c in cores:
        W = np.ascontiguousarray(np.asarray(c, dtype=np.complex128).transpose(0, 2, 1, 3))
        legs = [Leg(-1, {0: W.shape[0]}), Leg(+1, {0: 2}), Leg(-1, {0: 2}), Leg(+1, {0: W.shape[3]})]
        ts.append(from_blocks(legs, {(0, 0, 0, 0): W}))
    return MPO(ts)


def heston_mpo(g: Grid, p: HestonParams, adjoint=False) -> MPO:
    """``heston_mpo(g, params)`` (``heston.jl:69``): the generator as the solver MPO on device."""
    return cores_to_mpo(heston_cores(g, p, adjoint))


def heston_op(g: Grid, p: HestonParams, adjoint=False):
    """``heston_op(g, params)`` (``heston.jl:36-61``): the generator as host operator cores."""
    return heston_cores(g, p, adjoint)


def qtt_to_mpo(cores) -> MPO:
    """``qtt_to_mpo`` (``state_adapter.jl:96-109``): operator cores as the solver MPO on device."""
    return cores_to_mpo(cores)


# ── the QTT BUG step of a linear flow (src/QTTS/Tooling/nonlinear_step.jl) ───────────────────

QTT_KRYLOV_MARGIN = 0.5       # _QTT_KRYLOV_MARGIN, nonlinear_step.jl:8
QTT_RATIONAL_MAXITER = 200    # _QTT_RATIONAL_MAXITER, nonlinear_step.jl:17
QTT_TOL_FLOOR = 1e-14         # _QTT_TOL_FLOOR, nonlinear_step.jl:23
_QTT_ROOTS = {2: "trapezoid", 3: "radau2", 4: "radau3"}  # qtt_root_for_order, stage_solvers.jl:161-165


def qtt_step_tolerance(tol, h, order, scaling="order", h_ref=0.1):
    """``qtt_step_tolerance`` (``nonlinear_step.jl:25-47``): the per-step value of a tolerance,
    ``tol (|h| / h_ref)^(order + 1)`` (never looser than ``tol``) floored at 1e-14 unless ``tol``
    is already below it; ``scaling = "fixed"`` returns ``tol``."""
    if scaling not in ("order", "fixed"):
        raise ValueError(f"tol_scaling must be :order or :fixed, got :{scaling}")
    if not h_ref > 0:
        raise ValueError(f"tol_h_ref must be positive, got {h_ref}")
    if scaling == "fixed" or tol == 0:
        return float(tol)
    factor = min(1.0, (abs(float(h)) / float(h_ref)) ** (order + 1))
    return max(float(tol) * factor, min(float(tol), QTT_TOL_FLOOR))


def qtt_root_for_order(order):
    """The rational root of BUG order 2, 3, 4: trapezoid, Radau IIA (2 stages), Radau IIA (3)."""
    if order not in _QTT_ROOTS:
        raise ValueError(f"nonlinear BUG orders are 2, 3, 4; got {order}")
    return _QTT_ROOTS[order]


def qtt_bug_step(psi, mpo, t, h, *, pref=1.0, order=2, root=None, tol_stage=1e-10, tol_basis=1e-6,
                 tol_trunc=1e-8, maxdim=128, stage_solver="auto", tol_scaling="order",
                 tol_h_ref=0.1, tol_krylov=None, rng=None, **kwargs):
    """``qtt_bug_step!(psi, fl, t, h; ...)`` (``src/QTTS/Tooling/nonlinear_step.jl:102-371``) for a
    linear flow ``F = pref H psi`` with ``H`` the operator of ``mpo`` (``LinearFlow``,
    ``src/BUG/TimeEvolution/flows.jl:20-31``), in place on the device. For a linear flow
    ``stage_solver = "auto"`` is ``krylov_rational``: one native BUG step (``bug_mps_step``) at
    ``order`` whose root is the rational stability function ``root`` (trapezoid / Radau IIA) of
    the Galerkin operator on its Arnoldi basis, applied unshifted (``root_shift = False``, at most
    200 Arnoldi vectors), then compressed; the tolerances are ``qtt_step_tolerance`` values. The
    Newton-GMRES stage equations of nonlinear flows (``stage_solver = "newton_gmres"``) are not built.
    ``t`` is the start time (a linear flow does not depend on it). Returns the step report:
    ``converged`` (the root's Krylov error within the stage tolerance), ``residual``, ``krylov``,
    ``discarded``, ``chi``, ``rank_capped``, ``tol_step`` and the step's ``info``."""
    if stage_solver not in ("auto", "krylov_rational", "newton_gmres"):
        raise ValueError("stage_solver must be :auto, :newton_gmres or :krylov_rational, "
                         f"got :{stage_solver}")
    if stage_solver == "newton_gmres":
        raise NotImplementedError("stage_solver = :newton_gmres (the nonlinear stage equations)")
    from .native import cbe_bug_step

    root = qtt_root_for_order(order) if root is None else root

    def st(tol):
        return qtt_step_tolerance(tol, h, order, scaling=tol_scaling, h_ref=tol_h_ref)

    tol_step = dict(basis=st(tol_basis), trunc=st(tol_trunc), stage=st(tol_stage),
                    scaling=tol_scaling, h_ref=float(tol_h_ref))
    tol_kry = st(QTT_KRYLOV_MARGIN * tol_basis if tol_krylov is None else tol_krylov)
    info = cbe_bug_step(psi, mpo, complex(pref * h), order=order, tol_basis=tol_step["basis"],
                        tol_trunc=tol_step["trunc"], maxdim=maxdim, hermitian=False, eshift=0.0,
                        tol_krylov=tol_kry, root_method=root, tol_root=tol_step["stage"],
                        root_shift=False, root_maxiter=QTT_RATIONAL_MAXITER, truncate=True,
                        rng=rng, **kwargs)
    err = info["ledger"].expv_err
    chi = max(psi.bond_dims())
    return dict(solver="krylov_rational", root=root, order=order, converged=err <= tol_step["stage"],
                residual=err, krylov=info["ledger"].expv_iters, discarded=info["discarded"],
                chi=chi, rank_capped=chi >= maxdim, tol_step=tol_step, bond_dims=info["bond_dims"],
                status=info["status"], info=info)
