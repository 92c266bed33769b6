"""Pins of the CPU oracle against the reference's own known answers and frozen runs.

* Test A lists: ``test/BUG/Randomised/test_expansion.jl:15-88``.
* The two-spin entangling step: ``test_expansion.jl:90-109``.
* ``expv`` against sector-diagonal closed forms, its degenerate generators, reorthogonalisation, zero
  input and the root stability functions: ``test/BUG/Core/LocalSolvers/test_krylov.jl:21-216``.
* The Krylov stopping weights (``test/BUG/Core/LocalSolvers/test_krylov_weights.jl:44-117``): the
  residual integral on the 2 x 2 where Saad's scalar cancels (weight 1), its bound on random
  Hermitian generators, the root's tail guarded over the step, ``_tridiag_eigen`` exact and naming
  non-finite input.
* The b155550 frozen trajectories, with the reference's own tolerances and settings
  (``test/BUG/TimeEvolution/test_fixtures_b155550.jl:23-97``): S^z within 1e-5 of the frozen
  profile and within ``2 err_exact + 1e-6`` of free fermions, status as frozen; the frozen runs used
  ``work_ceiling_rule = :maxdim`` and the Arnoldi recurrence.
"""

import json
import math
import os

import numpy as np
import pytest
import scipy.linalg

from oracle import blocks as B
from oracle import krylov as K
from oracle import models as M
from oracle import step as S
from oracle.budget import tail_rank

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "b155550.json")))


def mk(sig, degs=None):
    degs = degs or [1] * len(sig)
    return [(s, d, None, None) for s, d in zip(sig, degs)]


def test_tail_rank_lists():
    lst = mk([10.0, 9.0, 3.0, 0.1])
    assert tail_rank(lst, 1.0, 1.0, 4)[0] == 3
    assert tail_rank(lst, 1.0, 4.0, 4)[0] == 2
    assert tail_rank(lst, 1.0, 9.6, 4)[0] == 1
    assert tail_rank(lst, 1.0, 0.05, 4)[0] == 4
    lst = mk([1.0, 1e-2, 1e-4, 1e-6])
    k, tail = tail_rank(lst, 1.0, 2e-4, 4)
    assert k == 2 and tail <= 2e-4
    assert tail_rank(lst, 1.0, 5e-5, 4)[0] == 3
    assert tail_rank(lst, 1.0, 2e-2, 4)[0] == 1
    lst = mk([1.0, 0.5, 0.2, 0.05, 0.01, 1e-3])
    ks = [tail_rank(lst, 1.0, a, 6)[0] for a in (1e-6, 1e-3, 1e-2, 0.1, 0.5, 2.0)]
    assert ks == sorted(ks, reverse=True) and ks[0] == 6 and ks[-1] == 0
    assert tail_rank(mk([1.0, 0.1]), 1.0, 0.5, 2)[0] == 1
    assert tail_rank(mk([1.0, 0.1], [1, 100]), 1.0, 0.5, 2)[0] == 2
    lst = mk([1.0, 1e-3])
    assert tail_rank(lst, 1.0, 0.1, 2)[0] == 1
    k, tail = tail_rank(lst, 1.0, 0.1, 2, base=0.25)
    assert k == 2 and tail > 0.1
    assert tail_rank(mk([1.0, 1e-2]), 1.0, 2e-2, 2)[0] == 1
    assert tail_rank(mk([1.0, 1e-2]), 10.0, 2e-2, 2)[0] == 2
    k, tail = tail_rank(mk([1.0] * 4), 1.0, 1e-12, 2)
    assert k == 2 and tail > 1e-12
    assert tail_rank(mk([]), 1.0, 1e-3, 4)[0] == 0
    assert tail_rank(mk([1.0]), 1.0, 1e-3, 0)[0] == 0


def test_two_spin_entangling_step():
    mpo = M.xxz_mpo(2, J=1.0, delta=0.0)
    psi = M.product_state(["up", "down"])
    t = 0.3
    info = S.cbe_bug_step(psi, mpo, -1j * t, tol_basis=1e-10, tol_trunc=1e-14, tol_expv=1e-13,
                          maxdim=4)
    v = M.mps_to_dense(psi)
    v /= np.linalg.norm(v)
    assert abs(abs(v[1]) - math.cos(t / 2)) < 1e-10
    assert abs(abs(v[2]) - math.sin(t / 2)) < 1e-10
    assert info["record"]["policy"] == "dd_qr_streamed"


def _multi_sector():
    rng = np.random.default_rng(7)
    legs = [B.Leg(-1, {0: 2}), B.Leg(-1, {-1: 1, 1: 1}), B.Leg(+1, {-1: 3, 1: 2})]
    blocks = {}
    for qs in (-1, 1):
        shape = (2, 1, legs[2].sectors[qs])
        blocks[(0, qs, qs)] = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    return B.BT(legs, blocks)


def _diag(x, scale):
    return B.BT(x.legs, {k: scale(k[2]) * v for k, v in x.blocks.items()})


@pytest.mark.parametrize("tau", [-0.4 + 0j, -0.7j, 0.25 + 0.3j])
def test_expv_closed_form(tau):
    x = _multi_sector()
    scale = lambda q: 0.5 * q + 1.0
    want = B.BT(x.legs, {k: np.exp(tau * scale(k[2])) * v for k, v in x.blocks.items()})
    for herm in (True, False):
        y, rep = K.expv(K.VecOps(), lambda v: _diag(v, scale), tau, x, hermitian=herm)
        assert B.norm(B.sub(y, want)) < 1e-11


def test_arnoldi_terminates_at_true_krylov_dimension():
    x = _multi_sector()
    scale = lambda q: (0.5 * q + 1.0) + 0.3j * q
    tau = -0.35 + 0j
    want = B.BT(x.legs, {k: np.exp(tau * scale(k[2])) * v for k, v in x.blocks.items()})
    y, rep = K.expv(K.VecOps(), lambda v: _diag(v, scale), tau, x, hermitian=False, maxiter=60)
    assert B.norm(B.sub(y, want)) < 1e-12
    assert rep[0] == 2
    y, rep = K.expv(K.VecOps(), lambda v: _diag(v, scale), tau, x, hermitian=True, maxiter=60)
    assert rep[0] == 60


def test_expv_degenerate_generators():
    """``test_krylov.jl:38-58,175-179``: the identity generator gives exp(tau) x, the zero generator
    the identity, a Hermitian generator keeps the norm in real time, Arnoldi matches Lanczos on it,
    and a zero input returns zero on both paths."""
    x = _multi_sector()
    ops = K.VecOps()
    y, _ = K.expv(ops, lambda v: v, -1.0 + 0j, x, hermitian=True)
    assert B.norm(B.sub(y, B.scale(x, np.exp(-1.0)))) < 1e-12
    y, _ = K.expv(ops, lambda v: B.scale(v, 0.0), -0.1j, x, hermitian=True)
    assert B.norm(B.sub(y, x)) < 1e-14
    y, _ = K.expv(ops, lambda v: B.scale(v, 2.0), -0.3j, x, hermitian=True)
    assert abs(B.norm(y) - B.norm(x)) < 1e-12
    yl, _ = K.expv(ops, lambda v: B.scale(v, 2.0), -0.2j, x, hermitian=True)
    ya, _ = K.expv(ops, lambda v: B.scale(v, 2.0), -0.2j, x, hermitian=False)
    assert B.norm(B.sub(yl, ya)) < 1e-11
    z = B.scale(x, 0.0)
    for herm in (True, False):
        y, _ = K.expv(ops, lambda v: B.scale(v, 2.0), -0.1j, z, hermitian=herm)
        assert B.norm(y) < 1e-15


def test_lanczos_reorthogonalisation_spans_the_same_space():
    """``test_krylov.jl:126-131``: full reorthogonalisation changes nothing on a diagonal generator."""
    x = _multi_sector()
    scale = lambda q: 0.5 * q + 1.0
    y0, _ = K.expv(K.VecOps(), lambda v: _diag(v, scale), -0.5j, x, hermitian=True, reorth=False)
    y1, _ = K.expv(K.VecOps(), lambda v: _diag(v, scale), -0.5j, x, hermitian=True, reorth=True)
    assert B.norm(B.sub(y0, y1)) < 1e-11


def test_inner_is_zero_when_no_blocks_match():
    """``test_krylov.jl:181-191``: stored sectors disjoint on equal spaces give 0, not an error."""
    x = _multi_sector()
    a = B.BT(x.legs, {k: v for k, v in x.blocks.items() if k[2] == -1})
    b = B.BT(x.legs, {k: v for k, v in x.blocks.items() if k[2] == 1})
    assert B.inner(a, b) == 0
    assert B.inner(a, a) != 0


def test_root_stability_functions():
    """``test_krylov.jl:194-216``: A-stability on the negative axis and the imaginary axis, the
    classical order from the error ratio, L-stability of the Radau roots, the trapezoid's -1 limit,
    damping of stiff scalars."""
    zs = list(-(10.0 ** np.linspace(-3, 8, 60))) + [0.0]
    for m, q in (("trapezoid", 2), ("radau2", 3), ("radau3", 5)):
        assert all(abs(K.root_stability(m, z)) <= 1 + 1e-14 for z in zs)
        assert all(abs(K.root_stability(m, 1j * y)) <= 1 + 1e-12 for y in np.arange(-50, 50.5, 0.5))
        err = lambda z: abs(K.root_stability(m, z) - np.exp(z))
        assert abs(math.log2(err(-0.1) / err(-0.05)) - (q + 1)) < 0.25
        for lh in (0.1, 10.0, 1e4):
            assert abs(K.root_stability(m, -lh)) < 1
    assert abs(K.root_stability("radau2", -1e8)) < 1e-6
    assert abs(K.root_stability("radau3", -1e8)) < 1e-6
    assert abs(K.root_stability("trapezoid", -1e8) + 1) < 1e-6
    assert K.root_stability("exp", -0.3) == pytest.approx(math.exp(-0.3))


FROZEN = dict(work_ceiling_rule="maxdim", expansion=S.DDQRExpansion(krylov_mode="arnoldi"))


@pytest.mark.parametrize("name,order", [("xx_u1_bug_order1", 1), ("xx_u1_bug_order2", 2)])
def test_b155550_u1(name, order):
    fz = GOLDEN[name]
    L, dt = fz["L"], fz["dt"]
    mpo = M.xxz_mpo(L, J=1.0, delta=0.0)
    psi = M.neel_state(L)
    rng = np.random.default_rng(1234)
    for step, row in enumerate(fz["trajectory"][:3], start=1):
        info = S.cbe_bug_step(psi, mpo, -1j * dt, order=order, rng=rng, **FROZEN)
        sz = M.sz_profile(psi)
        exact = M.free_fermion_sz(L, step * dt, occupied=range(0, L, 2))
        assert np.max(np.abs(sz - np.array(row["sz"]))) <= 1e-5
        assert np.max(np.abs(sz - exact)) <= 2 * row["err_exact"] + 1e-6
        assert info["status"] == row["status"]


def test_b155550_none():
    fz = GOLDEN["xx_none_bug_order2"]
    L, dt = fz["L"], fz["dt"]
    mpo = M.xxz_mpo(L, J=1.0, delta=0.0, symmetry="none")
    psi = M.neel_state(L, symmetry="none")
    v0 = M.mps_to_dense(psi)
    rng = np.random.default_rng(1234)
    for row in fz["trajectory"][:3]:
        info = S.cbe_bug_step(psi, mpo, -1j * dt, order=2, rng=rng, **FROZEN)
        assert info["status"] == row["status"]
        assert abs(B.norm(psi[psi.center]) - row["norm"]) <= 1e-8
    H = M.dense_xxz(L, 1.0, 0.0)
    ex = scipy.linalg.expm(-1j * 3 * dt * H) @ v0
    err = np.linalg.norm(M.mps_to_dense(psi) - ex) / np.linalg.norm(ex)
    assert err <= 2 * fz["err_dense"] + 1e-6


@pytest.mark.parametrize("name,order,min_dims", [("xx_u1_bug_order1", 1, 20), ("xx_u1_bug_order2", 2, 19)])
def test_b155550_adaptive_mode(name, order, min_dims):
    """The fixtures were frozen with the :adaptive DD controller (two-pass pivoted thin QR,
    holdout-checked widths). In that mode the restatement reproduces the frozen runs' bond
    dimensions at 20 of 20 (order 1) and 19 of 20 (order 2) steps and S^z within 1e-7, though its
    Gaussian draws differ from the reference's."""
    fz = GOLDEN[name]
    L, dt = fz["L"], fz["dt"]
    mpo = M.xxz_mpo(L, J=1.0, delta=0.0)
    psi = M.neel_state(L)
    rng = np.random.default_rng(1234)
    same_dims = 0
    for step, row in enumerate(fz["trajectory"], start=1):
        info = S.cbe_bug_step(psi, mpo, -1j * dt, order=order, rng=rng, work_ceiling_rule="maxdim",
                              expansion=S.DDQRExpansion(krylov_mode="arnoldi", mode="adaptive"))
        assert np.max(np.abs(M.sz_profile(psi) - np.array(row["sz"]))) <= 1e-7
        assert info["status"] == row["status"]
        same_dims += psi.bond_dims() == row["bond_dims"]
    assert same_dims >= min_dims


def test_thin_qr_against_scipy_pivoted():
    """The thin QR keeps the numerical rank of each sector, with R_kk real positive."""
    from oracle import cbe as C

    rng = np.random.default_rng(4)
    legs = [B.Leg(-1, {0: 6, 2: 4}), B.Leg(-1, {-1: 1, 1: 1}), B.Leg(+1, {-1: 3, 1: 5})]
    blocks = {}
    for key in [(0, -1, -1), (0, 1, 1), (2, -1, 1)]:
        shp = tuple(l.sectors[q] for l, q in zip(legs, key))
        blocks[key] = rng.standard_normal(shp) + 1j * rng.standard_normal(shp)
    for key in [(0, 1, 1), (2, -1, 1)]:  # column 4 of sector +1 depends on column 0
        blocks[key][..., 4] = blocks[key][..., 0] * 2.0
    T = B.BT(legs, blocks)
    Q = C.thin_qr(T, 2, +1, 1e-10)
    assert Q.legs[2].sectors == {-1: 3, 1: 4}  # sector +1: 10 rows, 5 columns of rank 4
    for c, (_, _, _, _, M_) in B.sector_matrix(Q, (0, 1)).items():
        assert np.allclose(M_.conj().T @ M_, np.eye(M_.shape[1]), atol=1e-12)


def test_pivoted_qr_is_geqp3_on_distinct_norms():
    """Where column norms are distinct, the restated pivoted QR is LAPACK geqp3's factorisation:
    the same pivots, |R_kk| and Q columns (phase-fixed) as scipy, tall, wide and square."""
    import scipy.linalg as sla
    from oracle import cbe as C

    rng = np.random.default_rng(3)
    for m, n in [(12, 7), (5, 9), (30, 30), (40, 3)]:
        A = rng.standard_normal((m, n)) + 1j * rng.standard_normal((m, n))
        A *= np.geomspace(1, 1e-4, n)[None, rng.permutation(n)]
        Q, r = C.pivoted_qr(A)
        Qs, Rs, _ = sla.qr(A, mode="economic", pivoting=True)
        d = np.diag(Rs)
        assert np.max(np.abs(Q - Qs * (d / np.abs(d))[None, :])) < 1e-13
        assert np.max(np.abs(r - np.abs(d))) < 1e-14 * np.abs(d).max()


def test_pivoted_qr_tie_rule():
    """Orthonormal columns (every norm 1 to rounding): the tie rule keeps the given order, so Q is
    the input up to the R_kk >= 0 phase."""
    from oracle import cbe as C

    rng = np.random.default_rng(5)
    X, _ = np.linalg.qr(rng.standard_normal((20, 6)) + 1j * rng.standard_normal((20, 6)))
    Q, r = C.pivoted_qr(X)
    assert np.allclose(r, 1.0, atol=1e-14)
    ph = np.array([np.vdot(Q[:, j], X[:, j]) for j in range(6)])
    assert np.allclose(np.abs(ph), 1.0, atol=1e-13)


def test_tdvp2_baseline_fixture():
    """The two-site TDVP restatement against the reference's frozen ``baseline_tdvp2_xx`` run
    (L = 10 XX from Neel, dt 0.05, maxdim 64, trunc_thresh 1e-12), with the bars of
    ``test/Baselines/test_baselines.jl`` (S^z within 1e-5 of the frozen run and within
    2 err_exact + 1e-6 of free fermions) and, tighter, the frozen bond dimensions and S^z to
    1e-12."""
    from oracle import tdvp as T

    fz = GOLDEN["baseline_tdvp2_xx"]
    L, dt = fz["L"], fz["dt"]
    psi = M.neel_state(L)
    mpo = M.xxz_mpo(L, J=1.0, delta=0.0)
    for step, row in enumerate(fz["trajectory"][:4], start=1):
        T.tdvp2_step(psi, mpo, -1j * dt, maxdim=64, trunc_thresh=1e-12)
        sz = M.sz_profile(psi)
        exact = M.free_fermion_sz(L, step * dt, occupied=range(0, L, 2))
        assert np.max(np.abs(sz - np.array(row["sz"]))) <= 1e-12
        assert np.max(np.abs(sz - exact)) <= 2 * row["err_exact"] + 1e-6
        assert psi.bond_dims() == row["bond_dims"]


def test_ite_heisenberg_fixture():
    """Normalised imaginary time (``ite_evolve!``, two steps of dbeta 0.125 per row) on the
    Heisenberg chain from Neel, under the defaults the reference froze ``heisenberg_ite`` with
    (``:adaptive`` DD, Arnoldi, the ``:maxdim`` ceiling): the frozen energies to 1e-12 at
    beta 0.25 and 0.5 and 1e-8 at 0.75 and 1, the frozen statuses, monotone decrease and never
    below the ground state (the reference test's bars)."""
    from oracle import ite as I

    fz = GOLDEN["heisenberg_ite"]
    L = fz["L"]
    mpo = M.xxz_mpo(L, J=1.0, delta=1.0)
    psi = M.neel_state(L)
    rng = np.random.default_rng(1234)
    kw = dict(work_ceiling_rule="maxdim", expansion=S.DDQRExpansion(mode="adaptive", krylov_mode="arnoldi"))
    prev = np.inf
    for i, row in enumerate(fz["trajectory"][:4]):
        hist = I.ite_evolve(psi, mpo, I.uniform_beta_steps(0.25, 2), order=2, rng=rng, **kw)
        e = I.ite_energy(psi, mpo)
        assert abs(e - row["energy"]) <= (1e-12 if i < 2 else 1e-8), (row["beta"], e, row["energy"])
        assert [h["status"] for h in hist] == row["status"]
        assert e < prev and e >= fz["e_exact_ground"] - 1e-10
        prev = e


def test_ite_schedules():
    """``log_panel_steps`` / ``uniform_beta_steps`` / ``geometric_schedule`` (``schedules.jl``)."""
    from oracle import ite as I

    s = I.log_panel_steps(8.0, 3, per_panel=4)
    assert len(s) == 12 and abs(sum(s) - 8.0) < 1e-12
    assert s[:4] == [0.5] * 4 and s[4:8] == [0.5] * 4 and s[8:] == [1.0] * 4
    assert I.beta_grid([0.5, 0.25])[-1] == 0.75
    assert I.uniform_beta_steps(2.0, 8) == [0.25] * 8
    assert I.geometric_schedule(0.1, 2.0, 0.5, 4) == [0.1, 0.2, 0.4, 0.5]


@pytest.mark.parametrize("method", ["trapezoid", "radau2", "radau3"])
@pytest.mark.parametrize("tau", [-0.7j, -0.4 + 0j])
def test_implicit_roots_closed_form(method, tau):
    """The implicit roots apply their stability function R(z) exactly when the Krylov space is
    complete: R(tau A) x in real time, R(tau (A - sigma)) x in imaginary time with sigma the
    eigenvalue maximising Re(tau lambda) (the reference's spectral shift), for Lanczos and
    Arnoldi; R is the (k, k+1) Pade approximant (R(z) - exp(z) = O(z^(2k+2)))."""
    x = _multi_sector()
    scale = lambda q: 0.5 * q + 1.0
    lam = {k: scale(k[2]) for k in x.blocks}
    sigma = max(lam.values(), key=lambda v: (tau * v).real) if tau.real != 0 else 0.0
    want = B.BT(x.legs, {k: K.root_stability(method, tau * (lam[k] - sigma)) * v
                         for k, v in x.blocks.items()})
    for herm in (True, False):
        y, _ = K.expv(K.VecOps(), lambda v: _diag(v, scale), tau, x, hermitian=herm,
                      root_method=method)
        assert B.norm(B.sub(y, want)) < 1e-12 * B.norm(want)
    order = {"trapezoid": 2, "radau2": 3, "radau3": 5}[method]
    z = 1e-2
    assert abs(K.root_stability(method, z) - np.exp(z)) < 10 * z ** (order + 1)


@pytest.mark.parametrize("tau", [-0.7j, -0.4 + 0j])
def test_radau2_gmres_is_radau2(tau):
    """The coupled-stage Radau IIA(2) solved by shifted GMRES converges to the same step as the
    rational ``radau2`` root: R(tau (A - sigma)) x on a diagonal operator, with the stage residual
    it reports at rounding level."""
    x = _multi_sector()
    scale = lambda q: 0.5 * q + 1.0
    lam = {k: scale(k[2]) for k in x.blocks}
    sigma = max(lam.values(), key=lambda v: (tau * v).real) if tau.real != 0 else 0.0
    want = B.BT(x.legs, {k: K.root_stability("radau2", tau * (lam[k] - sigma)) * v
                         for k, v in x.blocks.items()})
    y, rep = K.expv(K.VecOps(), lambda v: _diag(v, scale), tau, x, hermitian=True,
                    root_method="radau2_gmres", conv_tol=1e-12)
    assert B.norm(B.sub(y, want)) < 1e-12 * B.norm(want)
    assert rep[2] < 1e-12


# ── the Krylov stopping weights (test_krylov_weights.jl) ─────────────────────────────────────


def _krylov_module(which):
    """The oracle's Krylov routines."""
    from oracle import krylov

    return krylov


def _arnoldi(H, seed, depth):
    """Plain Arnoldi with two Gram-Schmidt passes, the test's own recurrence (not the oracle's)."""
    basis = np.zeros((len(seed), depth + 1), dtype=np.complex128)
    hess = np.zeros((depth + 1, depth + 1), dtype=np.complex128)
    basis[:, 0] = seed / np.linalg.norm(seed)
    for step in range(depth):
        image = H @ basis[:, step]
        for _ in range(2):
            proj = basis[:, : step + 1].conj().T @ image
            hess[: step + 1, step] += proj
            image = image - basis[:, : step + 1] @ proj
        hess[step + 1, step] = np.linalg.norm(image)
        basis[:, step + 1] = image / hess[step + 1, step]
    return basis, hess


def _krylov_error(H, seed, tau, basis, hess, depth):
    exact = scipy.linalg.expm(tau * H) @ seed
    reduced = scipy.linalg.expm(tau * hess[:depth, :depth])[:, 0]
    return np.linalg.norm(exact - basis[:, :depth] @ reduced)


@pytest.mark.parametrize("which", ["oracle"])
def test_kry_weight_does_not_cancel_on_two_by_two(which):
    """|tau| beta int_0^1 |exp(-2 pi i s)| ds = 1 where one direction leaves an O(1) error."""
    K = _krylov_module(which)
    H = np.array([[2 * np.pi, 1], [1, 0]], dtype=np.complex128)
    seed = np.array([1, 0], dtype=np.complex128)
    basis, hess = _arnoldi(H, seed, 1)
    err = _krylov_error(H, seed, -1j, basis, hess, 1)
    w = K.kry_weight(hess, 1, -1j)
    assert err > 0.1
    assert w == pytest.approx(1.0, rel=1e-10)
    assert w >= err


@pytest.mark.parametrize("which", ["oracle"])
def test_kry_weight_bounds_random_hermitian_errors(which):
    K = _krylov_module(which)
    rng = np.random.default_rng(11)
    dim, depth, checked = 30, 16, 0
    for _ in range(3):
        for tau in (-0.1j, -1j, -3j):
            raw = rng.standard_normal((dim, dim)) + 1j * rng.standard_normal((dim, dim))
            H = (raw + raw.conj().T) / 2
            seed = rng.standard_normal(dim) + 1j * rng.standard_normal(dim)
            seed /= np.linalg.norm(seed)
            basis, hess = _arnoldi(H, seed, depth)
            for step in range(1, depth):
                err = _krylov_error(H, seed, tau, basis, hess, step)
                if err < 1e-13:
                    break
                checked += 1
                assert err <= (1 + 1e-3) * K.kry_weight(hess, step, tau) + 1e-14, (tau, step)
    assert checked > 30


@pytest.mark.parametrize("which", ["oracle"])
def test_root_tail_is_guarded_over_the_step(which):
    """T_2 = [0 pi; pi 0] from e_1 on [0 pi 0; pi 0 1; 0 1 0]: [exp(-i T_2)]_{2,1} = -i sin(pi) = 0,
    so the endpoint tail vanishes with an O(1) error; the guarded tail samples |sin(pi s)|."""
    K = _krylov_module(which)
    chain = np.array([[0, np.pi, 0], [np.pi, 0, 1], [0, 1, 0]], dtype=np.complex128)
    tau = -1j
    vals, vecs = K.tridiag_eigen([0.0, 0.0], [np.pi])

    def evalcoeff(step):
        return K.coeffs_from_eigen(vals, vecs, complex(step))

    endpoint = K.tail(evalcoeff(tau)[0], 1.0)
    guarded = K.tail_sup(evalcoeff, complex(tau), 1.0)
    true_err = np.linalg.norm(scipy.linalg.expm(tau * chain) @ np.array([1, 0, 0])
                              - np.concatenate([evalcoeff(tau)[0], [0]]))
    assert true_err > 0.1
    assert endpoint < 1e-12
    assert guarded >= 0.9
    assert abs(tau) * guarded >= true_err
    for step in (-0.3j, -2.7j):
        assert K.tail_sup(evalcoeff, step, 1.0) >= K.tail(evalcoeff(step)[0], 1.0)
    for step in (-0.5 + 0j, -0.5 - 1j):  # imaginary time and loss keep the endpoint value
        assert K.tail_sup(evalcoeff, step, 1.0) == K.tail(evalcoeff(step)[0], 1.0)


@pytest.mark.parametrize("which", ["oracle"])
def test_tridiag_eigen_exact_and_names_non_finite_input(which):
    K = _krylov_module(which)
    d = [0.3, -1.2, 2.5, 0.0, 1e-9]
    e = [1.0, 1e-12, 0.7, 2.0]
    vals, vecs = K.tridiag_eigen(d, e)
    T = np.diag(d) + np.diag(e, 1) + np.diag(e, -1)
    assert np.linalg.norm(T @ vecs - vecs @ np.diag(vals)) < 1e-12
    assert np.linalg.norm(vecs.T @ vecs - np.eye(5)) < 1e-12
    with pytest.raises(ValueError, match="non-finite"):
        K.tridiag_eigen([0.0, np.nan], [1.0])
    with pytest.raises(ValueError, match="non-finite"):
        K.tridiag_eigen([0.0, 1.0], [np.inf])


# ── the interacting chain against the dense exponential (test/common/dense_reference.jl) ─────


def test_xxz_mpo_is_the_dense_hamiltonian():
    """The XXZ MPO at delta = 0.5 (the headline's interaction) contracts to ``dense_xxz``."""
    mpo = M.xxz_mpo(6, J=1.0, delta=0.5, symmetry="none")
    v = B.to_dense(mpo.tensors[0])
    for t in mpo.tensors[1:]:
        v = np.tensordot(v, B.to_dense(t), axes=([v.ndim - 1], [0]))
    v = v.reshape(v.shape[1:-1])
    dense = v.transpose(list(range(0, 12, 2)) + list(range(1, 12, 2))).reshape(64, 64)
    assert np.max(np.abs(dense - M.dense_xxz(6, 1.0, 0.5))) < 1e-15


@pytest.mark.parametrize("order", [1, 2])
def test_step_converges_at_order_p_plus_one(order):
    """With tolerances far below the time error, the order-p step on the interacting L = 10
    quench (delta 0.5, domain wall, to t = 1) converges at global order p + 1 against the dense
    exponential: halving tau divides the error by 4.0 (p = 1) and 8.0 (p = 2), measured
    1.8e-3 -> 4.4e-4 and 2.9e-5 -> 3.7e-6."""
    L, T = 10, 1.0
    exact = scipy.linalg.expm(-1j * T * M.dense_xxz(L, 1.0, 0.5)) @ M.mps_to_dense(M.domain_wall_state(L))
    errs = []
    for dt in (0.1, 0.05):
        psi, mpo = M.domain_wall_state(L), M.xxz_mpo(L, J=1.0, delta=0.5)
        rng = np.random.default_rng(1234)
        for _ in range(int(round(T / dt))):
            info = S.cbe_bug_step(psi, mpo, -1j * dt, order=order, tol_basis=1e-8, tol_trunc=1e-12,
                                  maxdim=256, rng=rng)
            assert info["status"] == "met"
        errs.append(np.linalg.norm(M.mps_to_dense(psi) - exact) / np.linalg.norm(exact))
    assert errs[0] / errs[1] > 0.85 * 2 ** (order + 1), errs
    assert errs[1] < (1e-3 if order == 1 else 1e-5), errs


# ── per-bond work ceilings (test/BUG/Core/RankAdaptation/test_bond_work_ceiling.jl) ─────────


def test_bond_work_ceilings_known_answers():
    """``test_bond_work_ceiling.jl:23-30`` in the oracle (the native step's ceilings are held to the
    oracle's by the device parity tests: identical widths and dimensions every step)."""
    from oracle import budget as OB

    for bwc in (OB.bond_work_ceilings,):
        assert bwc([1, 3, 8], 2, 1024) == [4, 12, 32]
        assert bwc([0, 5], 4, 1024) == [1, 40]  # never 0, which admits nothing
        assert bwc([1, 3, 8, 40], 2, 16) == [4, 12, 16, 16]
        assert bwc([1, 5, 10, 65], 2, 1024, factor=1.2) == [3, 12, 24, 156]
        assert bwc([1, 5, 10], 3, 1024, factor=1.2) == [4, 18, 36]
        assert bwc([1, 5, 10], 4, 1024, factor=1.2) == [5, 24, 48]
        assert bwc([0, 65], 2, 70, factor=1.2) == [1, 70]


def test_work_ceilings_bound_every_frame():
    """``test_bond_work_ceiling.jl:36-119`` on the Heisenberg chain L = 8 (U(1), tau = -0.2i): from
    the Neel state and from an entangled start, orders 2 and 3, every frame width and every bond
    stays within its ceiling under the default (1.2), the older 2 d D_b rule and a binding maxdim;
    the explicit default is the default bit for bit. (The reference runs these with the exact DD
    probe, which is not built; the bounds hold for the randomised probe the same way.)"""
    from oracle.budget import bond_work_ceilings

    L, d = 8, 2
    mpo = M.xxz_mpo(L, J=1.0, delta=1.0)
    settings = dict(tol_basis=1e-8, tol_expv=1e-12, tol_trunc=1e-12, maxdim=64)

    def step(state, **kw):
        return S.cbe_bug_step(state, mpo, -0.2j, rng=np.random.default_rng(7), **settings, **kw)

    for factor, kw in ((1.2, {}), (0.0, dict(work_ceiling_rule="bond", bond_ceiling_factor=0.0))):
        psi = M.neel_state(L)
        start = psi.bond_dims()
        assert all(b == 1 for b in start)
        info = step(psi, order=2, **kw)
        ceil = bond_work_ceilings(start, d, 64, factor=factor)
        assert all(e <= c for e, c in zip(info["expanded"], ceil))
        assert all(b <= c for b, c in zip(psi.bond_dims(), ceil))

    start_state = M.neel_state(L)
    for _ in range(2):
        step(start_state, order=2)
    start = start_state.bond_dims()
    twice = dict(work_ceiling_rule="bond", bond_ceiling_factor=0.0)
    ceil2 = bond_work_ceilings(start, d, 64)
    tight = bond_work_ceilings(start, d, 64, factor=1.2)
    assert all(t < c for t, c in zip(tight, ceil2))
    for order in (2, 3):
        a, b = start_state.copy(), start_state.copy()
        step(a, order=order)
        step(b, order=order, work_ceiling_rule="bond", bond_ceiling_factor=1.2)
        assert np.array_equal(M.mps_to_dense(a), M.mps_to_dense(b))
        for kw, ceil in ((twice, ceil2), (dict(work_ceiling_rule="bond", bond_ceiling_factor=1.2),
                                          tight)):
            s = start_state.copy()
            info = step(s, order=order, **kw)
            assert all(e <= c for e, c in zip(info["expanded"], ceil)), (order, kw)
            assert all(x <= c for x, c in zip(s.bond_dims(), ceil)), (order, kw)
    small = max(max(start), 2)
    capped = bond_work_ceilings(start, d, small)
    assert any(c < x for c, x in zip(capped, ceil2))
    s = start_state.copy()
    info = S.cbe_bug_step(s, mpo, -0.2j, rng=np.random.default_rng(7), order=2,
                          **dict(settings, maxdim=small), **twice)
    assert all(e <= c for e, c in zip(info["expanded"], capped))
    assert all(x <= small for x in s.bond_dims())


# ── the tolerance budget (test/BUG/Core/RankAdaptation/test_basis_budget.jl) ─────────────────


@pytest.mark.parametrize("which", ["oracle"])
def test_basis_budget_known_answers(which):
    """``test_basis_budget.jl:21-97``: the budget's validation, the RSS allocation rule, tau = 0 as
    a basis question, the indicator's one scaling, the work ceiling and the conservative ledger
    merge, in the oracle (the native step's budget is held to it by the device parity tests)."""
    from oracle import budget as BB
    b = BB.Budget(1e-5, 1e-7, 1e-10)
    assert (b.basis, b.trunc, b.expv) == (1e-5, 1e-7, 1e-10)
    for bad in ((0.0, 1e-7, 1e-10), (-1e-5, 1e-7, 1e-10), (1e-5, 1e-7, 0.0), (1e-5, -1e-7, 1e-10)):
        with pytest.raises(ValueError):
            BB.Budget(*bad)
    assert BB.Budget(1e-5, 0.0, 1e-10).trunc == 0.0  # "discard nothing" is meaningful

    bb = BB.Budget(1e-4, 1e-7, 1e-10)
    a = BB.basis_allocation(bb, 19, tau=0.05, nrm=1.0)
    assert a.per_bond == pytest.approx(1e-4 / math.sqrt(19))
    for share in (a.sample, a.tail, a.krylov):
        assert share == pytest.approx(a.per_bond / 2)
    assert a.scale == pytest.approx(0.05)
    assert BB.basis_allocation(bb, 76, tau=0.05, nrm=1.0).per_bond == pytest.approx(a.per_bond / 2)
    assert BB.basis_allocation(bb, 19, tau=0.05, nrm=2.0).scale == pytest.approx(0.025)

    a0 = BB.basis_allocation(BB.Budget(1e-5, 1e-7, 1e-10), 11, tau=0, nrm=1.0)
    assert a0.scale == 1.0 and BB.indicator(a0, 0.25) == 0.25
    a1 = BB.basis_allocation(BB.Budget(1e-5, 1e-7, 1e-10), 9, tau=0.1, nrm=4.0)
    assert a1.scale == pytest.approx(0.025) and BB.indicator(a1, 8.0) == pytest.approx(0.2)

    assert BB.work_ceiling(128, 10) == 256
    assert BB.work_ceiling(128, 200) == 400  # r > maxdim: the floor governs
    assert BB.work_ceiling(0, 0) == 1  # never zero
    assert BB.work_ceiling(128, 10, 4) == 512
    assert BB.work_ceiling(128, 200, 4) == 800

    x, y = BB.Ledger(), BB.Ledger()
    assert x.tolerance_met and not x.workcap_reached
    x.max_sample, x.n_probes = 1e-6, 12
    y.max_sample, y.n_probes = 3e-6, 7
    y.workcap_reached, y.tolerance_met = True, False
    x.merge(y)
    assert x.max_sample == 3e-6 and x.n_probes == 19
    assert x.workcap_reached and not x.tolerance_met


def test_retired_knobs_are_refused_before_the_state_is_touched():
    """``test_basis_budget.jl:8-19``: a retired fixed-width knob is no keyword of the step (the
    reference's MethodError is a TypeError here), refused before any evolution, in the oracle
    and the native step."""
    from bondupdategalerkin_b200 import native as N

    for step in (S.cbe_bug_step, N.cbe_bug_step):
        psi, mpo = M.neel_state(6), M.xxz_mpo(6, J=1.0, delta=0.0)
        dims0 = psi.bond_dims()
        for kw in (dict(tol_basis=1e-5, dex=4), dict(trunc_thresh=1e-10)):
            with pytest.raises(TypeError):
                step(psi, mpo, -0.05j, **kw)
        assert psi.bond_dims() == dims0


# ── the XX defaults and the local Krylov recurrence (test_krylov_defaults.jl,
#    test_local_lanczos.jl) ───────────────────────────────────────────────────────────────────


def test_expansion_defaults_and_recurrence_resolution():
    """``test_krylov_defaults.jl:21-48``: the DDQRExpansion defaults (oracle and product), the
    recurrence ``auto`` resolves to, an unknown recurrence refused, and the shared stop rule."""
    from bondupdategalerkin_b200.options import DDQRExpansion, resolve_krylov_recurrence

    for cls in (S.DDQRExpansion, DDQRExpansion):
        e = cls()
        assert (e.mode, e.fixed_width, e.tail_factor, e.krylov_mode, e.krylov_fixed_depth) == \
            ("rank_tail", 8, 0.10, "auto", 0)
    assert resolve_krylov_recurrence("auto", True) == "lanczos"
    assert resolve_krylov_recurrence("auto", False) == "arnoldi"
    assert resolve_krylov_recurrence("arnoldi", True) == "arnoldi"
    with pytest.raises(ValueError):
        resolve_krylov_recurrence("gmres", True)
    psi, mpo = M.domain_wall_state(6), M.xxz_mpo(6, J=1.0, delta=0.0)
    with pytest.raises(ValueError):
        S.cbe_bug_step(psi, mpo, -0.1j, expansion=S.DDQRExpansion(krylov_mode="gmres"))
    for stop in (K.krylov_stop,):
        assert stop(1e-3, 1e-2, 1, 0) == (True, True)     # adaptive: within the allowance
        assert stop(1e-1, 1e-2, 1, 0) == (False, False)   # adaptive: go on
        assert stop(1e-3, 1e-2, 2, 4) == (False, False)   # fixed depth not reached yet
        assert stop(1e-3, 1e-2, 4, 4) == (True, True)
        assert stop(1e-1, 1e-2, 4, 4) == (True, False)    # never claims a missed tolerance


def test_defaults_reach_the_step():
    """``test_krylov_defaults.jl:50-90``: on an entangled XX start (L = 8, U(1)), the default step
    is bit for bit the explicit-Lanczos step, with ``hermitian = false`` the explicit-Arnoldi step,
    and every frame and bond stays within ``min(ceil(1.2 d D_b), maxdim)``."""
    from oracle.budget import bond_work_ceilings

    mpo = M.xxz_mpo(8, J=1.0, delta=0.0)
    start = M.domain_wall_state(8)
    for _ in range(3):
        S.cbe_bug_step(start, mpo, -0.1j, order=2)

    def one(**kw):
        s = start.copy()
        info = S.cbe_bug_step(s, mpo, -0.1j, order=2, tol_basis=1e-4,
                              rng=np.random.default_rng(7), **kw)
        return s, info

    d, info = one()
    lz, _ = one(expansion=S.DDQRExpansion(krylov_mode="lanczos"))
    assert np.array_equal(M.mps_to_dense(d), M.mps_to_dense(lz))
    nh, _ = one(hermitian=False)
    ar, _ = one(hermitian=False, expansion=S.DDQRExpansion(krylov_mode="arnoldi"))
    assert np.array_equal(M.mps_to_dense(nh), M.mps_to_dense(ar))
    ceil = bond_work_ceilings(start.bond_dims(), 2, 128, factor=1.2)
    assert all(e <= c for e, c in zip(info["expanded"], ceil))
    assert all(b <= c for b, c in zip(d.bond_dims(), ceil))


class _ArrayOps:
    """The chains' vector operations on plain arrays (the reference test's vectors)."""

    @staticmethod
    def inner(a, b):
        return complex(np.vdot(a, b))

    @staticmethod
    def norm(a):
        return float(np.linalg.norm(a))

    @staticmethod
    def lin(terms):
        return sum(c * v for c, v in terms)

    @staticmethod
    def inner_many(vs, x):
        return [complex(np.vdot(v, x)) for v in vs]


@pytest.mark.parametrize("which", ["oracle"])
def test_local_lanczos_and_arnoldi_chains(which):
    """``test_local_lanczos.jl``: on random Hermitian generators (n = 24, 40; |tau| = 0.1, 1, 4)
    both chains close, their bases capture exp(tau H) seed to 2e-7, the Lanczos basis is
    orthonormal to 1e-7 and its depth within 4 of Arnoldi's; a fixed depth that misses the
    tolerance reports itself capped, not closed."""
    from oracle import krylov as K  # noqa: N811
    rng = np.random.default_rng(45912)
    ops = _ArrayOps()
    for n in (24, 40):
        for t in (0.1, 1.0, 4.0):
            A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
            H = (A + A.conj().T) / 2
            seed = rng.standard_normal(n) + 1j * rng.standard_normal(n)
            seed /= np.linalg.norm(seed)
            tau = -1j * t
            score = lambda *_: True
            ar = K.arnoldi_chain(ops, seed, lambda x: H @ x, tau, 1e-9, score, maxdepth=n)
            la = K.lanczos_chain(ops, seed, lambda x: H @ x, tau, 1e-9, score, maxdepth=n)
            ref = scipy.linalg.expm(tau * H) @ seed
            QA, QL = np.column_stack(ar["basis"]), np.column_stack(la["basis"])
            assert ar["closed"] and la["closed"]
            assert np.linalg.norm(ref - QA @ (QA.conj().T @ ref)) <= 2e-7
            assert np.linalg.norm(ref - QL @ (QL.conj().T @ ref)) <= 2e-7
            assert abs(la["n_h1"] - ar["n_h1"]) <= 4
            assert all(np.isfinite(la["weights"]))
            assert np.linalg.norm(QL.conj().T @ QL - np.eye(QL.shape[1])) <= 1e-7
    n = 20
    H = np.diag(np.ones(n - 1), 1) + np.diag(np.ones(n - 1), -1)
    seed = np.zeros(n, dtype=np.complex128)
    seed[0] = 1
    r = K.lanczos_chain(ops, seed, lambda x: H @ x, -2j, 1e-12, lambda *_: True, maxdepth=n,
                        fixed_depth=4)
    assert r["n_h1"] == 4 and r["capped"] and not r["closed"]


# ── bond frames and the discarded-space projection (test_frames.jl, test_sectors.jl) ────────


def _frame_checks(psi, bond):
    from oracle.cbe import frame_theta, perp_left

    S.canonical(psi, bond)
    f = S.frame_from(psi[bond], psi[bond + 1])
    gl = B.contract(f.U0, (0, 1), f.U0, (0, 1), conja=True)
    gr = B.contract(f.V0, (1, 2), f.V0, (1, 2), conjb=True)
    assert np.allclose(B.to_dense(gl), np.eye(f.U0.dim(2)), atol=1e-12)  # left isometry
    assert np.allclose(B.to_dense(gr), np.eye(f.V0.dim(0)), atol=1e-12)  # right isometry
    two_site = B.contract(psi[bond], (2,), psi[bond + 1], (0,))
    assert B.norm(B.sub(frame_theta(f), two_site)) < 1e-12
    assert f.old_rank == psi[bond].dim(2)
    nrm = B.norm(psi[psi.center])
    assert abs(B.norm(f.S0) - nrm) < 1e-12 and abs(B.norm(frame_theta(f)) - nrm) < 1e-12
    # a vector inside U0's range has no component outside it
    K1 = B.contract(f.U0, (2,), f.S0, (0,))
    assert B.norm(perp_left(f.U0, K1)) < 1e-12
    return f


def test_bond_frames_are_exact_canonical_snapshots():
    """``test_frames.jl:8-99`` and ``test_sectors.jl:61-69``: U0 a left and V0 a right isometry,
    U0 S0 V0 the two-site block exactly, the old rank the link dimension, the snapshot
    norm-preserving, and perp(U0, K) = 0 for K in U0's range; on a product state and on every
    interior bond of an entangled state whose bonds carry several charge sectors."""
    _frame_checks(M.domain_wall_state(6), 2)
    psi = M.domain_wall_state(6)
    mpo = M.xxz_mpo(6, J=1.0, delta=0.5)
    for _ in range(2):
        S.cbe_bug_step(psi, mpo, -0.3j, order=2, rng=np.random.default_rng(5))
    assert max(len(psi[i].legs[2].sectors) for i in range(1, 6)) > 1  # multi-sector bonds
    for bond in range(1, 6):
        _frame_checks(psi, bond)


# ── the symmetric MPS and its canonical moves (test_symmetric_mps.jl,
#    test_state_conformance.jl) ───────────────────────────────────────────────────────────────


def _inner(a, b):
    """<a|b> of two oracle MPS by transfer contraction (charges that do not meet give no block)."""
    E = None
    for i in range(1, len(a) + 1):
        if E is None:
            E = B.contract(a[i], (0, 1), b[i], (0, 1), conja=True)
        else:
            t = B.contract(E, (0,), a[i], (0,), conjb=True)
            E = B.contract(t, (0, 1), b[i], (0, 1))
    return complex(sum(np.sum(v) for v in E.blocks.values()))


def test_symmetric_mps_layout_and_canonical_moves():
    """``test_symmetric_mps.jl:9-70``: the domain wall is a normalised product state with the
    documented leg layout (link, site of dimension 2, link; opposite arrows across every bond);
    canonical moves keep the norm and the arrows, move the centre, and leave left isometries
    left of the centre and right isometries right of it."""
    psi = M.domain_wall_state(6)
    assert len(psi) == 6 and abs(abs(_inner(psi, psi)) - 1.0) < 1e-14
    assert all(b == 1 for b in psi.bond_dims())
    for i in range(1, 7):
        assert len(psi[i].legs) == 3 and psi[i].dim(1) == 2
    for i in range(1, 6):
        assert psi[i].legs[2].dir != psi[i + 1].legs[0].dir
    n0 = abs(_inner(psi, psi))
    for centre in (3, 6):
        S.canonical(psi, centre)
        assert psi.center == centre and abs(abs(_inner(psi, psi)) - n0) < 1e-13
    psi = M.neel_state(6)
    S.canonical(psi, 2)
    for i in range(1, 6):
        assert psi[i].legs[2].dir != psi[i + 1].legs[0].dir
    # an entangled state, so the isometries are not trivially product tensors
    mpo = M.xxz_mpo(6, J=1.0, delta=0.5)
    S.cbe_bug_step(psi, mpo, -0.3j, order=2, rng=np.random.default_rng(2))
    S.canonical(psi, 4)
    for i in range(1, 4):
        g = B.contract(psi[i], (0, 1), psi[i], (0, 1), conja=True)
        assert np.allclose(B.to_dense(g), np.eye(psi[i].dim(2)), atol=1e-12)
    for i in range(5, 7):
        g = B.contract(psi[i], (1, 2), psi[i], (1, 2), conjb=True)
        assert np.allclose(B.to_dense(g), np.eye(psi[i].dim(0)), atol=1e-12)


def test_inner_products_against_dense_and_across_charges():
    """``test_state_conformance.jl:81-94``: <a|b> matches the dense vectors' product and is
    Hermitian; states of different total S^z give an exact zero."""
    a = M.neel_state(6)
    b2 = M.neel_state(6)
    S.cbe_bug_step(b2, M.xxz_mpo(6, J=1.0, delta=0.5), -0.4j, order=2, rng=np.random.default_rng(4))
    ab = _inner(a, b2)
    assert abs(ab - np.vdot(M.mps_to_dense(a), M.mps_to_dense(b2))) < 1e-12
    assert abs(_inner(b2, a) - np.conj(ab)) < 1e-12
    c = M.product_state(["up", "up", "up", "up", "down", "down"])
    assert _inner(a, c) == 0


@pytest.mark.parametrize("which", ["oracle"])
def test_ite_schedule_grids(which):
    """``test_schedules.jl`` (IT-U1): log-panel grids reach beta_max without gaps, uniform inside a
    panel, the first two panels equal and then doubling, the first step beta_max / (2^(P-1) k),
    the coarsest (beta_max / 2) / k, reproducible; uniform steps; the refusals."""
    if which == "product":
        from bondupdategalerkin_b200 import ite as I
    else:
        from oracle import ite as I
    for bmax, P, k in ((8.0, 5, 4), (1.0, 1, 4), (30.0, 7, 2)):
        s = I.log_panel_steps(bmax, P, per_panel=k)
        g = I.beta_grid(s)
        assert len(s) == P * k and all(x > 0 for x in s)
        assert g[0] == 0.0 and g[-1] == pytest.approx(bmax, rel=1e-14)
        assert all(b > a for a, b in zip(g, g[1:]))
        panels = [s[j * k:(j + 1) * k] for j in range(P)]
        assert all(all(x == pytest.approx(p[0]) for x in p) for p in panels)
        widths = [sum(p) for p in panels]
        if P >= 2:
            assert widths[1] == pytest.approx(widths[0])
        if P >= 3:
            assert all(widths[j + 1] == pytest.approx(2 * widths[j]) for j in range(1, P - 1))
        assert s[0] == pytest.approx(bmax / (2.0 ** (P - 1) * k))
        assert max(s) == pytest.approx((bmax if P == 1 else bmax / 2) / k)
        assert I.log_panel_steps(bmax, P, per_panel=k) == s
    u = I.uniform_beta_steps(2.0, 8)
    assert all(x == 0.25 for x in u) and I.beta_grid(u)[-1] == pytest.approx(2.0)
    for bad in (lambda: I.log_panel_steps(1.0, 0), lambda: I.log_panel_steps(-1.0, 3),
                lambda: I.uniform_beta_steps(1.0, 0)):
        with pytest.raises(ValueError):
            bad()


def test_fused_sectors_cover_the_frames_charges():
    """``test_sectors.jl:18-59``: the fused space link (x) site of every bond frame's U0 has the
    full dimension with no duplicate charge, U0's new-leg charges are among the fused charges and
    every stored block conserves charge; links with a non-zero charge are covered (a vacuum link is
    its own dual and would hide a sign error)."""
    mpo = M.xxz_mpo(6, J=1.0, delta=0.5)
    ent = M.neel_state(6)
    S.cbe_bug_step(ent, mpo, -0.3j, order=2, rng=np.random.default_rng(9))
    saw_charged = False
    for psi in (M.domain_wall_state(4), M.neel_state(6), ent):
        for bond in range(1, len(psi)):
            S.canonical(psi, bond)
            U0 = S.frame_from(psi[bond], psi[bond + 1]).U0
            la, lb, lc = U0.legs
            fused = B.fused_sectors(la, lb, lc.dir)
            assert sum(la.sectors[qa] * lb.sectors[qb] for v in fused.values() for qa, qb in v) \
                == U0.dim(0) * U0.dim(1)
            assert len(set(fused)) == len(fused)
            assert set(lc.sectors) <= set(fused)
            for qa, qb, qc in U0.blocks:
                assert la.dir * qa + lb.dir * qb + lc.dir * qc == 0
            saw_charged |= any(q != 0 for q in la.sectors)
    assert saw_charged

