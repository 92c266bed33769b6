"""``exact = true`` in the oracle: the deterministic reference selection, on the CPU.

With ``exact = true`` every DD expansion sketches the complete fused basis of the opposite frame's
local legs with that frame projected out (``_dd_probe(...; exact = true)``, ``dd_cbe.jl:140-161``)
and keeps what ``_dd_select``'s two-pass pivoted QR admits in one pass (``dd_cbe_expand.jl:91,
346-360``); above order 1 the frontier leaks default to the exact leak of the formed two-site action
(``fold_omega = order > 1 && !exact``, ``bug_step_stages.jl:67``; ``krylov_frontier_bonds.jl:80-100``).
Such a step draws no random numbers. The cases are the reference's own:
``test/BUG/TimeEvolution/test_parallel_half_sweeps.jl:35-44`` (serial and parallel agree to
round-off, verdicts included), ``test/BUG/Core/RankAdaptation/test_bond_work_ceiling.jl:36-64``
(from a product state every bond stays within its work ceiling) and the accuracy of the exact
selection against the dense propagator (``test_frontier_compression.jl:17-48``, without the
``frontier_tol`` compression, which is not restated).
"""

import numpy as np
import pytest
import scipy.linalg

from oracle import blocks as B
from oracle import models as M
from oracle import step as S
from oracle.cbe import dd_probe_exact
from tests.gpu_util import fidelity

REF = dict(tol_basis=1e-7, tol_trunc=1e-9, tol_expv=1e-10, maxdim=64)


@pytest.mark.parametrize("order", [1, 2])
def test_exact_parallel_equals_serial(order):
    serial, par = M.neel_state(6), M.neel_state(6)
    mpo = M.xxz_mpo(6, J=1.0, delta=1.0)
    rs, rp = np.random.default_rng(1), np.random.default_rng(1)
    for _ in range(2):
        a = S.cbe_bug_step(serial, mpo, -0.05j, order=order, exact=True, parallel=False, rng=rs, **REF)
        b = S.cbe_bug_step(par, mpo, -0.05j, order=order, exact=True, parallel=True, rng=rp, **REF)
        assert a["status"] == b["status"]
        assert a["ledger"].n_probes == b["ledger"].n_probes == 0
    assert 1.0 - fidelity(serial, par) < 1e-12
    assert serial.bond_dims() == par.bond_dims()


@pytest.mark.parametrize("order", [1, 2, 3])
def test_exact_steps_draw_nothing(order):
    psi, mpo = M.neel_state(8), M.xxz_mpo(8, J=1.0, delta=1.0)
    rng = np.random.default_rng(3)
    before = rng.bit_generator.state
    for _ in range(2):
        info = S.cbe_bug_step(psi, mpo, -0.2j, order=order, exact=True, rng=rng, tol_basis=1e-8,
                              tol_root=1e-12, tol_trunc=1e-12, maxdim=64)
    assert rng.bit_generator.state == before
    # one exact two-site leak per frontier bond (the root bond in both halves)
    assert info["ledger"].n_h2_leak == (0 if order == 1 else (order - 1) * 8)


@pytest.mark.parametrize("factor,rule", [(1.2, {}), (0.0, dict(work_ceiling_rule="bond",
                                                                 bond_ceiling_factor=0.0))])
def test_exact_bonds_within_their_work_ceilings(factor, rule):
    L = 8
    psi, mpo = M.neel_state(L), M.xxz_mpo(L, J=1.0, delta=1.0)
    start = psi.bond_dims()
    assert all(b == 1 for b in start)
    info = S.cbe_bug_step(psi, mpo, -0.2j, order=2, exact=True, tol_basis=1e-8, tol_root=1e-12,
                          tol_trunc=1e-12, maxdim=64, rng=np.random.default_rng(0), **rule)
    ceilings = S.bond_work_ceilings(start, 2, 64, factor=factor)
    assert all(e <= c for e, c in zip(info["expanded"], ceilings))
    assert all(b <= c for b, c in zip(psi.bond_dims(), ceilings))


@pytest.mark.parametrize("order", [2, 3])
def test_exact_selection_tracks_the_dense_propagator(order):
    L, tau = 6, -0.2j
    mpo = M.xxz_mpo(L, J=1.0, delta=1.0)
    psi = M.neel_state(L)
    kw = dict(tol_basis=1e-8, tol_trunc=1e-12, maxdim=64, exact=True, rng=np.random.default_rng(0))
    for _ in range(2):
        S.cbe_bug_step(psi, mpo, tau, order=2, **kw)
    v0 = M.mps_to_dense(psi)
    S.cbe_bug_step(psi, mpo, tau, order=order, **kw)
    want = scipy.linalg.expm(tau * M.dense_xxz(L, 1.0, 1.0)) @ v0
    err = np.linalg.norm(M.mps_to_dense(psi) - want) / np.linalg.norm(v0)
    assert err < 1e-3


def test_exact_probe_is_the_discarded_space():
    """The exact probe spans exactly the fused space minus the frame: its columns are the
    projector ``I - U U^dag`` (left frame) applied to every fused basis vector, so ``P P^dag`` is
    that projector."""
    psi = M.neel_state(6)
    mpo = M.xxz_mpo(6, J=1.0, delta=1.0)
    for _ in range(2):
        S.cbe_bug_step(psi, mpo, -0.05j, order=1, exact=True, rng=np.random.default_rng(0), **REF)
    S.canonical(psi, 4)
    U = psi[2]  # left-canonical (link, site, bond), 3 of its 4 fused directions kept
    om = dd_probe_exact(U, "left")
    P = B.to_dense(om).reshape(-1, om.dim(2))
    Ud = B.to_dense(U).reshape(-1, U.dim(2))
    proj = np.eye(Ud.shape[0]) - Ud @ Ud.conj().T
    np.testing.assert_allclose(P @ P.conj().T, proj, atol=1e-13)
    assert np.linalg.matrix_rank(P, tol=1e-10) == Ud.shape[0] - Ud.shape[1]
