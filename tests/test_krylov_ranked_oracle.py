"""``krylov_rank_tol`` in the oracle: the ranked local Krylov selection (CPU).

With ``krylov_rank_tol > 0`` each local Krylov stage collects every direction above its allowance
against the start frame and, at the end, keeps the fewest top ones of one SVD of their weighted
residuals whose discarded tail fits the ranked share (``_append_ranked``,
``krylov_enrichment.jl:176-292``); ``0`` is the sequential rule. The cases are the reference's
``test/BUG/Core/RankAdaptation/test_krylov_ranked.jl`` (Heisenberg L = 8, U(1), exact selection,
orders 2 and 3): a tight rank tolerance is as accurate as the sequential step, a loose one gives a
stage frame no wider and stays accurate to its looser share, a negative one is refused.
"""

import numpy as np
import pytest
import scipy.linalg

from oracle import budget as BG
from oracle import models as M
from oracle import step as S

L = 8
SETTINGS = dict(tol_basis=1e-8, tol_root=1e-12, tol_trunc=1e-12, maxdim=64, exact=True)


def test_krylov_rank_defaults_and_apportioning():
    budget = BG.Budget(1e-8, 1e-10, 1e-10)
    assert BG.basis_allocation(budget, 9).krylov_rank == 0.0
    alloc = BG.basis_allocation(budget, 9, rule="linear", krylov=1e-6, krylov_rank=1e-6)
    assert alloc.krylov_rank == pytest.approx(alloc.krylov)
    with pytest.raises(ValueError):
        BG.basis_allocation(budget, 9, krylov_rank=-1.0)


@pytest.fixture(scope="module")
def chain():
    mpo = M.xxz_mpo(L, J=1.0, delta=1.0)
    start = M.neel_state(L)
    for _ in range(2):
        S.cbe_bug_step(start, mpo, -0.2j, order=2, **SETTINGS)
    v0 = M.mps_to_dense(start)
    want = scipy.linalg.expm(-0.2j * M.dense_xxz(L, 1.0, 1.0)) @ v0
    return mpo, start, v0, want


def _error_and_stage(chain, **kw):
    mpo, start, v0, want = chain
    psi = start.copy()
    info = S.cbe_bug_step(psi, mpo, -0.2j, **SETTINGS, **kw)
    return np.linalg.norm(M.mps_to_dense(psi) - want) / np.linalg.norm(v0), info["record"]["r_aug"]


@pytest.mark.parametrize("order", [2, 3])
def test_ranked_against_sequential(chain, order):
    plain_err, plain_stage = _error_and_stage(chain, order=order)
    tight_err, tight_stage = _error_and_stage(chain, order=order, krylov_rank_tol=1e-12)
    loose_err, loose_stage = _error_and_stage(chain, order=order, krylov_rank_tol=1e-6)
    assert tight_err <= 10 * plain_err + 1e-10
    assert loose_stage <= plain_stage
    assert loose_stage <= tight_stage
    assert loose_err < 1e-4


def test_negative_rank_tolerance_is_refused(chain):
    mpo, start, _, _ = chain
    with pytest.raises(ValueError, match="krylov_rank_tol"):
        S.cbe_bug_step(start.copy(), mpo, -0.2j, order=2, krylov_rank_tol=-1.0, **SETTINGS)


def _vec(i, scale=1.0):
    """The i-th unit vector of the fused (link 2 x site 2) space as a left-frame-shaped tensor
    (one charge sector, a bond leg of width 1)."""
    from oracle import blocks as B

    v = np.zeros((2, 2, 1), dtype=np.complex128)
    v.reshape(4)[i] = scale
    legs = [B.Leg(-1, {0: 2}), B.Leg(-1, {0: 2}), B.Leg(+1, {0: 1})]
    return B.BT(legs, {(0, 0, 0): v})


@pytest.mark.parametrize("allowance,workcap,added,fits", [
    (1e-2, 0, 1, True),    # the weak direction's weight fits the allowance: only the strong one
    (1e-4, 0, 2, True),    # it does not: both
    (1e-4, 2, 1, False),   # the ceiling leaves room for one: the strongest, and the rest is unmet
    (1e-4, 1, 0, False),   # no room at all
])
def test_append_ranked_keeps_the_strongest_directions(allowance, workcap, added, fits):
    frame = _vec(0)
    cands = [_vec(1, 1e-3), _vec(2, 1.0)]  # collected weak first: ranking, not chain order
    out, n, ok = S.append_ranked(frame, cands, "left", allowance, workcap)
    assert (n, ok) == (added, fits)
    assert out.dim(2) == 1 + added
    if added == 1:  # the direction kept is the strong one, e_2
        from oracle import blocks as B

        m = B.to_dense(out).reshape(4, 2)
        assert abs(abs(m[2, 1]) - 1.0) < 1e-12
