"""``keep_states`` / ``keep_tols`` in the oracle: the trial space contains the kept states (CPU).

Each half-sweep unions every kept state's carried site tensor into the new frame
(``_union_fresh``, ``half_sweeps.jl:143-204``, loops at ``:281-297`` and ``:385-398``): with
``keep_tols = 0`` the state is contained exactly (an MPDO's identity, Heston's mass); admitted at a
tolerance it widens the frames no more than that; under ``work_ceiling_rule = :bond`` an admitted
state fills a frame only up to its bond's work ceiling (``_keep_room``). The cases are those of
``test/BUG/TimeEvolution/test_step_keep_states.jl:12-60`` (Heisenberg L = 8, U(1), exact
selection, order 2), with its ``frames_only`` / ``frames_report`` half: a frames-only step returns
the state in the frames of the full step.
"""

import pytest

from oracle import models as M
from oracle import step as S
from tests.gpu_util import fidelity

L = 8
SETTINGS = dict(order=2, tol_basis=1e-8, tol_trunc=1e-12, maxdim=64, exact=True)


@pytest.fixture(scope="module")
def chain():
    mpo = M.xxz_mpo(L, J=1.0, delta=1.0)
    start = M.neel_state(L)
    S.cbe_bug_step(start, mpo, -0.2j, **SETTINGS)
    kept = start.copy()  # a more entangled state of the same sector
    for _ in range(3):
        S.cbe_bug_step(kept, mpo, -0.3j, **SETTINGS)
    return mpo, start, kept


def _step(chain, **kw):
    mpo, start, _ = chain
    psi = start.copy()
    k = dict(SETTINGS)
    k.update(kw)
    info = S.cbe_bug_step(psi, mpo, -0.2j, truncate=False, **k)
    return info["expanded"], psi


def test_kept_state_widens_and_admission_widens_less(chain):
    kept = chain[2]
    plain, _ = _step(chain)
    exact, _ = _step(chain, keep_states=[kept])
    admitted, _ = _step(chain, keep_states=[kept], keep_tols=[1e-6])
    assert any(e > p for e, p in zip(exact, plain))  # fixture guard: the state widens
    assert all(a <= e for a, e in zip(admitted, exact))


def test_admitted_state_stays_within_the_bond_ceilings(chain):
    _, start, kept = chain
    bonds = start.bond_dims()
    small = max(max(bonds), 2)
    ceilings = S.bond_work_ceilings(bonds, 2, small)
    capped, _ = _step(chain, keep_states=[kept], keep_tols=[1e-12], maxdim=small,
                      work_ceiling_rule="bond")
    assert all(c <= x for c, x in zip(capped, ceilings))


def test_exactly_kept_state_lies_in_the_frames(chain):
    """The frames the step ends with (``frames_report``, after the frontier sweep) contain the
    kept state: its projection miss on them is round-off; without the keep they miss it."""
    kept = chain[2]
    root = S.bug_root_link(L)
    k = kept.copy()
    S.canonical(k, root)
    nk = S.B.norm(k[k.center])
    with_keep, without = {}, {}
    _step(chain, keep_states=[kept], frames_report=with_keep)
    _step(chain, frames_report=without)
    assert with_keep["root_link"] == root
    miss = S.projection_miss(k, with_keep["left_frames"], with_keep["right_frames"], root)
    assert miss <= 1e-12 * nk
    assert S.projection_miss(k, without["left_frames"], without["right_frames"], root) > 1e-6 * nk


def test_frames_only_returns_the_state_in_the_full_steps_frames(chain):
    """``frames_only`` skips the root solve: the state comes back as itself in the frames, and the
    frames are those of the full step (``test_step_keep_states.jl:62-80``)."""
    mpo, start, _ = chain
    full, only = {}, {}
    _step(chain, frames_report=full)
    psi = start.copy()
    info = S.cbe_bug_step(psi, mpo, -0.2j, truncate=False, frames_only=True, frames_report=only,
                          **SETTINGS)
    assert 1.0 - fidelity(psi, start) < 1e-12
    assert info["ledger"].expv_iters == 0
    widths = {b: f.dim(2) for b, f in only["left_frames"].items()}
    assert widths == {b: f.dim(2) for b, f in full["left_frames"].items()}


def test_frames_only_with_a_truncation_is_refused(chain):
    mpo, start, _ = chain
    with pytest.raises(ValueError, match="frames_only"):
        S.cbe_bug_step(start.copy(), mpo, -0.2j, frames_only=True, **SETTINGS)


def test_two_kept_states_and_their_tolerances(chain):
    _, start, kept = chain
    both, _ = _step(chain, keep_states=[kept, start], keep_tols=[0.0, 0.0])
    one, _ = _step(chain, keep_states=[kept])
    assert both == one  # the start state is already in every frame


def test_mismatched_keep_tols_are_refused(chain):
    with pytest.raises(ValueError, match="keep_tols"):
        _step(chain, keep_states=[chain[2]], keep_tols=[1e-6, 1e-6])
