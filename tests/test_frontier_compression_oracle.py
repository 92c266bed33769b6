"""``frontier_tol`` in the oracle: each frontier compressed to its own rank before its sweep (CPU).

Written in the frames, a frontier's bonds are as wide as the frames; with ``frontier_tol > 0`` it
is compressed at that weight tolerance, with no rank cap, before the sweep
(``frontier_closure.jl:102-120``). The cases are the reference's
``test/BUG/Core/Sweeps/test_frontier_compression.jl`` (Heisenberg L = 6, U(1), exact selection,
order 3): the compressed step agrees with the plain one and is no less accurate against the dense
propagator, parallel and serial compressed steps agree, a negative tolerance is refused. A
longer chain shows the compression cutting the frontiers' bonds with the step unchanged.
"""

import numpy as np
import pytest
import scipy.linalg

from oracle import models as M
from oracle import step as S
from tests.gpu_util import fidelity

SETTINGS = dict(order=3, tol_basis=1e-8, tol_trunc=1e-12, maxdim=64, exact=True)


def _entangled(L, start, delta, steps):
    mpo = M.xxz_mpo(L, J=1.0, delta=delta)
    psi = getattr(M, start)(L)
    for _ in range(steps):
        S.cbe_bug_step(psi, mpo, -0.2j, **{**SETTINGS, "order": 2})
    return mpo, psi


def test_reference_case():
    L = 6
    mpo, start = _entangled(L, "neel_state", 1.0, 2)
    v0 = M.mps_to_dense(start)
    n0 = np.linalg.norm(v0)
    want = scipy.linalg.expm(-0.2j * M.dense_xxz(L, 1.0, 1.0)) @ v0
    plain, comp, par = start.copy(), start.copy(), start.copy()
    S.cbe_bug_step(plain, mpo, -0.2j, parallel=False, **SETTINGS)
    S.cbe_bug_step(comp, mpo, -0.2j, parallel=False, frontier_tol=1e-12, **SETTINGS)
    S.cbe_bug_step(par, mpo, -0.2j, parallel=True, frontier_tol=1e-12, **SETTINGS)
    vp, vc = M.mps_to_dense(plain), M.mps_to_dense(comp)
    assert np.linalg.norm(vc - vp) < 1e-9 * n0
    assert np.linalg.norm(vc - want) / n0 <= np.linalg.norm(vp - want) / n0 + 1e-9
    assert 1.0 - fidelity(par, comp) < 1e-12
    assert par.bond_dims() == comp.bond_dims()
    with pytest.raises(ValueError, match="frontier_tol"):
        S.cbe_bug_step(start.copy(), mpo, -0.2j, frontier_tol=-1.0, **SETTINGS)


def test_compression_cuts_the_frontier_bonds(monkeypatch):
    L = 10
    mpo, start = _entangled(L, "domain_wall_state", 0.5, 3)
    cuts = []
    orig = S.truncate_recursive

    def spy(psi, root, maxdim, weight_tol, bond_weights):
        before = psi.bond_dims()
        out = orig(psi, root, maxdim, weight_tol, bond_weights)
        cuts.append((before, psi.bond_dims()))
        return out

    monkeypatch.setattr(S, "truncate_recursive", spy)
    comp = start.copy()
    S.cbe_bug_step(comp, mpo, -0.2j, frontier_tol=1e-12, **SETTINGS)
    monkeypatch.setattr(S, "truncate_recursive", orig)
    plain = start.copy()
    S.cbe_bug_step(plain, mpo, -0.2j, **SETTINGS)
    frontiers = cuts[:-1]  # the last compression is the step's own
    assert len(frontiers) == SETTINGS["order"] - 1
    assert any(sum(after) < sum(before) for before, after in frontiers)
    assert 1.0 - fidelity(comp, plain) < 1e-12
    assert comp.bond_dims() == plain.bond_dims()
