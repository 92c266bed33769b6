"""The work-ceiling rules ``:bond_strict`` and ``:frame_root`` (CPU).

``bond_work_ceilings_strict`` (``ceil(f D_b)``, no local dimension) and
``bond_frame_root_ceilings`` (``ceil(2 D_b)`` on frames, ``ceil(1.2 D_root)`` at the root bond;
``basis_budget.jl:497-545``) as the reference tests them
(``test/BUG/Core/RankAdaptation/test_bond_work_ceiling.jl:121-163``), the oracle step held to
them, and the engine's ``bug_work_ceilings`` (the function the device step takes its ceilings
from; host code, no GPU) equal to the oracle's for every rule.
"""

import ctypes

import numpy as np
import pytest

from oracle import budget as BG
from oracle import models as M
from oracle import step as S

SETTINGS = dict(tol_basis=1e-8, tol_root=1e-12, tol_trunc=1e-12, maxdim=64, exact=True)


def test_reference_values():
    assert BG.bond_frame_root_ceilings([1, 5, 10, 65], 1024, 2) == [2, 6, 20, 130]
    assert BG.bond_frame_root_ceilings([1, 5, 10, 65], 1024, 3) == [2, 10, 12, 130]
    assert BG.bond_frame_root_ceilings([1, 5, 10, 65], 64, 3) == [2, 10, 12, 64]
    with pytest.raises(ValueError):
        BG.bond_frame_root_ceilings([1, 2, 3], 64, 2, frame_factor=1.1, root_factor=1.2)
    with pytest.raises(ValueError):
        BG.bond_frame_root_ceilings([1, 2, 3], 64, 4)
    assert BG.bond_work_ceilings_strict([1, 5, 10, 65], 64, 1.2) == [2, 6, 12, 64]
    with pytest.raises(ValueError, match="strict"):
        BG.bond_work_ceilings_strict([1, 2], 64, 1.0)


@pytest.fixture(scope="module")
def chain():
    L = 8
    mpo = M.xxz_mpo(L, J=1.0, delta=1.0)
    start = M.neel_state(L)
    for _ in range(2):
        S.cbe_bug_step(start, mpo, -0.2j, order=2, **SETTINGS)
    return mpo, start


@pytest.mark.parametrize("order", [2, 3])
def test_frame_root_step_within_its_caps(chain, order):
    mpo, start = chain
    L = len(start)
    root = L // 2
    bonds = start.bond_dims()
    caps = BG.bond_frame_root_ceilings(bonds, 64, root)
    assert caps[root - 1] == min(64, BG._ceil9(1.2 * bonds[root - 1]))
    psi = start.copy()
    info = S.cbe_bug_step(psi, mpo, -0.2j, order=order, work_ceiling_rule="frame_root",
                          bond_ceiling_factor=2.0, root_ceiling_factor=1.2, closure_checks=True,
                          **SETTINGS)
    assert info["root_link"] == root
    assert all(e <= c for e, c in zip(info["expanded"], caps))
    assert info["root_frame_width"] <= caps[root - 1]
    assert all(b <= c for b, c in zip(psi.bond_dims(), caps))
    assert all(e["width"] <= caps[e["bond"] - 1] for e in info["ledger"].bond_log)
    assert info["expanded"][root - 1] * info["root_frame_width"] <= caps[root - 1] ** 2


def test_bond_strict_step_within_its_caps(chain):
    mpo, start = chain
    caps = BG.bond_work_ceilings_strict(start.bond_dims(), 64, 1.5)
    psi = start.copy()
    info = S.cbe_bug_step(psi, mpo, -0.2j, order=2, work_ceiling_rule="bond_strict",
                          bond_ceiling_factor=1.5, **SETTINGS)
    assert all(e <= c for e, c in zip(info["expanded"], caps))
    assert all(b <= c for b, c in zip(psi.bond_dims(), caps))
    with pytest.raises(ValueError, match="strict bond factor"):
        S.cbe_bug_step(start.copy(), mpo, -0.2j, order=2, work_ceiling_rule="bond_strict",
                       **SETTINGS)


def _engine_ceilings(lib, rule, bonds, d, maxdim, factor, root, root_factor):
    n = len(bonds)
    b = (ctypes.c_int64 * n)(*bonds)
    out = (ctypes.c_int64 * n)()
    rc = lib.bug_work_ceilings(rule, n, b, ctypes.c_int64(d), ctypes.c_int64(maxdim),
                               ctypes.c_double(factor), root, ctypes.c_double(root_factor), out)
    return rc, list(out)


def test_engine_ceilings_equal_the_oracle():
    from bondupdategalerkin_b200 import _engine

    lib = _engine.load()
    rng = np.random.default_rng(4)
    for _ in range(50):
        n = int(rng.integers(1, 20))
        bonds = [int(x) for x in rng.integers(1, 300, n)]
        maxdim = int(rng.integers(1, 400))
        root = int(rng.integers(1, n + 1))
        f = float(rng.choice([1.1, 1.2, 1.5, 2.0, 2.5]))
        rf = float(rng.choice([1.05, 1.2, f]))
        assert _engine_ceilings(lib, 0, bonds, 2, maxdim, -1.0, root, -1.0) == \
            (0, BG.bond_work_ceilings(bonds, 2, maxdim, factor=1.2))
        assert _engine_ceilings(lib, 0, bonds, 3, maxdim, 0.0, root, -1.0) == \
            (0, BG.bond_work_ceilings(bonds, 3, maxdim, factor=0.0))
        assert _engine_ceilings(lib, 1, bonds, 2, maxdim, -1.0, root, -1.0) == \
            (0, [BG.work_ceiling(maxdim, max(bonds), 2)] * n)
        assert _engine_ceilings(lib, 2, bonds, 2, maxdim, f, root, -1.0) == \
            (0, BG.bond_work_ceilings_strict(bonds, maxdim, f))
        if rf <= f:
            assert _engine_ceilings(lib, 3, bonds, 2, maxdim, f, root, rf) == \
                (0, BG.bond_frame_root_ceilings(bonds, maxdim, root, frame_factor=f,
                                                root_factor=rf))
        assert _engine_ceilings(lib, 3, bonds, 2, maxdim, 0.0, root, -1.0) == \
            (0, BG.bond_frame_root_ceilings(bonds, maxdim, root))


def test_engine_refuses_what_the_reference_refuses():
    from bondupdategalerkin_b200 import _engine

    lib = _engine.load()
    bonds = [1, 2, 3]
    assert _engine_ceilings(lib, 2, bonds, 2, 64, -1.0, 2, -1.0)[0] == 1
    assert _engine_ceilings(lib, 3, bonds, 2, 64, 1.1, 2, 1.2)[0] == 1
    assert _engine_ceilings(lib, 3, bonds, 2, 64, 2.0, 4, 1.2)[0] == 1
    assert _engine_ceilings(lib, 1, bonds, 2, 64, 1.5, 2, -1.0)[0] == 1
    assert _engine_ceilings(lib, 4, bonds, 2, 64, -1.0, 2, -1.0)[0] == 1
