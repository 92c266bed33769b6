"""The step's keyword checks against the reference's (``bug_step_stages.jl:40-142``), on CPU.

Every keyword of ``cbe_bug_step!`` is accepted by name. The oracle and the native step's Python
entry must refuse what the reference refuses
(``ArgumentError`` / ``DimensionMismatch`` -> ``ValueError``) and name what they do not build
(``NotImplementedError``), with the same outcome for the same keywords; an option the oracle
restates ahead of the device step (``ORACLE_AHEAD``) is named as not built by the product only.
The checks run before any device work, so the product hosts are called here with the oracle's
chain objects and never reach the engine.
"""

import numpy as np
import pytest

from oracle import models as M
from oracle import step as S

L = 6
BAD = [
    (dict(mpo_sites=5), ValueError),
    (dict(root=0), ValueError),
    (dict(root=L), ValueError),
    (dict(tol_root=1e-6, tol_expv=1e-6), ValueError),
    (dict(order=0), ValueError),
    (dict(frontier_tol=-1.0), ValueError),
    (dict(work_ceiling_rule="foo"), ValueError),
    (dict(work_ceiling_rule="bond_strict"), ValueError),  # its default factor 0 is no strict factor
    (dict(work_ceiling_rule="bond_strict", bond_ceiling_factor=1.0), ValueError),
    (dict(bond_ceiling_factor=0.5), ValueError),
    (dict(bond_ceiling_factor=1.5, work_ceiling_rule="maxdim"), ValueError),
    (dict(root_ceiling_factor=1.0), ValueError),
    (dict(work_ceiling_rule="frame_root", bond_ceiling_factor=1.5, root_ceiling_factor=1.8),
     ValueError),
    (dict(closure_probe=-1), ValueError),
    (dict(keep_tols=[0.1]), ValueError),
    (dict(keep_states="psi", keep_tols=[-1.0]), ValueError),
    (dict(frames_only=True), ValueError),
    (dict(order=2, fold_omega=False, outside_residual=True, root_report={}), NotImplementedError),
    (dict(exact=True, order=2, outside_residual=True, root_report={}), NotImplementedError),
    (dict(kls="foo"), ValueError),
    (dict(kls="sequential", outside_residual=True, root_report={}), ValueError),
    (dict(kls="sequential"), NotImplementedError),
    (dict(parallel="bogus"), ValueError),
    (dict(parallel="full"), NotImplementedError),
]


def _args(kw):
    kw = dict(kw)
    psi = M.domain_wall_state(L)
    mpo = M.xxz_mpo(kw.pop("mpo_sites", L), J=1.0, delta=0.5)
    if kw.get("keep_states") == "psi":
        kw["keep_states"] = [psi.copy()]
    return psi, mpo, kw


def _hosts():
    from bondupdategalerkin_b200 import native as N

    return [("oracle", S.cbe_bug_step), ("native", N.cbe_bug_step)]


@pytest.mark.parametrize("kw,exc", BAD, ids=[repr(k) for k, _ in BAD])
def test_hosts_refuse_as_the_reference_does(kw, exc):
    for name, step in _hosts():
        psi, mpo, k = _args(kw)
        with pytest.raises(exc):
            step(psi, mpo, -0.05j, rng=np.random.default_rng(0), **k)


# restated in the oracle ahead of the device step: the product names them as not built
ORACLE_AHEAD = [dict(krylov_rank_tol=0.1), dict(frontier_tol=1e-3), dict(closure_probe=2)]


@pytest.mark.parametrize("kw", ORACLE_AHEAD, ids=[repr(k) for k in ORACLE_AHEAD])
def test_product_names_what_only_the_oracle_restates(kw):
    from bondupdategalerkin_b200 import native as N

    psi, mpo, k = _args(kw)
    with pytest.raises(NotImplementedError):
        N.cbe_bug_step(psi, mpo, -0.05j, rng=np.random.default_rng(0), **k)


def test_fewer_than_two_sites():
    from bondupdategalerkin_b200.options import check_step_options

    with pytest.raises(ValueError, match="two sites"):
        check_step_options(1, 1)
    with pytest.raises(ValueError, match="two sites"):
        S.step_options(1, 1, None, False, None, None, None, 1, "bond", None, 1.2, 0.0, 0.0, 0, (),
                       (), False, None, False, None, True, False)


def test_tol_root_is_tol_expv():
    """``tol_root`` is another name for ``tol_expv``: the same step, bit for bit."""
    out = []
    for kw in (dict(tol_root=1e-9), dict(tol_expv=1e-9)):
        psi, mpo = M.domain_wall_state(L), M.xxz_mpo(L, J=1.0, delta=0.5)
        info = S.cbe_bug_step(psi, mpo, -0.05j, order=2, rng=np.random.default_rng(3), **kw)
        out.append((M.mps_to_dense(psi), info["ledger"].expv_err, info["bond_dims"]))
    assert np.array_equal(out[0][0], out[1][0]) and out[0][1:] == out[1][1:]
    from bondupdategalerkin_b200.options import check_step_options

    assert check_step_options(L, L, tol_root=1e-9) == 1e-9
    assert check_step_options(L, L, tol_expv=1e-7) == 1e-7


def test_root_ceiling_factor_alone_is_accepted():
    """A valid ``root_ceiling_factor`` only matters under ``:frame_root``; elsewhere the step runs
    unchanged (the reference checks it and ignores it)."""
    psi, mpo = M.domain_wall_state(L), M.xxz_mpo(L, J=1.0, delta=0.5)
    S.cbe_bug_step(psi, mpo, -0.05j, root_ceiling_factor=1.5, rng=np.random.default_rng(0))
    from bondupdategalerkin_b200.options import check_step_options

    assert check_step_options(L, L, root_ceiling_factor=1.5) is None


def test_tdvp2_keywords_checked_as_the_reference_does():
    """``tdvp2_step!`` (``tdvp2.jl:182-228``): two sites at least, matching chain lengths, a
    non-negative ``weight_tol``; the backward amplification reports are named as not built."""
    from bondupdategalerkin_b200 import native as N
    from oracle import tdvp as T

    for step in (T.tdvp2_step, N.tdvp2_step):
        psi = M.domain_wall_state(L)
        with pytest.raises(ValueError):
            step(psi, M.xxz_mpo(L - 1), -0.05j)
        with pytest.raises(ValueError):
            step(psi, M.xxz_mpo(L), -0.05j, weight_tol=-1.0)
        with pytest.raises(NotImplementedError):
            step(psi, M.xxz_mpo(L), -0.05j, backward_norms=[])
