"""``keep_states`` / ``keep_tols`` on the device, against the oracle (GPU).

Each half-sweep unions the kept states' carried sites into its frames (``_union_fresh``,
``half_sweeps.jl:143-204``). The device step and the oracle step start from the same state with
the same kept state (uploaded bit for bit) on the reference's setting
(``test/BUG/TimeEvolution/test_step_keep_states.jl:12-60``: Heisenberg L = 8, U(1), exact
selection, order 2, no final compression) and must agree on the frame widths, the bond dimensions
and the state (infidelity <= 1e-12): contained exactly, admitted at a tolerance, and admitted under
the per-bond work ceiling. ``frames_report`` and ``frames_only`` (``bug_step.jl:381-382,
455-467``) are checked on the same setting.
"""

import numpy as np
import pytest

from oracle import models as OM
from oracle import step as OS
from tests.gpu_util import fidelity, mps_to_host, to_dev, to_host
from tests.test_gpu_step import dev  # noqa: F401  (the module fixture)

pytestmark = pytest.mark.gpu

L = 8
SETTINGS = dict(order=2, tol_basis=1e-8, tol_trunc=1e-12, maxdim=64, exact=True)


def _upload(DM, psi):
    return DM.MPS([to_dev(t) for t in psi.tensors], psi.center)


@pytest.fixture(scope="module")
def chain():
    mpo = OM.xxz_mpo(L, J=1.0, delta=1.0)
    start = OM.neel_state(L)
    OS.cbe_bug_step(start, mpo, -0.2j, **SETTINGS)
    kept = start.copy()
    for _ in range(3):
        OS.cbe_bug_step(kept, mpo, -0.3j, **SETTINGS)
    return start, kept


@pytest.mark.parametrize("case", ["exact", "admitted", "capped", "two_states"])
def test_kept_states_vs_oracle(dev, chain, case):  # noqa: F811
    DM, _ = dev
    from bondupdategalerkin_b200 import native as DN

    start, kept = chain
    kw = dict(SETTINGS, truncate=False)
    keep = [kept]
    if case == "admitted":
        kw["keep_tols"] = [1e-6]
    if case == "capped":
        kw.update(keep_tols=[1e-12], maxdim=max(max(start.bond_dims()), 2), work_ceiling_rule="bond")
    if case == "two_states":
        keep = [kept, start]
        kw["keep_tols"] = [0.0, 1e-6]
    ops = start.copy()
    oi = OS.cbe_bug_step(ops, OM.xxz_mpo(L, J=1.0, delta=1.0), -0.2j, keep_states=keep,
                         rng=np.random.default_rng(0), **kw)
    dps = _upload(DM, start)
    di = DN.cbe_bug_step(dps, DM.xxz_mpo(L, J=1.0, delta=1.0), -0.2j,
                         keep_states=[_upload(DM, k) for k in keep],
                         rng=np.random.default_rng(0), **kw)
    assert di["expanded"] == oi["expanded"]
    assert di["bond_dims"] == oi["bond_dims"]
    assert di["status"] == oi["status"]
    assert 1.0 - fidelity(mps_to_host(dps), ops) <= 1e-12


def _projector(frame, left):
    """The dense orthogonal projector onto a frame's span (left: over (link, site); right: over
    (site, link))."""
    from oracle import blocks as OB

    d = OB.to_dense(frame)
    m = d.reshape(-1, d.shape[2]) if left else d.reshape(d.shape[0], -1).T
    return m @ m.conj().T


@pytest.mark.parametrize("frames_only", [False, True])
def test_frames_report_and_frames_only_vs_oracle(dev, chain, frames_only):  # noqa: F811
    """``frames_report`` hands back the frames the step integrated in, ``frames_only`` skips the
    root solve (``bug_step.jl:381-382, 455-467``): the device's frames span the oracle's (dense
    projectors within 1e-10) and a frames-only step returns the state itself."""
    DM, _ = dev
    from bondupdategalerkin_b200 import native as DN

    start, _ = chain
    kw = dict(SETTINGS, truncate=False, frames_only=frames_only)
    orep, drep = {}, {}
    ops = start.copy()
    OS.cbe_bug_step(ops, OM.xxz_mpo(L, J=1.0, delta=1.0), -0.2j, frames_report=orep,
                    rng=np.random.default_rng(0), **kw)
    dps = _upload(DM, start)
    di = DN.cbe_bug_step(dps, DM.xxz_mpo(L, J=1.0, delta=1.0), -0.2j, frames_report=drep,
                         rng=np.random.default_rng(0), **kw)
    assert drep["root_link"] == orep["root_link"]
    assert sorted(drep["left_frames"]) == sorted(orep["left_frames"])
    assert sorted(drep["right_frames"]) == sorted(orep["right_frames"])
    for side, left in (("left_frames", True), ("right_frames", False)):
        for b, f in orep[side].items():
            pd = _projector(to_host(drep[side][b]), left)
            assert np.max(np.abs(pd - _projector(f, left))) <= 1e-10, (side, b)
    assert drep["lenv"] is not None and drep["renv"] is not None
    assert 1.0 - fidelity(mps_to_host(dps), ops) <= 1e-12
    if frames_only:
        assert 1.0 - fidelity(mps_to_host(dps), start) <= 1e-12
        assert di["ledger"].expv_iters == 0
