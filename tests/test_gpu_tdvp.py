"""The device two-site TDVP baseline (``bug_tdvp2_step``) against the reference's frozen run and
against the CPU restatement (``oracle/tdvp.py``) on identical inputs."""

import json
import os

import numpy as np
import pytest

from oracle import models as OM
from oracle import tdvp as OT
from tests.gpu_util import fidelity, mps_to_host

pytestmark = pytest.mark.gpu
GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "b155550.json")))


@pytest.fixture(scope="module")
def dev():
    from bondupdategalerkin_b200 import build

    build.build()
    from bondupdategalerkin_b200 import models as DM
    from bondupdategalerkin_b200 import native as N

    return DM, N


def test_tdvp2_frozen_xx_trajectory(dev):
    """The reference's ``baseline_tdvp2_xx`` run (L = 10 XX from Neel, dt 0.05, maxdim 64,
    trunc_thresh 1e-12), all 20 steps: the frozen bond dimensions, S^z within 1e-12 of the frozen
    values, and within 2 err_exact + 1e-6 of free fermions (the reference test's bar)."""
    DM, N = dev
    fz = GOLDEN["baseline_tdvp2_xx"]
    L, dt = fz["L"], fz["dt"]
    psi = DM.neel_state(L)
    mpo = DM.xxz_mpo(L, J=1.0, delta=0.0)
    for step, row in enumerate(fz["trajectory"], start=1):
        info = N.tdvp2_step(psi, mpo, -1j * dt, maxdim=64, trunc_thresh=1e-12)
        sz = N.observable_sz(psi)
        exact = OM.free_fermion_sz(L, step * dt, occupied=range(0, L, 2))
        assert psi.bond_dims() == row["bond_dims"], step
        assert np.max(np.abs(sz - np.array(row["sz"]))) <= 1e-12, step
        assert np.max(np.abs(sz - exact)) <= 2 * row["err_exact"] + 1e-6, step
        assert info["max_bond"] == max(row["bond_dims"])


CASES = {
    "real_time_lanczos": dict(L=10, start="domain_wall_state", delta=0.5, tau=-0.05j,
                              kw=dict(maxdim=16, trunc_thresh=1e-10)),
    "imag_time_arnoldi_shift_budget": dict(L=8, start="neel_state", delta=1.0, tau=-0.1,
                                           kw=dict(maxdim=12, hermitian=False, eshift=-3.0,
                                                   weight_tol=1e-6, substeps=2, conv_tol=1e-12)),
}


@pytest.mark.parametrize("name", list(CASES))
def test_tdvp2_matches_oracle(dev, name):
    DM, N = dev
    c = CASES[name]
    opsi = getattr(OM, c["start"])(c["L"])
    dpsi = getattr(DM, c["start"])(c["L"])
    ompo = OM.xxz_mpo(c["L"], J=1.0, delta=c["delta"])
    dmpo = DM.xxz_mpo(c["L"], J=1.0, delta=c["delta"])
    for step in range(1, 4):
        oi = OT.tdvp2_step(opsi, ompo, c["tau"], **c["kw"])
        di = N.tdvp2_step(dpsi, dmpo, c["tau"], **c["kw"])
        assert dpsi.bond_dims() == opsi.bond_dims(), step
        for f in ("max_bond", "theta_elements", "peak_elements", "krylov_dims"):
            assert di[f] == oi[f], (step, f)
        for f in ("discarded", "cumulative"):
            assert abs(di[f] - oi[f]) <= 1e-8 * max(abs(oi[f]), 1e-300) + 1e-14, (step, f)
        h = mps_to_host(dpsi)
        assert 1.0 - fidelity(h, opsi) <= 1e-12, step
        so, sd = OM.sz_profile(opsi), OM.sz_profile(h)
        assert np.max(np.abs(sd - so)) <= 1e-10 * max(np.max(np.abs(so)), 1e-300), step
