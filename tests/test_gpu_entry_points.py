"""The kernel-granular C-ABI entry points (env push, H1/H0 apply, sketch streams, perp, root
expv, site populations and S^z) against the oracle's functions, on an evolved XXZ state
(L = 8, delta = 0.5, three oracle steps from the domain wall) at its centre bond."""

import numpy as np
import pytest

from oracle import cbe as OC
from oracle import env as OE
from oracle import krylov as OK
from oracle import models as OM
from oracle import step as OS
from tests.gpu_util import same, to_dev, to_host

pytestmark = pytest.mark.gpu
BOND = 4


@pytest.fixture(scope="module")
def case():
    from bondupdategalerkin_b200 import build

    build.build()
    from bondupdategalerkin_b200 import native as N

    L = 8
    psi = OM.domain_wall_state(L)
    mpo = OM.xxz_mpo(L, J=1.0, delta=0.5)
    rng = np.random.default_rng(7)
    for _ in range(3):
        OS.cbe_bug_step(psi, mpo, -0.1j, order=2, rng=rng, tol_basis=1e-6, maxdim=16)
    OS.canonical(psi, BOND)
    lst = OE.left_env_stack(psi, mpo, upto=BOND - 1)
    rst = OE.right_env_stack(psi, mpo, downto=BOND + 2)
    fr = OS.frame_from(psi[BOND], psi[BOND + 1])
    return N, psi, mpo, lst, rst, fr, rng


def test_env_boundaries_and_steps(case):
    N, psi, mpo, lst, rst, fr, _ = case
    from bondupdategalerkin_b200 import _engine as E

    ctx = E.context()
    assert same(to_host(N.env_boundary(ctx, "left")), OE.left_boundary()) == 0
    q = OE.total_charge(psi)
    assert same(to_host(N.env_boundary(ctx, "right", q)), OE.right_boundary(q)) == 0
    got = to_host(N.env_step(to_dev(lst[BOND]), to_dev(psi[BOND]), to_dev(mpo[BOND]), "left"))
    assert same(got, OE.left_step(lst[BOND], psi[BOND], mpo[BOND])) < 1e-13
    got = to_host(N.env_step(to_dev(rst[BOND + 2]), to_dev(psi[BOND + 1]), to_dev(mpo[BOND + 1]),
                             "right"))
    assert same(got, OE.right_step(rst[BOND + 2], psi[BOND + 1], mpo[BOND + 1])) < 1e-13


def test_one_and_zero_site(case):
    N, psi, mpo, lst, rst, fr, _ = case
    renv = OE.right_step(rst[BOND + 2], psi[BOND + 1], mpo[BOND + 1])
    want = OE.apply_one_site(lst[BOND], mpo[BOND], renv, psi[BOND])
    got = N.apply_one_site(to_dev(lst[BOND]), to_dev(mpo[BOND]), to_dev(renv), to_dev(psi[BOND]))
    assert same(to_host(got), want) < 1e-13
    h0 = OE.ZeroSiteH(mpo, BOND, lst[BOND], rst[BOND + 2], fr.U0, fr.V0)
    got = N.apply_zero_site(to_dev(h0.l), to_dev(h0.r), to_dev(fr.S0))
    assert same(to_host(got), h0.apply(fr.S0)) < 1e-13


@pytest.mark.parametrize("hermitian", [True, False])
def test_root_expv(case, hermitian):
    N, psi, mpo, lst, rst, fr, _ = case
    h0 = OE.ZeroSiteH(mpo, BOND, lst[BOND], rst[BOND + 2], fr.U0, fr.V0)
    tau = -0.1j
    want, rep = OK.expv(OS.VOPS, h0.apply, tau, fr.S0, hermitian=hermitian, maxiter=30, tol=1e-15,
                        reorth=True, conv_tol=1e-10, substeps=0)
    got, iters, err = N.root_expv(to_dev(h0.l), to_dev(h0.r), to_dev(fr.S0), tau,
                                  hermitian=hermitian, maxiter=30, reorth=True, tol_expv=1e-10)
    assert iters == rep[0]
    # the tail estimate is the last Krylov coefficient, a sum of O(1) terms cancelling to ~1e-12:
    # it agrees to rounding of those terms (1e-16 absolute), not relatively
    assert abs(err - rep[2]) <= 1e-6 * abs(rep[2]) + 1e-16
    assert same(to_host(got), want) < 1e-12


def test_sketch_streams_and_perp(case):
    N, psi, mpo, lst, rst, fr, rng = case
    lenv, renv = lst[BOND], rst[BOND + 2]
    Om = OC.dd_probe(fr.V0, "right", 6, rng)
    core = OE.contract(fr.U0, (2,), fr.S0, (0,))
    want = OE.stream_left(core, fr.V0, mpo, BOND, lenv, renv, Om)
    got = N.sketch_stream("left", to_dev(core), to_dev(fr.V0), to_dev(mpo[BOND]),
                          to_dev(mpo[BOND + 1]), to_dev(lenv), to_dev(renv), to_dev(Om))
    assert same(to_host(got), want) < 1e-13
    assert same(to_host(N.perp("left", to_dev(fr.U0), got)), OC.perp_left(fr.U0, want)) < 1e-12
    Om = OC.dd_probe(fr.U0, "left", 6, rng)
    core = OE.contract(fr.S0, (1,), fr.V0, (0,))
    want = OE.stream_right(fr.U0, core, mpo, BOND, lenv, renv, Om)
    got = N.sketch_stream("right", to_dev(fr.U0), to_dev(core), to_dev(mpo[BOND]),
                          to_dev(mpo[BOND + 1]), to_dev(lenv), to_dev(renv), to_dev(Om))
    assert same(to_host(got), want) < 1e-13
    assert same(to_host(N.perp("right", to_dev(fr.V0), got)), OC.perp_right(fr.V0, want)) < 1e-12


@pytest.mark.parametrize("sym", ["U1", "none"])
def test_observable_sz_and_populations(sym):
    from bondupdategalerkin_b200 import build

    build.build()
    from bondupdategalerkin_b200 import models as DM
    from bondupdategalerkin_b200 import native as N
    from tests.gpu_util import mps_to_host

    L = 8
    dpsi = DM.domain_wall_state(L, symmetry=sym)
    dmpo = DM.xxz_mpo(L, J=1.0, delta=0.5, symmetry=sym)
    rng = np.random.default_rng(3)
    for _ in range(3):
        N.cbe_bug_step(dpsi, dmpo, -0.1j, order=2, rng=rng, tol_basis=1e-6, maxdim=16)
    want = OM.sz_profile(mps_to_host(dpsi))
    assert np.max(np.abs(N.observable_sz(dpsi) - want)) < 1e-12
    for p, sz in zip(N.site_populations(dpsi), want):
        assert abs(p.sum() - 1.0) < 1e-12
        up = p[1] if sym == "U1" else p[0]  # U(1): sectors (-1, +1); none: (up, down)
        assert abs(up - (0.5 + sz)) < 1e-12
