"""The device BUG step against the CPU oracle on identical inputs and identical Gaussian draws.

Both sides start from the same state, take their probes from generators seeded alike, and must
agree after every step on: bond dimensions, ledger verdict and its failed checks, the root
solve's Krylov iterations, the state (infidelity <= 1e-12) and the S^z profile (relative error
<= 1e-10). Cases: the b155550 XX fixtures' setting (L = 10 Neel, U(1) order 1 and 2, and the
no-symmetry L = 8 run), the XX domain-wall chain L = 20 at maxdim 64 and tol_basis 1e-3
(checked against free fermions as well), an XXZ quench, and the two-spin known answer.
"""

import numpy as np
import pytest

from oracle import models as OM
from oracle import step as OS
from tests.gpu_util import fidelity, mps_to_host, perturbed_mpo

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    from bondupdategalerkin_b200 import build

    build.build()
    from bondupdategalerkin_b200 import models as DM
    from bondupdategalerkin_b200 import options as DS

    return DM, DS


def run_pair(dev, L, steps, start, delta, order, sym="U1", tau=-0.05j, check_every=1,
             native=False, widths=True, selected_ties=0, sz_tol=1e-10, **kw):
    """The device step against the oracle's on the same seeded chain, step by step. With
    ``selected_ties = n`` the oracle also runs n copies whose MPO cores are perturbed at 1e-14, and
    the device's ``n_selected`` may equal any of theirs: under ``exact = true`` the first QR pass
    admits directions whose pivots sit at round-off level beside its floor, so that count is not a
    function of the exact inputs (everything else is still held to the unperturbed oracle).
    ``sz_tol`` is the bar on the relative S^z difference (default 1e-10)."""
    DM, DS = dev
    from bondupdategalerkin_b200 import native as DN

    dstep = DN.cbe_bug_step
    ostate = getattr(OM, start)(L, symmetry=sym)
    dstate = getattr(DM, start)(L, symmetry=sym)
    ompo = OM.xxz_mpo(L, J=1.0, delta=delta, symmetry=sym)
    dmpo = DM.xxz_mpo(L, J=1.0, delta=delta, symmetry=sym)
    orng, drng = np.random.default_rng(1234), np.random.default_rng(1234)
    okw = dict(kw)
    dkw = dict(kw)
    if "expansion" in kw:
        e = kw["expansion"]
        okw["expansion"] = OS.DDQRExpansion(**e)
        dkw["expansion"] = DS.DDQRExpansion(**e)
    copies = [(getattr(OM, start)(L, symmetry=sym), perturbed_mpo(ompo, s), np.random.default_rng(1234))
              for s in range(1, selected_ties + 1)]
    worst = (0.0, 0.0)
    for n in range(1, steps + 1):
        oi = OS.cbe_bug_step(ostate, ompo, tau, order=order, rng=orng, **okw)
        ties = {oi["ledger"].n_selected} | {
            OS.cbe_bug_step(p, m, tau, order=order, rng=r, **okw)["ledger"].n_selected
            for p, m, r in copies}
        di = dstep(dstate, dmpo, tau, order=order, rng=drng, **dkw)
        assert di["bond_dims"] == oi["bond_dims"], (n, di["bond_dims"], oi["bond_dims"])
        assert di["status"] == oi["status"], n
        assert di["ledger"].unmet == oi["ledger"].unmet, n
        assert di["ledger"].expv_iters == oi["ledger"].expv_iters, n
        if widths:
            assert di["expanded"] == oi["expanded"], n
            for f in ("n_probes", "n_holdout", "n_targeted"):
                assert getattr(di["ledger"], f) == getattr(oi["ledger"], f), (n, f)
            assert di["ledger"].n_selected in ties, (n, di["ledger"].n_selected, ties)
        if n % check_every == 0 or n == steps:
            h = mps_to_host(dstate)
            inf = 1.0 - fidelity(h, ostate)
            sz_o = OM.sz_profile(ostate)
            sz_d = OM.sz_profile(h)
            rel = np.max(np.abs(sz_d - sz_o)) / max(np.max(np.abs(sz_o)), 1e-300)
            worst = (max(worst[0], inf), max(worst[1], rel))
            assert inf <= 1e-12, (n, inf)
            assert rel <= sz_tol, (n, rel)
    return ostate, dstate, worst


FROZEN = dict(work_ceiling_rule="maxdim", expansion=dict(krylov_mode="arnoldi"))


HOSTS = [pytest.param(True, id="native-step")]


@pytest.mark.parametrize("native", HOSTS)
@pytest.mark.parametrize("order", [1, 2])
def test_fixture_setting_u1(dev, order, native):
    run_pair(dev, 10, 5, "neel_state", 0.0, order, native=native, **FROZEN)


@pytest.mark.parametrize("native", HOSTS)
def test_fixture_setting_none(dev, native):
    run_pair(dev, 8, 3, "neel_state", 0.0, 2, sym="none", native=native, **FROZEN)


@pytest.mark.parametrize("native", HOSTS)
def test_xx_domain_wall_l20(dev, native):
    ostate, dstate, worst = run_pair(dev, 20, 20, "domain_wall_state", 0.0, 2, tol_basis=1e-3,
                                     maxdim=64, check_every=5, native=native,
                                     expansion=dict(mode="rank_tail", fixed_width=8))
    h = mps_to_host(dstate)
    exact = OM.free_fermion_sz(20, 20 * 0.05)
    assert np.max(np.abs(OM.sz_profile(h) - exact)) < 1e-3


@pytest.mark.parametrize("native", HOSTS)
def test_xxz_quench(dev, native):
    run_pair(dev, 12, 6, "domain_wall_state", 0.5, 2, tol_basis=1e-4, maxdim=32, check_every=3,
             native=native)


@pytest.mark.parametrize("native", HOSTS)
def test_xxz_quench_l64_native_vs_oracle(dev, native):
    """The benchmark workload (L = 64, delta = 0.5, maxdim 256, tol 1e-4) over its first 25 steps,
    which include every step the default benchmark times (6..25): dimensions, verdicts, widths and
    iterations every step, the state and S^z every 5 steps."""
    run_pair(dev, 64, 25, "domain_wall_state", 0.5, 2, tol_basis=1e-4, maxdim=256, check_every=5,
             native=native)


def test_xxz_quench_l64_full_trajectory(dev):
    """The whole 100-step trajectory of the benchmark workload on the native step (chi reaches
    39): dimensions, verdicts, widths and iterations every step, the state and S^z every 10."""
    _, _, worst = run_pair(dev, 64, 100, "domain_wall_state", 0.5, 2, tol_basis=1e-4, maxdim=256,
                           check_every=10, native=True)
    assert worst[0] <= 1e-12 and worst[1] <= 1e-10


@pytest.mark.parametrize("native", HOSTS)
def test_two_spin(dev, native):
    DM, DS = dev
    from bondupdategalerkin_b200 import native as DN

    step = DN.cbe_bug_step
    mpo = DM.xxz_mpo(2, J=1.0, delta=0.0)
    psi = DM.product_state(["up", "down"])
    t = 0.3
    step(psi, mpo, -1j * t, tol_basis=1e-10, tol_trunc=1e-14, tol_expv=1e-13, maxdim=4)
    v = OM.mps_to_dense(mps_to_host(psi))
    v /= np.linalg.norm(v)
    assert abs(abs(v[1]) - np.cos(t / 2)) < 1e-10
    assert abs(abs(v[2]) - np.sin(t / 2)) < 1e-10


def test_profiled_step_identical(dev):
    """Profiling launches every operation on its own; the fused stage lists of the normal run must
    give bit-identical states (same arithmetic, same order)."""
    DM, _ = dev
    from bondupdategalerkin_b200 import _engine as E
    from bondupdategalerkin_b200 import native as DN
    from bondupdategalerkin_b200 import tensor as DT

    ctx = E.context()
    states = []
    for profile in (False, True):
        psi = DM.domain_wall_state(16)
        mpo = DM.xxz_mpo(16, J=1.0, delta=0.5)
        rng = np.random.default_rng(99)
        ctx.set_profiling(profile)
        try:
            for _ in range(6):
                DN.cbe_bug_step(psi, mpo, -0.05j, order=2, rng=rng, tol_basis=1e-4, maxdim=64)
        finally:
            ctx.set_profiling(False)
        states.append([DT.to_blocks(t) for t in psi.tensors])
    for (la, ba), (lb, bb) in zip(*states):
        assert [(l.dir, l.sectors) for l in la] == [(l.dir, l.sectors) for l in lb]
        assert ba.keys() == bb.keys()
        for k in ba:
            assert np.array_equal(ba[k], bb[k]), k


@pytest.mark.parametrize("idx", [0, 3, 7])
def test_random_sz0_chains_native_vs_oracle(dev, idx):
    """Chains of the batched workload (seeded random product states with total S^z = 0, order 2,
    tau = -0.02i): their first SVDs see many exactly degenerate and noise-level pairs."""
    DM, _ = dev
    from bondupdategalerkin_b200 import native as DN
    from bondupdategalerkin_b200 import workloads as WL

    sp = WL.batch_specs(64)[idx]
    opsi = OM.product_state(sp["spins"])
    ompo = OM.xxz_mpo(sp["L"], J=1.0, delta=sp["delta"])
    dpsi = DM.product_state(sp["spins"])
    dmpo = DM.xxz_mpo(sp["L"], J=1.0, delta=sp["delta"])
    orng, drng = np.random.default_rng(sp["seed"]), np.random.default_rng(sp["seed"])
    for n in range(1, 3):
        oi = OS.cbe_bug_step(opsi, ompo, sp["tau"], rng=orng, **sp["kw"])
        di = DN.cbe_bug_step(dpsi, dmpo, sp["tau"], rng=drng, **sp["kw"])
        assert di["bond_dims"] == oi["bond_dims"], (n, di["bond_dims"], oi["bond_dims"])
        assert di["status"] == oi["status"], n
        h = mps_to_host(dpsi)
        inf = 1.0 - fidelity(h, opsi)
        assert inf <= 1e-12, (n, inf)


ADAPTIVE = dict(work_ceiling_rule="maxdim", expansion=dict(krylov_mode="arnoldi", mode="adaptive"))


@pytest.mark.parametrize("native", HOSTS)
@pytest.mark.parametrize("order", [1, 2])
def test_adaptive_fixture_setting(dev, order, native):
    """The :adaptive DD controller (holdout-checked block growth, two-pass pivoted thin QR on
    device) in the b155550 fixtures' setting, against the oracle's controller step by step."""
    run_pair(dev, 10, 8, "neel_state", 0.0, order, native=native, **ADAPTIVE)


@pytest.mark.parametrize("native", HOSTS)
def test_adaptive_capped_vs_exact(dev, native):
    """:adaptive with a binding work cap (every step ends work-limited, the sample check unmet).
    A capped controller trims its basis to the room by column order, and the second-pass QR's
    columns all have norm 1 to within a few ulps: its pivot order, and so the trimmed subset, is
    decided by rounding (in LAPACK too). These runs are therefore compared through what does not
    depend on that choice: the verdict per step, and the error against exact evolution (sparse
    Krylov on the full 2^16 space), which must match the oracle's within half again."""
    import scipy.sparse.linalg as ssl

    DM, DS = dev
    from bondupdategalerkin_b200 import native as DN

    dstep = DN.cbe_bug_step
    L, tau = 16, -0.1j
    H = OM.sparse_xxz(L, 1.0, 0.5)
    opsi, dpsi = OM.neel_state(L), DM.neel_state(L)
    ompo, dmpo = OM.xxz_mpo(L, J=1.0, delta=0.5), DM.xxz_mpo(L, J=1.0, delta=0.5)
    orng, drng = np.random.default_rng(1234), np.random.default_rng(1234)
    v = OM.mps_to_dense(opsi)
    kw = dict(order=2, tol_basis=1e-6, maxdim=16)

    def err(w):
        return 1.0 - abs(np.vdot(v, w)) ** 2 / (np.vdot(v, v).real * np.vdot(w, w).real)

    for n in range(1, 7):
        oi = OS.cbe_bug_step(opsi, ompo, tau, rng=orng, expansion=OS.DDQRExpansion(mode="adaptive"), **kw)
        di = dstep(dpsi, dmpo, tau, rng=drng, expansion=DS.DDQRExpansion(mode="adaptive"), **kw)
        v = ssl.expm_multiply(tau * H, v)
        assert di["status"] == oi["status"] == "budget_unmet", n
        assert di["ledger"].workcap_reached and oi["ledger"].workcap_reached, n
        assert max(di["bond_dims"]) <= 16
        eo, ed = err(OM.mps_to_dense(opsi)), err(OM.mps_to_dense(mps_to_host(dpsi)))
        assert ed <= 1.5 * eo + 1e-10, (n, ed, eo)


@pytest.mark.parametrize("native", HOSTS)
def test_adaptive_targeted(dev, native):
    """:adaptive at a tight tolerance: the holdout targets sectors (boosted probe columns) in
    the last step."""
    run_pair(dev, 14, 6, "neel_state", -0.5, 2, tau=-0.1j, tol_basis=1e-8, maxdim=32,
             check_every=3, native=native, work_ceiling_rule="maxdim",
             expansion=dict(mode="adaptive"))


@pytest.mark.parametrize("native", HOSTS)
def test_adaptive_cap_selection_svd(dev, native):
    """``cap_selection = :svd``: past the cap the controller keeps the strongest directions of the
    projected sketch by SVD instead of the first columns (10 times in this run), a choice that
    does not hang on pivot order, so the run is held to the bit-level bars."""
    run_pair(dev, 16, 8, "domain_wall_state", 0.5, 2, tau=-0.1j, tol_basis=1e-6, maxdim=8,
             check_every=4, native=native, expansion=dict(mode="adaptive", cap_selection="svd"))


@pytest.mark.parametrize("native", HOSTS)
def test_adaptive_batch_blocks(dev, native):
    """``batch_blocks = 3`` (targeted blocks per holdout; two failed holdouts enter the batched
    branch here), ``holdout_width = 6`` and ``acceptance_factor = 0.5``. At tol_basis 1e-8 the
    Lanczos chains of the Krylov enrichment run long enough to amplify rounding from 1e-16 to
    1e-5 in their score SVDs, so one enrichment width of one bond can
    differ by a direction carrying no weight; the widths are not compared here, the bond
    dimensions, verdicts and states are."""
    run_pair(dev, 14, 6, "neel_state", -0.5, 2, tau=-0.1j, tol_basis=1e-8, maxdim=32,
             check_every=3, native=native, work_ceiling_rule="maxdim", widths=False,
             expansion=dict(mode="adaptive", batch_blocks=3, holdout_width=6, acceptance_factor=0.5))


@pytest.mark.parametrize("native", [pytest.param(True, id="native-step")])
def test_closure_checks(dev, native):
    """``closure_checks = true``: every frontier measured first, then the closure loop in passes
    and degree 0 measured again (``_krylov_closure!`` with checks), against the oracle: the
    Heisenberg chain from Neel in imaginary time (the closure unmet in the first steps) and an
    XXZ quench in real time."""
    run_pair(dev, 10, 3, "neel_state", 1.0, 2, tau=-0.125, maxdim=64, native=native,
             closure_checks=True)
    run_pair(dev, 12, 4, "domain_wall_state", 0.5, 2, tol_basis=1e-4, maxdim=32, check_every=2,
             native=native, closure_checks=True)


@pytest.mark.parametrize("method", ["trapezoid", "radau2", "radau3", "radau2_gmres"])
def test_implicit_root_methods(dev, method):
    """The implicit root integrators (one stage of the Pade stability function on the root's
    Krylov basis) against the oracle, in real time and, with the spectral shift, imaginary time."""
    run_pair(dev, 12, 3, "domain_wall_state", 0.5, 2, tau=-0.05j, tol_basis=1e-4, maxdim=32,
             native=True, root_method=method)
    run_pair(dev, 10, 3, "neel_state", 1.0, 2, tau=-0.1, maxdim=32, native=True,
             root_method=method)


@pytest.mark.parametrize("order", [1, 2])
def test_native_step_converges_at_order_p_plus_one(dev, order):
    """The native step on the interacting L = 10 quench (delta 0.5, domain wall, to t = 1, tight
    tolerances) against the dense exponential: global order p + 1 in tau, as the oracle's
    (error ratios 4.0 and 8.0 when tau halves; 4.4e-4 and 3.7e-6 at tau = 0.05)."""
    import scipy.linalg

    DM, _ = dev
    from bondupdategalerkin_b200 import native as DN

    L, T = 10, 1.0
    exact = scipy.linalg.expm(-1j * T * OM.dense_xxz(L, 1.0, 0.5)) @ \
        OM.mps_to_dense(OM.domain_wall_state(L))
    errs = []
    for dt in (0.1, 0.05):
        psi, mpo = DM.domain_wall_state(L), DM.xxz_mpo(L, J=1.0, delta=0.5)
        rng = np.random.default_rng(1234)
        for _ in range(int(round(T / dt))):
            info = DN.cbe_bug_step(psi, mpo, -1j * dt, order=order, tol_basis=1e-8,
                                   tol_trunc=1e-12, maxdim=256, rng=rng)
            assert info["status"] == "met"
        dense = OM.mps_to_dense(mps_to_host(psi))
        errs.append(np.linalg.norm(dense - exact) / np.linalg.norm(exact))
    assert errs[0] / errs[1] > 0.85 * 2 ** (order + 1), errs
    assert errs[1] < (1e-3 if order == 1 else 1e-5), errs


def _zero_padded_domain_wall(L):
    """The domain-wall state with a second, all-zero charge sector on its middle bond (charge
    h - 2 beside h = L / 2, reached from site h's left sector by a down spin and left into site
    h + 1's right sector by an up spin): the same state, but a canonical move across that bond
    meets singular values that are exactly zero, which the reference's cutoff-0 SVD drops."""
    from oracle.blocks import BT, Leg

    h = L // 2
    psi = OM.domain_wall_state(L)
    a, b = psi[h], psi[h + 1]
    z = np.zeros((1, 1, 1), dtype=np.complex128)
    mid = {h - 2: 1, h: 1}
    psi.tensors[h - 1] = BT([a.legs[0], a.legs[1], Leg(+1, mid)], {**a.blocks, (h - 1, -1, h - 2): z})
    psi.tensors[h] = BT([Leg(-1, mid), b.legs[1], b.legs[2]], {**b.blocks, (h - 2, 1, h - 1): z.copy()})
    return psi


@pytest.mark.parametrize("parallel", [False, True])
def test_exact_zero_singular_values_redo_the_moves(dev, parallel):
    """Canonical moves take their SVDs ahead of the read-back and assume no exactly zero singular
    value; on a state padded with an all-zero sector that assumption fails, the moves are redone
    with read-backs, and the step follows the oracle (which drops the zero sector) at the usual
    bars."""
    DM, _ = dev
    from bondupdategalerkin_b200 import native as DN
    from tests.gpu_util import to_dev

    L = 12
    ostate = _zero_padded_domain_wall(L)
    assert ostate.bond_dims()[L // 2 - 1] == 2
    dstate = DM.MPS([to_dev(t) for t in ostate.tensors], ostate.center)
    ompo, dmpo = OM.xxz_mpo(L, J=1.0, delta=0.5), DM.xxz_mpo(L, J=1.0, delta=0.5)
    orng, drng = np.random.default_rng(7), np.random.default_rng(7)
    kw = dict(order=2, tol_basis=1e-4, maxdim=32, parallel=parallel)
    for n in range(3):
        oi = OS.cbe_bug_step(ostate, ompo, -0.05j, rng=orng, **kw)
        di = DN.cbe_bug_step(dstate, dmpo, -0.05j, rng=drng, **kw)
        assert di["bond_dims"] == oi["bond_dims"], (n, di["bond_dims"], oi["bond_dims"])
        assert di["status"] == oi["status"] and di["expanded"] == oi["expanded"], n
        assert 1.0 - fidelity(mps_to_host(dstate), ostate) <= 1e-12, n


_REDO_SCRIPT = r"""
import sys, numpy as np
from bondupdategalerkin_b200 import models as DM, native as DN
from tests.gpu_util import mps_to_host
L, parallel, out = 16, sys.argv[1] == "1", sys.argv[2]
psi, mpo = DM.domain_wall_state(L), DM.xxz_mpo(L, J=1.0, delta=0.5)
rng = np.random.default_rng(3)
dims = []
for _ in range(4):
    info = DN.cbe_bug_step(psi, mpo, -0.05j, order=2, tol_basis=1e-4, maxdim=32, rng=rng,
                           parallel=parallel)
    dims.append(info["bond_dims"] + list(info["expanded"]))
h = mps_to_host(psi)
arrs = {f"{s}:{k}": v for s in range(1, L + 1) for k, v in h[s].blocks.items()}
np.savez(out, dims=np.array(dims), **{f"b{i}": arrs[k] for i, k in enumerate(sorted(arrs))},
         keys=np.array(sorted(arrs)))
"""


@pytest.mark.parametrize("parallel", [False, True])
def test_svd_ahead_redo_gives_the_same_steps(dev, tmp_path, parallel):
    """With BUG_SVD_AHEAD_REDO=1 every computation that took SVDs ahead (canonical moves, the
    projection miss, the frontier halves) is run a second time the exact way, rewinding the draws
    of a frontier half; the steps must come out bit for bit as without it."""
    import os
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    res = []
    for redo in ("0", "1"):
        out = str(tmp_path / f"run{redo}.npz")
        env = dict(os.environ, BUG_SVD_AHEAD_REDO=redo, PYTHONPATH=root)
        subprocess.run([sys.executable, "-c", _REDO_SCRIPT, "1" if parallel else "0", out],
                       check=True, cwd=root, env=env, timeout=600)
        res.append(np.load(out))
    a, b = res
    assert np.array_equal(a["dims"], b["dims"])
    assert list(a["keys"]) == list(b["keys"])
    for i in range(len(a["keys"])):
        assert np.array_equal(a[f"b{i}"], b[f"b{i}"]), a["keys"][i]
