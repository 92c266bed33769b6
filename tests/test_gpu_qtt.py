"""The device BUG step on the Heston quantics workload against the CPU oracle (GPU).

Symmetry ``:none`` (one dense block per tensor), a non-Hermitian generator (Arnoldi), real step
tau = 0.02, the separable start exp(0.5 x) exp(-v). The device state is built by the product's
builders (carry-automaton MPO, device canonical moves), the oracle's by its own route (dense
TT-SVD); both draw their Gaussians from generators seeded alike. After every step: identical bond
dimensions, ledger verdict and unmet checks, expv iterations; state infidelity <= 1e-12 (the
normalised overlap; the generator does not conserve the norm, so the norms are compared too,
to 1e-10 relative).

On 10 + 10 bits the step is ill-conditioned in the state's NORM (the generator's spectrum
reaches ~1e5, tau |A| ~ 1e3): perturbing the oracle's own input by 1e-15 moves its norm by ~1e-8
after two steps and ~1e-5 after three, with bond dimensions and verdicts unchanged. No FP64
implementation short of bit-identical arithmetic meets a fixed 1e-10 norm bar there, so the
full-size cases run two perturbed oracle copies beside the reference one and hold the device to
max(1e-10, 10x the oracle's own spread); dimensions, verdicts, expv iterations and the 1e-12
infidelity bar stay exact. The product's MPO (carry automaton) and the oracle's (dense TT-SVD)
are two compressions of one generator, so one full-size case uploads the oracle's MPO (its copies
perturb the state) and one runs the product's (its copies perturb the MPO cores at 1e-14, another
compression of the same generator).
"""

import numpy as np
import pytest

from oracle import qtt as Q
from oracle import step as OS
from tests.gpu_util import mps_to_host, overlap, perturbed_mpo

pytestmark = pytest.mark.gpu

HP = (0.03, 0.01, 2.0, 0.09, 0.4, -0.7)


def _norm(psi):
    t = psi[psi.center]
    return np.sqrt(sum(np.vdot(b, b).real for b in t.blocks.values()))


def _perturbed(psi, seed, eps=1e-15):
    """A copy of the oracle state with its first site tensor perturbed by eps (relative)."""
    from oracle.blocks import BT

    q = psi.copy()
    t = q[1]
    r = np.random.default_rng(seed)
    q[1] = BT(t.legs, {k: v * (1 + eps * r.standard_normal(v.shape)) for k, v in t.blocks.items()})
    return q


def _perturbed_mpo(mpo, seed, eps=1e-14):
    return perturbed_mpo(mpo, seed, eps)


def run_heston(nbits, steps, maxdim, native, mpo_from="product", norm_tol=1e-10, spread=None,
               dom=None, hp=HP, fx=None, fv=None, **kw):
    from bondupdategalerkin_b200 import build

    build.build()
    from bondupdategalerkin_b200 import native as DN
    from bondupdategalerkin_b200 import qtt as P

    dstep = DN.cbe_bug_step
    dom = dom or dict(x=(-1.0, 1.0), y=(0.0, 0.5), periodic_x=False, periodic_y=False)
    og, pg = Q.qtt_grid(nbits, nbits, **dom), P.qtt_grid(nbits, nbits, **dom)
    fx = fx or (lambda x: np.exp(0.5 * x))
    fv = fv or (lambda v: np.exp(-v))
    opsi = Q.qtt_mps(Q.qtt_separable(og, fx, fv), center=1)
    dpsi = P.qtt_mps(P.qtt_separable(pg, fx, fv), center=1)
    ompo = Q.heston_mpo(og, Q.HestonParams(*hp))
    if mpo_from == "product":
        dmpo = P.heston_mpo(pg, P.HestonParams(*hp))
    else:
        from bondupdategalerkin_b200 import models as DM
        from tests.gpu_util import to_dev

        dmpo = DM.MPO([to_dev(t) for t in ompo.tensors])
    orng, drng = np.random.default_rng(1234), np.random.default_rng(1234)
    # the oracle's own spread: copies with the state (or the MPO) perturbed at roundoff level
    copies = []
    for s in ((1, 2) if spread else ()):
        if spread == "state":
            copies.append((_perturbed(opsi, s), ompo, np.random.default_rng(1234)))
        else:
            copies.append((opsi.copy(), _perturbed_mpo(ompo, s), np.random.default_rng(1234)))
    for n in range(1, steps + 1):
        oi = OS.cbe_bug_step(opsi, ompo, 0.02, maxdim=maxdim, hermitian=False, rng=orng, **kw)
        tol = norm_tol
        for cpsi, cmpo, crng in copies:
            OS.cbe_bug_step(cpsi, cmpo, 0.02, maxdim=maxdim, hermitian=False, rng=crng, **kw)
            tol = max(tol, 10.0 * abs(_norm(cpsi) - _norm(opsi)) / _norm(opsi))
        di = dstep(dpsi, dmpo, 0.02, maxdim=maxdim, hermitian=False, rng=drng, **kw)
        assert di["bond_dims"] == oi["bond_dims"], (n, di["bond_dims"], oi["bond_dims"])
        assert di["status"] == oi["status"], n
        assert di["ledger"].unmet == oi["ledger"].unmet, n
        assert di["ledger"].expv_iters == oi["ledger"].expv_iters, n
        h = mps_to_host(dpsi)
        ab = overlap(h, opsi)
        aa, bb = overlap(h, h).real, overlap(opsi, opsi).real
        inf = 1.0 - abs(ab) ** 2 / (aa * bb)
        assert inf <= 1e-12, (n, inf)
        assert abs(np.sqrt(aa) - np.sqrt(bb)) <= tol * np.sqrt(bb), (n, tol)
    return opsi, dpsi


@pytest.mark.parametrize("native", [pytest.param(True, id="native-step")])
def test_heston_4x4_bits(native):
    run_heston(4, 4, 64, native, tol_basis=1e-8, tol_trunc=1e-12)


def test_heston_10x10_bits_config():
    """The config's grid (10 + 10 bits, maxdim 64), first steps (the oracle takes seconds each),
    with the oracle's MPO on both sides."""
    run_heston(10, 3, 64, True, mpo_from="oracle", spread="state")


def test_heston_10x10_bits_product_mpo():
    """The same with the product's own MPO on device."""
    run_heston(10, 2, 64, True, spread="mpo")


def test_heston_backward_fixture():
    """The reference's frozen Heston backward pricing run (5 + 5 bits, x in [-3, 3], v in [0, 1],
    r 0.03 q 0 kappa 1.5 theta 0.09 sigma 0.5 rho -0.7, softplus payoff, ten steps of 0.02):
    the native step on the product's builders follows the oracle step by step (dimensions,
    verdicts, iterations, infidelity <= 1e-12) and ends within 1e-4 of the frozen final state,
    as the oracle does (2.8e-5)."""
    import json
    import os

    d = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "b155550.json")))
    d = d["qtt_heston_backward"]
    ref = np.array(d["final_state"]["re"]) + 1j * np.array(d["final_state"]["im"])

    def payoff(x):
        z = (np.exp(x) - 1.0) / 0.02
        return 0.02 * (z if z > 30 else np.log1p(np.exp(z)))

    dom = dict(x=(-3.0, 3.0), y=(0.0, 1.0), periodic_x=False, periodic_y=False)
    opsi, dpsi = run_heston(d["N"], d["steps"], 64, True, dom=dom,
                            hp=(0.03, 0.0, 1.5, 0.09, 0.5, -0.7), fx=payoff, fv=lambda v: 1.0,
                            order=2, tol_basis=1e-8, tol_trunc=1e-10)
    dense = Q.qtt_dense(mps_to_host(dpsi))
    err = np.linalg.norm(dense - ref) / np.linalg.norm(ref)
    assert err < 1e-4, err


def test_qtt_bug_step_linear_flow_on_device():
    """``qtt_bug_step!`` on the Heston linear flow (the rational Radau IIA(2) root, unshifted) on the
    device from the reference's frozen Heston backward start (5 + 5 bits, ten steps of 0.02,
    tol_basis 1e-8, work ceiling at maxdim), the product's MPO against the oracle's.

    The root's Arnoldi stop on this generator is a near tie: the oracle's own iteration count moves
    between 7 and 11 (steps 8, 9) or 11 and 12 (step 6) when its MPO cores are perturbed at 1e-14
    (another compression of the same generator), and the enrichment widths move with it, which
    parts the Gaussian streams from there on. So every step holds the device to the oracle's
    bond dimensions exactly, to its verdict and Arnoldi count or those of one of six perturbed
    oracle copies, to a converged root, and to the oracle's state (infidelity <= 1e-12, norm
    within 1e-10); the final state lies within 5e-8 of the frozen one (the oracle: 7.1e-9)."""
    import json
    import os

    from bondupdategalerkin_b200 import build

    build.build()
    from bondupdategalerkin_b200 import qtt as P

    d = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "b155550.json")))
    d = d["qtt_heston_backward"]
    ref = np.array(d["final_state"]["re"]) + 1j * np.array(d["final_state"]["im"])

    def payoff(x):
        z = (np.exp(x) - 1.0) / 0.02
        return 0.02 * (z if z > 30 else np.log1p(np.exp(z)))

    dom = dict(x=(-3.0, 3.0), y=(0.0, 1.0), periodic_x=False, periodic_y=False)
    hp = (0.03, 0.0, 1.5, 0.09, 0.5, -0.7)
    og, pg = Q.qtt_grid(d["N"], d["N"], **dom), P.qtt_grid(d["N"], d["N"], **dom)
    ompo, dmpo = Q.heston_mpo(og, Q.HestonParams(*hp)), P.heston_mpo(pg, P.HestonParams(*hp))
    kw = dict(order=d["order"], maxdim=64, tol_trunc=1e-10, tol_stage=1e-9, tol_basis=1e-8,
              tol_scaling="fixed", work_ceiling_rule="maxdim")
    h = d["h"]

    def start(mod, grid):
        return mod.qtt_mps(mod.qtt_separable(grid, payoff, lambda v: 1.0, tol=1e-12))

    # the oracle and six copies with the MPO perturbed at 1e-14: the decisions each step admits
    runs = [(start(Q, og), mpo, np.random.default_rng(1234))
            for mpo in [ompo] + [_perturbed_mpo(ompo, s) for s in range(1, 7)]]
    opsi = runs[0][0]
    dpsi, drng = start(P, pg), np.random.default_rng(1234)
    for k in range(d["steps"]):
        reps = [Q.qtt_bug_step(psi, mpo, k * h, h, rng=rng, **kw) for psi, mpo, rng in runs]
        drep = P.qtt_bug_step(dpsi, dmpo, k * h, h, rng=drng, **kw)
        assert drep["bond_dims"] == reps[0]["bond_dims"], k
        assert drep["status"] in {r["status"] for r in reps} and drep["converged"], k
        assert drep["krylov"] in {r["krylov"] for r in reps}, (k, drep["krylov"], reps[0]["krylov"])
        hst = mps_to_host(dpsi)
        ab = overlap(hst, opsi)
        aa, bb = overlap(hst, hst).real, overlap(opsi, opsi).real
        assert 1.0 - abs(ab) ** 2 / (aa * bb) <= 1e-12, k
        assert abs(np.sqrt(aa) - np.sqrt(bb)) <= 1e-10 * np.sqrt(bb), k
    dense = Q.qtt_dense(mps_to_host(dpsi))
    assert np.linalg.norm(dense - ref) / np.linalg.norm(ref) < 5e-8
