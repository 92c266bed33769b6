"""``exact = true`` and ``fold_omega = false`` on the device, against the oracle (GPU).

``exact = true`` sketches the complete DD-projected fused basis at every expansion and keeps what
the two-pass pivoted QR admits (``_dd_probe(...; exact = true)``, ``dd_cbe.jl:140-161``;
``dd_cbe_expand.jl:91,346-360``); above order 1 it makes the exact two-site leak the default
(``bug_step_stages.jl:67``, ``krylov_frontier_bonds.jl:80-100``). The device step is held to the
oracle's at the bars of the serial parity tests (bond dimensions, verdicts, widths and Krylov
iterations every step; infidelity <= 1e-12, S^z <= 1e-10; the count of selected directions may
equal that of an oracle copy whose MPO is perturbed at 1e-14, since the full-basis sketch leaves
pivots at round-off level beside the QR's floor), and to the reference's own invariants
(``test_parallel_half_sweeps.jl:35-44``): serial and parallel agree to round-off with the same
verdicts, and an exact step draws no random numbers.
"""

import numpy as np
import pytest

from tests.gpu_util import fidelity, mps_to_host
from tests.test_gpu_step import dev, run_pair  # noqa: F401  (the module fixture)

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("order", [1, 2])
def test_exact_xxz_quench_vs_oracle(dev, order):  # noqa: F811
    run_pair(dev, 16, 8, "domain_wall_state", 0.5, order, tol_basis=1e-4, maxdim=64,
             check_every=2, exact=True, selected_ties=2)


def test_exact_order3_neel_vs_oracle(dev):  # noqa: F811
    run_pair(dev, 8, 3, "neel_state", 1.0, 3, tau=-0.2j, tol_basis=1e-8, tol_root=1e-12,
             tol_trunc=1e-12, maxdim=64, exact=True)


def test_exact_wide_bonds_vs_oracle(dev):  # noqa: F811
    """Bonds grow to 34 and frames to 48 in four steps: exact probes of up to about seventy
    columns per expansion. A direction admitted at the QR floor in one run and not in the other is
    a real direction of the frame, and the Galerkin step moves along it: the oracle's own copies
    with the MPO perturbed at 1e-14 differ from it in S^z by 1.7e-10 to 3.5e-10 at step 4 (the
    device: 4.2e-10) and by 7.6e-7 at step 5, where their selected counts spread over 245-248 and
    a truncation cut can fall either way. So the case stops at step 4 and its S^z bar is 1e-8;
    infidelity stays <= 1e-12."""
    run_pair(dev, 20, 4, "neel_state", 0.5, 2, tau=-0.2j, tol_basis=1e-6, maxdim=64,
             check_every=2, exact=True, selected_ties=2, sz_tol=1e-8)


def test_exact_parallel_vs_oracle(dev):  # noqa: F811
    run_pair(dev, 16, 6, "domain_wall_state", 0.5, 2, tol_basis=1e-4, maxdim=64, check_every=3,
             exact=True, parallel=True, selected_ties=2)


def test_unfolded_leak_with_randomised_selection_vs_oracle(dev):  # noqa: F811
    run_pair(dev, 16, 8, "domain_wall_state", 0.5, 2, tol_basis=1e-4, maxdim=64, check_every=2,
             fold_omega=False)


def test_exact_ignores_the_dd_mode(dev):  # noqa: F811
    run_pair(dev, 12, 5, "domain_wall_state", 0.5, 2, tol_basis=1e-4, maxdim=64, exact=True,
             expansion=dict(mode="adaptive"), selected_ties=2)


@pytest.mark.parametrize("order", [1, 2])
def test_exact_serial_equals_parallel_reference_setting(dev, order):  # noqa: F811
    DM, _ = dev
    from bondupdategalerkin_b200 import native as DN

    kw = dict(tol_basis=1e-7, tol_trunc=1e-9, tol_expv=1e-10, maxdim=64, exact=True)
    mpo = DM.xxz_mpo(6, J=1.0, delta=1.0)
    serial, par = DM.neel_state(6), DM.neel_state(6)
    rs = np.random.default_rng(9)
    before = rs.bit_generator.state
    for _ in range(2):
        a = DN.cbe_bug_step(serial, mpo, -0.05j, order=order, rng=rs, parallel=False, **kw)
        b = DN.cbe_bug_step(par, mpo, -0.05j, order=order, rng=np.random.default_rng(9),
                            parallel=True, **kw)
        assert a["status"] == b["status"]
        assert a["ledger"].n_probes == b["ledger"].n_probes == 0
    assert rs.bit_generator.state == before  # a serial exact step draws nothing
    hs, hp = mps_to_host(serial), mps_to_host(par)
    assert 1.0 - fidelity(hs, hp) < 1e-12
    assert serial.bond_dims() == par.bond_dims()
