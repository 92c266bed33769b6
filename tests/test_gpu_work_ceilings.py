"""The work-ceiling rules ``:bond_strict`` and ``:frame_root`` on the device, against the oracle
(GPU).

The device step takes its per-bond ceilings from ``bug_work_ceilings`` (checked against the
oracle's on the CPU in ``test_ceiling_rules.py``); here the whole step runs under each rule on the
XXZ domain-wall quench (L = 12, delta = 0.5, order 2, tol_basis 1e-4), where the ceilings bind on
18-19 bond visits over six steps, and is held to the oracle's at the bars of the serial parity
tests (bond dimensions, verdicts, widths and Krylov iterations every step; infidelity <= 1e-12,
S^z <= 1e-10).
"""

import pytest

from tests.test_gpu_step import dev, run_pair  # noqa: F401  (the module fixture)

pytestmark = pytest.mark.gpu

CASES = {
    "frame_root": dict(work_ceiling_rule="frame_root", bond_ceiling_factor=2.0,
                       root_ceiling_factor=1.2),
    "frame_root_checked": dict(work_ceiling_rule="frame_root", bond_ceiling_factor=2.0,
                               root_ceiling_factor=1.2, closure_checks=True),
    "bond_strict": dict(work_ceiling_rule="bond_strict", bond_ceiling_factor=1.5),
}


@pytest.mark.parametrize("case", list(CASES))
def test_ceiling_rule_vs_oracle(dev, case):  # noqa: F811
    run_pair(dev, 12, 6, "domain_wall_state", 0.5, 2, tol_basis=1e-4, maxdim=64, check_every=2,
             **CASES[case])
