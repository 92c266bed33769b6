"""``closure_probe`` in the oracle: the order-1 frontier measurement (CPU).

With ``order = 1`` and ``closure_probe = n > 0`` the step measures the root generator's frontiers
0..n-1 on the frames the half-sweeps built (``_measure_frontiers``, ``frontier_closure.jl:289-359``)
on a copy of its generator and leaves the frames alone (``bug_step_stages.jl:221-236``): the step
itself is bit-identical to the plain one, and the ledger gains the frontiers' leaks
(``leak_initial``) and scale-free ``||(I - P) A F_j|| / ||F_j||`` (``rho_initial``,
``basis_budget.jl:219-225``). The reference has no test of its own for it; these check that
contract.
"""

import numpy as np
import pytest

from oracle import models as M
from oracle import step as S


def _run(probe, parallel=False, steps=3, L=12):
    psi = M.domain_wall_state(L)
    mpo = M.xxz_mpo(L, J=1.0, delta=0.5)
    rng = np.random.default_rng(21)
    infos = [S.cbe_bug_step(psi, mpo, -0.05j, order=1, tol_basis=1e-4, maxdim=64, rng=rng,
                            closure_probe=probe, parallel=parallel) for _ in range(steps)]
    return psi, infos, rng


@pytest.mark.parametrize("parallel", [False, True])
def test_probe_leaves_the_step_bit_identical(parallel):
    a, ia, ra = _run(0, parallel)
    b, ib, rb = _run(3, parallel)
    assert ra.bit_generator.state == rb.bit_generator.state
    assert [i["bond_dims"] for i in ia] == [i["bond_dims"] for i in ib]
    assert [i["status"] for i in ia] == [i["status"] for i in ib]
    for s in range(1, len(a) + 1):
        assert sorted(a[s].blocks) == sorted(b[s].blocks)
        for k, v in a[s].blocks.items():
            assert np.array_equal(v, b[s].blocks[k])


def test_probe_records_the_frontiers():
    _, plain, _ = _run(0)
    _, probed, _ = _run(3)
    for p, q in zip(plain, probed):
        assert p["ledger"].rho_initial == [] and p["ledger"].leak_initial == []
        lg = q["ledger"]
        assert len(lg.rho_initial) == len(lg.leak_initial) == 3
        assert all(np.isfinite(x) and x >= 0 for x in lg.rho_initial + lg.leak_initial)
        assert lg.n_root_frontier == 2  # frontiers 1 and 2 from two root applications
    assert any(q["ledger"].rho_initial[1] > 0 for q in probed)


def test_negative_probe_is_refused():
    psi, mpo = M.domain_wall_state(6), M.xxz_mpo(6, J=1.0, delta=0.5)
    with pytest.raises(ValueError, match="closure_probe"):
        S.cbe_bug_step(psi, mpo, -0.05j, closure_probe=-1)
