"""``parallel = true`` on the device: the two half-sweeps, and the two halves of every frontier
sweep, run at once on the context's two streams from two host threads (GPU).

The right halves draw from streams forked off the step's generator exactly as the oracle's
``parallel = true`` does (one 64-bit draw seeds each), so the device step is held to the oracle's
parallel step at the bars of the serial parity tests: bond dimensions, verdicts, widths and root
iterations every step, infidelity <= 1e-12 and S^z <= 1e-10. The reference's own invariants
(``test_parallel_half_sweeps.jl:15-55``) follow: parallel matches serial to 1 - fidelity < 1e-8
on its L = 6 Neel setting, and repeated parallel runs agree (here bit for bit, whatever the
threads' timing).
"""

import numpy as np
import pytest

from tests.gpu_util import fidelity, mps_to_host
from tests.test_gpu_step import dev, run_pair  # noqa: F401  (the module fixture)

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("order", [1, 2])
def test_parallel_xxz_quench_vs_oracle(dev, order):  # noqa: F811
    run_pair(dev, 12, 6, "domain_wall_state", 0.5, order, tol_basis=1e-4, maxdim=32,
             check_every=2, native=True, parallel=True)


def test_parallel_headline_vs_oracle(dev):  # noqa: F811
    """The benchmark workload (L = 64, delta = 0.5, maxdim 256, tol 1e-4) with parallel = true over
    its first 25 steps."""
    run_pair(dev, 64, 25, "domain_wall_state", 0.5, 2, tol_basis=1e-4, maxdim=256, check_every=5,
             native=True, parallel=True)


def test_parallel_xx_domain_wall_rank_tail(dev):  # noqa: F811
    run_pair(dev, 20, 10, "domain_wall_state", 0.0, 2, tol_basis=1e-3, maxdim=64, check_every=5,
             native=True, parallel=True, expansion=dict(mode="rank_tail", fixed_width=8))


def _device_run(dev, parallel, L, steps, start, delta, order, seed=11, **kw):
    DM, _ = dev
    from bondupdategalerkin_b200 import native as DN

    psi = getattr(DM, start)(L)
    mpo = DM.xxz_mpo(L, J=1.0, delta=delta)
    rng = np.random.default_rng(seed)
    infos = [DN.cbe_bug_step(psi, mpo, -0.05j, order=order, rng=rng, parallel=parallel, **kw)
             for _ in range(steps)]
    return mps_to_host(psi), infos, rng


@pytest.mark.parametrize("order", [1, 2])
def test_parallel_matches_serial_reference_setting(dev, order):  # noqa: F811
    kw = dict(tol_basis=1e-7, tol_trunc=1e-9, tol_expv=1e-10, maxdim=64)
    ps, _, _ = _device_run(dev, False, 6, 2, "neel_state", 1.0, order, **kw)
    pp, _, _ = _device_run(dev, True, 6, 2, "neel_state", 1.0, order, **kw)
    assert 1.0 - fidelity(ps, pp) < 1e-8


def test_parallel_runs_repeat_bit_for_bit(dev):  # noqa: F811
    kw = dict(tol_basis=1e-4, maxdim=64)
    a, ia, ra = _device_run(dev, True, 32, 6, "domain_wall_state", 0.5, 2, **kw)
    b, ib, rb = _device_run(dev, True, 32, 6, "domain_wall_state", 0.5, 2, **kw)
    assert [i["bond_dims"] for i in ia] == [i["bond_dims"] for i in ib]
    assert ra.bit_generator.state == rb.bit_generator.state
    for s in range(1, len(a) + 1):
        assert sorted(a[s].blocks) == sorted(b[s].blocks)
        for k, v in a[s].blocks.items():
            assert np.array_equal(v, b[s].blocks[k]), (s, k)
