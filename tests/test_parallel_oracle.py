"""``parallel = true`` in the oracle: the reference's concurrency invariants on the CPU.

With ``parallel = true`` the right half-sweep, and the right half of every frontier sweep, draw
from a stream seeded by one 64-bit draw of the step's generator (``bug_step.jl:222-268``,
``frontier_closure.jl:121-145``); the halves touch disjoint state, so the oracle runs them one after
the other. ``test/BUG/TimeEvolution/test_parallel_half_sweeps.jl:15-55`` runs the L = 6 Neel chain
(XXZ, delta = 1, tau = -0.05i, tol_basis 1e-7, tol_trunc 1e-9, tol_expv 1e-10, maxdim 64) for two
steps at order 1 and 2: with randomised selection the parallel state matches the serial one to
1 - fidelity < 1e-8 (the sketches differ) and two parallel runs agree to < 1e-13 (here: exactly);
its exact-selection half (no draws, agreement to round-off) is in ``test_exact_oracle.py``.
"""

import numpy as np

from oracle import models as OM
from oracle import step as OS
from tests.gpu_util import fidelity


def _run(parallel, steps, L=16, seed=5, order=2):
    psi = OM.domain_wall_state(L)
    mpo = OM.xxz_mpo(L, J=1.0, delta=0.5)
    rng = np.random.default_rng(seed)
    infos = [OS.cbe_bug_step(psi, mpo, -0.05j, order=order, tol_basis=1e-4, maxdim=64, rng=rng,
                             parallel=parallel) for _ in range(steps)]
    return psi, infos, rng


def _neel(parallel, order, seed=11):
    psi = OM.neel_state(6)
    mpo = OM.xxz_mpo(6, J=1.0, delta=1.0)
    rng = np.random.default_rng(seed)
    infos = [OS.cbe_bug_step(psi, mpo, -0.05j, order=order, tol_basis=1e-7, tol_trunc=1e-9,
                             tol_expv=1e-10, maxdim=64, rng=rng, parallel=parallel)
             for _ in range(2)]
    return psi, infos


def test_parallel_matches_serial():
    for order in (1, 2):
        ps, _ = _neel(False, order)
        p1, i1 = _neel(True, order)
        p2, i2 = _neel(True, order)
        assert 1.0 - fidelity(ps, p1) < 1e-8
        assert 1.0 - fidelity(p1, p2) < 1e-13
        assert [i["status"] for i in i1] == [i["status"] for i in i2]


def test_parallel_runs_repeat_exactly():
    p1, i1, r1 = _run(True, 4)
    p2, i2, r2 = _run(True, 4)
    assert [i["bond_dims"] for i in i1] == [i["bond_dims"] for i in i2]
    for s in range(1, len(p1) + 1):
        for k, v in p1[s].blocks.items():
            assert np.array_equal(v, p2[s].blocks[k])
    assert r1.bit_generator.state == r2.bit_generator.state


def test_fork_takes_one_draw_and_seeds_from_it():
    """The fork consumes exactly one 64-bit value of the step's stream and seeds the new stream
    with it."""
    a, b = np.random.default_rng(7), np.random.default_rng(7)
    sub = OS.fork_rng(a)
    seed = int(b.integers(0, np.iinfo(np.uint64).max, dtype=np.uint64, endpoint=True))
    assert a.bit_generator.state == b.bit_generator.state
    assert np.array_equal(sub.standard_normal(8), np.random.default_rng(seed).standard_normal(8))


def test_parallel_draws_differ_from_serial():
    """The right halves really draw from the forked streams: the step generator ends elsewhere."""
    _, _, rs = _run(False, 2)
    _, _, rp = _run(True, 2)
    assert rs.bit_generator.state != rp.bit_generator.state
