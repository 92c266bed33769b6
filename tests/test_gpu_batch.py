"""Chains stepped together (``bug_step_batch``) against the same chains stepped one at a time (GPU).

A batch runs every chain's sweep logic on its own host thread and context: each with its own
stream, or (``combine``) all on one stream with the chains' queued stages merged into shared
launches (one thread-block cluster per chain). The kernels are deterministic and each chain draws from its own generator, so every chain
must come out bit-identical to its own ``cbe_bug_step``: the same bond dimensions, verdicts and
site tensors to the last bit, at every step. The chains differ in length, anisotropy, start state
and maxdim, so their stage lists differ in length and shape within each merged launch.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CHAINS = [  # (L, delta, start, maxdim, seed)
    (12, 0.5, "domain_wall_state", 32, 11),
    (16, -0.3, "neel_state", 64, 12),
    (10, 1.0, "domain_wall_state", 32, 13),
    (20, 0.0, "neel_state", 64, 14),
]
STEPS = 4
KW = dict(order=2, tol_basis=1e-4)


def _on_ctx(t, ctx):
    from bondupdategalerkin_b200 import tensor as DT

    legs, blocks = DT.to_blocks(t)
    return DT.from_blocks(legs, blocks, ctx)


@pytest.mark.parametrize("combine", [False, True], ids=["stream-per-chain", "merged-launches"])
def test_batch_matches_solo_steps(combine):
    from bondupdategalerkin_b200 import build
    from bondupdategalerkin_b200 import models as DM
    from bondupdategalerkin_b200 import native as DN
    from bondupdategalerkin_b200 import tensor as DT

    build.build()
    batch = DN.Batch(len(CHAINS), combine=combine)
    bat, bat_mpo = [], []
    solo, solo_mpo, srng, brng = [], [], [], []
    for i, (L, delta, start, maxdim, seed) in enumerate(CHAINS):
        psi = getattr(DM, start)(L)
        mpo = DM.xxz_mpo(L, J=1.0, delta=delta)
        solo.append(psi)
        solo_mpo.append(mpo)
        ctx = batch.contexts[i]
        bat.append(DM.MPS([_on_ctx(t, ctx) for t in psi.tensors], psi.center))
        bat_mpo.append(DM.MPO([_on_ctx(w, ctx) for w in mpo.tensors]))
        srng.append(np.random.default_rng(seed))
        brng.append(np.random.default_rng(seed))
    launches0 = batch.launches()
    groups = {}  # the keywords are shared by a call: one batched call per distinct maxdim
    for i, c in enumerate(CHAINS):
        groups.setdefault(c[3], []).append(i)
    for n in range(1, STEPS + 1):
        solo_info = [DN.cbe_bug_step(solo[i], solo_mpo[i], -0.05j, rng=srng[i],
                                     maxdim=CHAINS[i][3], **KW) for i in range(len(CHAINS))]
        got = {}
        for md, idx in groups.items():
            res = batch.step([bat[i] for i in idx], [bat_mpo[i] for i in idx],
                             [-0.05j] * len(idx), [brng[i] for i in idx], maxdim=md, **KW)
            got.update(dict(zip(idx, res)))
        for i in range(len(CHAINS)):
            a, b = solo_info[i], got[i]
            assert a["bond_dims"] == b["bond_dims"], (n, i)
            assert a["status"] == b["status"], (n, i)
            assert a["ledger"].expv_iters == b["ledger"].expv_iters, (n, i)
            assert a["expanded"] == b["expanded"], (n, i)
            for ts, tb in zip(solo[i].tensors, bat[i].tensors):
                _, bs = DT.to_blocks(ts)
                _, bb = DT.to_blocks(tb)
                assert sorted(bs) == sorted(bb), (n, i)
                for k in bs:
                    assert np.array_equal(bs[k], bb[k]), (n, i, k)
    assert batch.launches() > launches0
