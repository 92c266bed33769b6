"""The native job server (batched / served chains) on the GPU.

* a job on the server gives bit-for-bit the state of the same steps taken directly;
* each chain's result is the same alone and in a mix of concurrently running chains (different
  lengths, couplings and seeds on four workers), and the mix did run concurrently;
* admission by projected footprint: with a budget that fits one chain at a time the running
  intervals never overlap and jobs start in FIFO order; a queued job can be cancelled.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    from bondupdategalerkin_b200 import build

    build.build()
    from bondupdategalerkin_b200 import models as DM
    from bondupdategalerkin_b200 import native as DN
    from bondupdategalerkin_b200 import server as S

    return DM, DN, S


def chain(DM, S, L, delta, spins_seed):
    rng = np.random.default_rng(spins_seed)
    spins = ["up"] * (L // 2) + ["down"] * (L - L // 2)
    rng.shuffle(spins)
    psi = DM.product_state(spins)
    mpo = DM.xxz_mpo(L, J=1.0, delta=delta)
    return psi, mpo, S.host_blocks(psi.tensors), S.host_blocks(mpo.tensors)


KW = dict(order=2, tol_basis=1e-4, maxdim=64)


def same_blocks(a, b):
    assert len(a) == len(b)
    for (la, ba), (lb, bb) in zip(a, b):
        assert [(l.dir, l.sectors) for l in la] == [(l.dir, l.sectors) for l in lb]
        assert ba.keys() == bb.keys()
        for k in ba:
            assert np.array_equal(ba[k], bb[k]), k


def test_server_job_matches_direct_steps(lib):
    DM, DN, S = lib
    psi, mpo, hs, hm = chain(DM, S, 12, 0.5, 3)
    rng = np.random.default_rng(7)
    for _ in range(4):
        DN.cbe_bug_step(psi, mpo, -0.02j, rng=rng, **KW)
    direct = S.host_blocks(psi.tensors)
    with S.Server(workers=1) as srv:
        job = srv.submit(hs, len(hs), hm, -0.02j, 4, seed=7, **KW)
        assert srv.wait(timeout=600)
        st = job.stats
        assert st["state"] == "done" and st["steps_done"] == 4 and len(st["step_s"]) == 4, st
        assert job.error is None
        same_blocks(job.result, direct)
        assert job.result_center == psi.center


def test_alone_and_in_a_mix_are_identical(lib):
    DM, DN, S = lib
    specs = [(10, 0.5, 1, 11), (16, -0.3, 2, 12), (12, 1.0, 3, 13), (20, 0.0, 4, 14), (14, 0.7, 5, 15)]
    inputs = [chain(DM, S, L, d, s)[2:] for L, d, s, _ in specs]
    alone = []
    with S.Server(workers=1) as srv:
        for (hs, hm), (_, _, _, seed) in zip(inputs, specs):
            job = srv.submit(hs, len(hs), hm, -0.02j, 3, seed=seed, **KW)
            assert srv.wait(job, timeout=600)
            alone.append(job.result)
    with S.Server(workers=4) as srv:
        jobs = [srv.submit(hs, len(hs), hm, -0.02j, 3, seed=seed, **KW)
                for (hs, hm), (_, _, _, seed) in zip(inputs, specs)]
        assert srv.wait(timeout=600)
        stats = [j.stats for j in jobs]
        for j, ref in zip(jobs, alone):
            assert j.error is None
            same_blocks(j.result, ref)
    assert all(s["state"] == "done" for s in stats)
    assert len({s["worker"] for s in stats}) > 1
    iv = sorted((s["t_start"], s["t_end"]) for s in stats)
    assert any(b[0] < a[1] for a, b in zip(iv, iv[1:])), iv  # some jobs ran at the same time


def test_admission_by_footprint_and_cancel(lib):
    DM, DN, S = lib
    inputs = [chain(DM, S, 10, 0.5, s)[2:] for s in range(4)]
    fp = S.projected_footprint(10, 2, 64, 5)
    with S.Server(workers=4, budget_bytes=fp + fp // 2) as srv:  # one job at a time fits
        jobs = [srv.submit(hs, len(hs), hm, -0.02j, 2, seed=i, **KW) for i, (hs, hm) in enumerate(inputs)]
        extra = srv.submit(inputs[0][0], len(inputs[0][0]), inputs[0][1], -0.02j, 50, seed=9, **KW)
        srv.cancel(extra)
        assert srv.wait(timeout=600)
        stats = [j.stats for j in jobs]
        assert srv.wait(extra, timeout=1)
        assert extra.stats["state"] in ("cancelled", "done")
    iv = [(s["t_start"], s["t_end"]) for s in stats]
    assert all(b[0] >= a[1] for a, b in zip(iv, iv[1:])), iv  # FIFO, never two at once
    assert all(s["state"] == "done" and s["t_submit"] <= s["t_start"] for s in stats)
