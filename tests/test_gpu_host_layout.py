"""Many tensors through the flat host layout on the device (GPU): ``bug_tensors_from_host`` /
``bug_tensors_to_host`` round-trip bit for bit, and ``api.step_host_flat`` gives the device step."""

import numpy as np
import pytest

from tests.gpu_util import rand_bt

pytestmark = pytest.mark.gpu


def test_from_host_to_host_round_trip():
    from bondupdategalerkin_b200 import build

    build.build()
    from bondupdategalerkin_b200 import tensor as DT

    rng = np.random.default_rng(5)
    ts = [rand_bt(rng, (-1, -1, 1), ({0: 4, 1: 7}, {-1: 1, 1: 1}, {0: 5, 1: 2, 2: 3}), 0.8)
          for _ in range(7)]
    host = [([DT.Leg(l.dir, l.sectors) for l in t.legs], t.blocks) for t in ts]
    ht = DT.host_from_blocks(host)
    dev = DT.from_host_many(ht)
    for d, (legs, blocks) in zip(dev, host):
        dl, db = DT.to_blocks(d)
        assert [(l.dir, l.sectors) for l in dl] == [(l.dir, l.sectors) for l in legs]
        for k, v in blocks.items():
            assert np.array_equal(db[k], v)
    back = DT.to_host_many(dev)
    assert np.array_equal(back.meta, ht.meta)
    assert np.array_equal(back.payload_off, ht.payload_off)
    assert np.array_equal(back.payload[:ht.payload.size], ht.payload)


def test_step_host_flat_is_the_device_step():
    from bondupdategalerkin_b200 import build

    build.build()
    from bondupdategalerkin_b200 import models as DM
    from bondupdategalerkin_b200 import native as DN
    from bondupdategalerkin_b200 import tensor as DT
    from bondupdategalerkin_b200.api import step_host_flat

    L = 16
    psi, mpo = DM.domain_wall_state(L), DM.xxz_mpo(L, J=1.0, delta=0.5)
    state = DT.to_host_many(psi.tensors)
    hmpo = DT.to_host_many(mpo.tensors)
    center = psi.center
    r1, r2 = np.random.default_rng(9), np.random.default_rng(9)
    kw = dict(order=2, tol_basis=1e-4, maxdim=32)
    for _ in range(4):
        DN.cbe_bug_step(psi, mpo, -0.05j, rng=r1, **kw)
        state, center, io = step_host_flat(state, center, hmpo, -0.05j, rng=r2, **kw)
        assert io["h2d_bytes"] > 0 and io["d2h_bytes"] > 0
    assert center == psi.center
    ref = DT.to_host_many(psi.tensors)
    assert np.array_equal(ref.meta, state.meta)
    assert np.array_equal(ref.payload, state.payload)
