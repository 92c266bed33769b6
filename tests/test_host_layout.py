"""The flat host layout of many tensors (``tensor.HostTensors``): host-side packing round trip."""

import numpy as np

from bondupdategalerkin_b200 import tensor as DT
from tests.gpu_util import rand_bt


def test_host_layout_round_trip():
    rng = np.random.default_rng(4)
    ts = [rand_bt(rng, (-1, -1, 1), ({0: 2, 1: 3}, {-1: 1, 1: 1}, {0: 2, 1: 3, 2: 1}), 0.8)
          for _ in range(5)]
    ts.append(rand_bt(rng, (-1, 1), ({0: 3}, {0: 3}), 1.0))
    host = [([DT.Leg(l.dir, l.sectors) for l in t.legs], t.blocks) for t in ts]
    ht = DT.host_from_blocks(host)
    assert len(ht) == len(ts)
    back = DT.host_to_blocks(ht)
    for (legs, blocks), t in zip(back, ts):
        assert [(l.dir, l.sectors) for l in legs] == [(l.dir, dict(l.sectors)) for l in t.legs]
        assert sorted(blocks) == sorted(t.blocks)
        for k, v in t.blocks.items():
            assert np.array_equal(blocks[k], v)
