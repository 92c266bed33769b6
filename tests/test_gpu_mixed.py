"""The tensor-core (tcgen05, 3xTF32) contraction path against the oracle (GPU).

Mixed precision computes an output block on the tensor cores when both its extents reach the
context's threshold: each FP64 operand value is split into two TF32 values (hi, lo: |x - hi - lo|
<= 2^-22 |x|) and the three products lo*hi, hi*lo, hi*hi of every complex K step, six real terms
per complex k, accumulate in FP32. With truncating FP32 adds (unit 2^-23) an element's error is
bounded by (6 K 2^-23 + 2^-21) sum_k |a_k||b_k|, the bound the contraction tests hold each element
to; blocks under the threshold stay in FP64 bit for bit. The step test runs the benchmark quench
with every contraction block on the tensor cores and records its observable error against the
FP64 oracle.
"""

import numpy as np
import pytest

from oracle import blocks as OB
from tests.gpu_util import rand_bt, to_dev, to_host

pytestmark = pytest.mark.gpu



def split_bound(K):
    """Error bound of a 3xTF32 product with FP32 accumulation over complex extent K, relative to
    sum |a||b| (see the module docstring)."""
    return 6 * K * 2.0 ** -23 + 2.0 ** -21


def _kmax(a, ia):
    """Largest contracted extent over a's blocks (product of the contracted legs' sector dims)."""
    k = 1
    for key, v in a.blocks.items():
        k = max(k, int(np.prod([v.shape[i] for i in ia])))
    return k


@pytest.fixture(scope="module")
def D():
    from bondupdategalerkin_b200 import build, tensor

    build.build()
    return tensor


@pytest.fixture
def mixed_ctx():
    from bondupdategalerkin_b200 import _engine as E

    ctx = E.context()
    yield ctx
    ctx.set_mixed(0)


def _abs(t):
    return OB.BT(t.legs, {k: np.abs(v) for k, v in t.blocks.items()})


def _rel_err(got, want, scale):
    err = 0.0
    for k, w in want.blocks.items():
        err = max(err, float(np.max(np.abs(got.blocks[k] - w) / np.maximum(scale.blocks[k], 1e-300))))
    return err


@pytest.mark.parametrize("case", range(8))
def test_mixed_contract_matches_oracle(D, mixed_ctx, case):
    """Every block on the tensor cores (threshold 1): within REL_TOL of sum |a||b|."""
    from tests.test_gpu_ops import _big_cases

    rng = np.random.default_rng(700 + case)
    a, ia, b, ib, ca, cb = _big_cases(rng)[case]
    want = OB.contract(a, ia, b, ib, conja=ca, conjb=cb)
    scale = OB.contract(_abs(a), ia, _abs(b), ib, conja=ca, conjb=cb)  # conj only flips arrows
    mixed_ctx.set_mixed(1)
    got = to_host(D.contract(to_dev(a), ia, to_dev(b), ib, conja=ca, conjb=cb))
    assert sorted(got.blocks) == sorted(want.blocks)
    err = _rel_err(got, want, scale)
    assert err <= split_bound(_kmax(a, ia)), (err, split_bound(_kmax(a, ia)))
    assert err > 1e-12  # the tensor cores ran (FP64 agrees to ~1e-16 of the scale)


def test_mixed_threshold_keeps_small_blocks_fp64(D, mixed_ctx):
    """With threshold 64 only blocks of at least 64 x 64 move: the others are the FP64 path's bits."""
    rng = np.random.default_rng(9)
    M = rand_bt(rng, (-1, +1), ({0: 256, 2: 20, 4: 64}, {0: 17, 2: 100, 4: 512}), 1.0)
    N = rand_bt(rng, (-1, +1), ({0: 17, 2: 100, 4: 512}, {0: 64, 2: 33, 4: 256}), 1.0)
    plain = to_host(D.contract(to_dev(M), (1,), to_dev(N), (0,)))
    mixed_ctx.set_mixed(64)
    got = to_host(D.contract(to_dev(M), (1,), to_dev(N), (0,)))
    want = OB.contract(M, (1,), N, (0,))
    scale = OB.contract(_abs(M), (1,), _abs(N), (0,))
    for k in want.blocks:
        m, n = want.blocks[k].shape
        if m >= 64 and n >= 64:
            e = float(np.max(np.abs(got.blocks[k] - want.blocks[k]) / scale.blocks[k]))
            assert 1e-12 < e <= split_bound(512), (k, e)
        else:
            assert np.array_equal(got.blocks[k], plain.blocks[k]), k


def test_mixed_step_observable_error(mixed_ctx):
    """The benchmark quench (L = 64, delta = 0.5, maxdim 256, tol 1e-4) for 25 steps with EVERY
    contraction block on the tensor cores (threshold 1; at chi <= 10 no block reaches 8 x 8): the
    S^z error against the FP64 oracle stays at the FP32 level the split product gives."""
    from bondupdategalerkin_b200 import build
    from bondupdategalerkin_b200 import models as DM
    from bondupdategalerkin_b200 import native as DN
    from oracle import models as OM
    from oracle import step as OS
    from tests.gpu_util import mps_to_host

    build.build()
    L = 64
    ostate, dstate = OM.domain_wall_state(L), DM.domain_wall_state(L)
    ompo, dmpo = OM.xxz_mpo(L, J=1.0, delta=0.5), DM.xxz_mpo(L, J=1.0, delta=0.5)
    orng, drng = np.random.default_rng(1234), np.random.default_rng(1234)
    kw = dict(order=2, tol_basis=1e-4, maxdim=256)
    mixed_ctx.reset_stats()
    mixed_ctx.set_mixed(1)
    worst = 0.0
    for n in range(1, 26):
        OS.cbe_bug_step(ostate, ompo, -0.05j, rng=orng, **kw)
        DN.cbe_bug_step(dstate, dmpo, -0.05j, rng=drng, **kw)
        if n % 5 == 0:
            sz_o = OM.sz_profile(ostate)
            sz_d = OM.sz_profile(mps_to_host(dstate))
            worst = max(worst, float(np.max(np.abs(sz_d - sz_o))))
    assert mixed_ctx.kernel_stats()["mixed"]["launches"] > 0
    print(f"mixed step: worst |S^z error| over 25 steps = {worst:.2e}")
    assert worst <= 1e-5, worst
