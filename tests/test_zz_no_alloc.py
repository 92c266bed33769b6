"""The allocation-free inner product against the engine's ordinary one (GPU).

``bug_inner_noalloc`` is for callers that cannot allocate device memory where they call it (a
fixed memory budget, a callback or hook that forbids cudaMalloc, code that must not create an
engine context): its reduction scratch is a static device array in the library. This checks,
through the C-ABI, that two calls in a row each agree with ``bug_inner`` (the entry point that
allocates its scratch from the engine's pool) to the tolerance of the other engine tests, and that a
length over the stated limit is refused. The file sorts last so that a run stopping at its first
failure has already run every other test.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LIMIT = 8_388_608


def _call(lib, a_ptr, b_ptr, n, out_ptr):
    return lib.bug_inner_noalloc(ctypes.c_void_p(a_ptr), ctypes.c_void_p(b_ptr), ctypes.c_int64(n),
                                 ctypes.c_void_p(out_ptr), ctypes.c_void_p(0))


def test_noalloc_inner_matches_bug_inner_twice():
    import torch

    from bondupdategalerkin_b200 import _engine as E
    from bondupdategalerkin_b200 import build
    from bondupdategalerkin_b200 import tensor as T

    build.build()
    lib = E.load()
    rng = np.random.default_rng(2024)
    for n in (1_000_003, 70_000):  # two calls in a row, different sizes
        x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        y = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        leg = T.Leg(-1, {0: n})
        ref = T.inner(T.from_blocks([leg], {(0,): x}), T.from_blocks([leg], {(0,): y}))
        a = torch.from_numpy(x).to("cuda")
        b = torch.from_numpy(y).to("cuda")
        out = torch.zeros(1, dtype=torch.complex128, device="cuda")
        torch.cuda.synchronize()
        E.check(_call(lib, a.data_ptr(), b.data_ptr(), n, out.data_ptr()))
        torch.cuda.synchronize()
        got = complex(out.cpu().numpy()[0])
        assert abs(got - ref) <= 1e-12 * max(1.0, abs(ref)) * np.sqrt(n), (n, got, ref)
        assert abs(got - np.vdot(x, y)) <= 1e-10 * np.linalg.norm(x) * np.linalg.norm(y)


def test_noalloc_inner_rejects_oversize():
    from bondupdategalerkin_b200 import _engine as E
    from bondupdategalerkin_b200 import build

    build.build()
    lib = E.load()
    code = _call(lib, 16, 16, LIMIT + 1, 16)  # refused before any device work
    assert code == 1
    assert "exceeds the no-alloc limit" in lib.bug_last_error().decode()
