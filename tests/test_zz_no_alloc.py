"""The allocation-free inner product against the engine's ordinary one (GPU).

``bug_inner_noalloc`` is for callers that cannot allocate device memory where they call it (a
fixed memory budget, a callback or hook that forbids cudaMalloc, code that must not create an
engine context): its reduction scratch is a static device array in the library. This checks,
through the C-ABI, that two calls in a row each agree with ``bug_inner`` (the entry point that
allocates its scratch from the engine's pool) to the tolerance of the other engine tests; that the
empty vector, the largest accepted length and a non-default stream work; that a length over the
stated limit is refused; and that the calls leave the device's free memory unchanged. The file
sorts last so that a run stopping at its first failure has already run every other test.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LIMIT = 8_388_608


def _call(lib, a_ptr, b_ptr, n, out_ptr, stream=0):
    return lib.bug_inner_noalloc(ctypes.c_void_p(a_ptr), ctypes.c_void_p(b_ptr), ctypes.c_int64(n),
                                 ctypes.c_void_p(out_ptr), ctypes.c_void_p(stream))


@pytest.fixture(scope="module")
def lib():
    from bondupdategalerkin_b200 import _engine as E
    from bondupdategalerkin_b200 import build

    build.build()
    return E.load()


def _engine_inner(x, y):
    from bondupdategalerkin_b200 import tensor as T

    leg = T.Leg(-1, {0: len(x)})
    return T.inner(T.from_blocks([leg], {(0,): x}), T.from_blocks([leg], {(0,): y}))


def _check(got, ref, x, y):
    n = len(x)
    assert abs(got - ref) <= 1e-12 * max(1.0, abs(ref)) * np.sqrt(n), (n, got, ref)
    assert abs(got - np.vdot(x, y)) <= 1e-10 * np.linalg.norm(x) * np.linalg.norm(y)


def test_noalloc_inner_matches_bug_inner_twice(lib):
    import torch

    from bondupdategalerkin_b200 import _engine as E

    rng = np.random.default_rng(2024)
    for n in (1_000_003, 70_000):  # two calls in a row, different sizes
        x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        y = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        ref = _engine_inner(x, y)
        a = torch.from_numpy(x).to("cuda")
        b = torch.from_numpy(y).to("cuda")
        out = torch.zeros(1, dtype=torch.complex128, device="cuda")
        torch.cuda.synchronize()
        E.check(_call(lib, a.data_ptr(), b.data_ptr(), n, out.data_ptr()))
        torch.cuda.synchronize()
        _check(complex(out.cpu().numpy()[0]), ref, x, y)


def test_noalloc_inner_edges_and_side_stream(lib):
    """n = 0 writes an exact zero; n at the limit fills every partial-sum slot of the scratch; a
    call on a torch side stream is ordered on that stream."""
    import torch

    from bondupdategalerkin_b200 import _engine as E

    out = torch.full((1,), 7.0 + 7.0j, dtype=torch.complex128, device="cuda")
    torch.cuda.synchronize()
    E.check(_call(lib, 0, 0, 0, out.data_ptr()))
    torch.cuda.synchronize()
    assert complex(out.cpu().numpy()[0]) == 0j

    rng = np.random.default_rng(7)
    x = rng.standard_normal(LIMIT) + 1j * rng.standard_normal(LIMIT)
    y = rng.standard_normal(LIMIT) + 1j * rng.standard_normal(LIMIT)
    ref = _engine_inner(x, y)
    a = torch.from_numpy(x).to("cuda")
    b = torch.from_numpy(y).to("cuda")
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        out2 = torch.zeros(1, dtype=torch.complex128, device="cuda")
        E.check(_call(lib, a.data_ptr(), b.data_ptr(), LIMIT, out2.data_ptr(), side.cuda_stream))
        host = out2.to("cpu", non_blocking=False)
    side.synchronize()
    _check(complex(host.numpy()[0]), ref, x, y)


def test_noalloc_inner_allocates_nothing(lib):
    """Once the first call on the device has looked up the scratch address (and loaded the
    kernels), further calls change neither torch's allocation count nor the device's free bytes."""
    import torch

    from bondupdategalerkin_b200 import _engine as E

    n = 300_001
    rng = np.random.default_rng(11)
    a = torch.from_numpy(rng.standard_normal(n) + 1j * rng.standard_normal(n)).to("cuda")
    b = torch.from_numpy(rng.standard_normal(n) + 1j * rng.standard_normal(n)).to("cuda")
    out = torch.zeros(1, dtype=torch.complex128, device="cuda")
    E.check(_call(lib, a.data_ptr(), b.data_ptr(), n, out.data_ptr()))
    E.check(_call(lib, 0, 0, 0, out.data_ptr()))
    torch.cuda.synchronize()
    alloc0 = torch.cuda.memory_allocated()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(2):
        E.check(_call(lib, a.data_ptr(), b.data_ptr(), n, out.data_ptr()))
        E.check(_call(lib, 0, 0, 0, out.data_ptr()))
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert torch.cuda.memory_allocated() == alloc0
    assert free1 == free0, (free0, free1)


def test_noalloc_inner_rejects_oversize(lib):
    code = _call(lib, 16, 16, LIMIT + 1, 16)  # refused before any device work
    assert code == 1
    assert "exceeds the no-alloc limit" in lib.bug_last_error().decode()
