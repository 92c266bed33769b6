"""The C-ABI library builds for sm_100a, loads without a GPU, and exports every function that
``include/bug_b200.h`` declares (no compute calls: this runs on CPU)."""

import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    src = open(os.path.join(ROOT, "include", "bug_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(bug_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    from bondupdategalerkin_b200 import build

    path = build.build()
    lib = ctypes.CDLL(path)
    names = declared()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_the_header():
    from bondupdategalerkin_b200 import _engine

    assert set(declared()) == set(_engine.SIGNATURES) | set(_engine.NATIVE_ONLY)
    lib = _engine.load()
    assert lib.bug_version().decode().startswith("bug_b200")


def test_noalloc_inner_refuses_misaligned_pointers():
    """The allocation-free inner product moves whole complex doubles, so a pointer that is 8- but
    not 16-byte aligned is refused with BUG_EINVAL before any device work (runs without a GPU)."""
    from bondupdategalerkin_b200 import _engine

    lib = _engine.load()

    def call(a, b, n, out):
        return lib.bug_inner_noalloc(ctypes.c_void_p(a), ctypes.c_void_p(b), ctypes.c_int64(n),
                                     ctypes.c_void_p(out), ctypes.c_void_p(0))

    for a, b, out in ((4104, 4096, 4096), (4096, 4104, 4096), (4096, 4096, 4104)):
        assert call(a, b, 10, out) == 1
        assert "16-byte aligned" in lib.bug_last_error().decode()
    assert call(0, 0, 0, 4104) == 1  # n == 0 still writes out


def test_context_creation_fails_loudly_without_a_device():
    import pytest
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    from bondupdategalerkin_b200 import _engine

    with pytest.raises(_engine.EngineError):
        _engine.Context(0)


def test_small_matrix_routines_match_scipy():
    """The host-side k x k routines the native step uses, against scipy (CPU only)."""
    import numpy as np
    import scipy.linalg

    from bondupdategalerkin_b200 import _engine

    lib = _engine.load()
    rng = np.random.default_rng(0)
    for n, scale in ((1, 1.0), (5, 0.3), (12, 3.0), (30, 20.0)):
        A = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) * scale / np.sqrt(n)
        a = np.ascontiguousarray(A).view(np.float64)
        out = np.zeros(2 * n * n)
        _engine.check(lib.bug_la_expm(n, a.ctypes.data_as(_engine._c_double_p),
                                      out.ctypes.data_as(_engine._c_double_p)))
        want = scipy.linalg.expm(A)
        got = out.view(np.complex128).reshape(n, n)
        assert np.max(np.abs(got - want)) <= 1e-12 * max(1.0, np.max(np.abs(want)))
        S = rng.standard_normal((n, n))
        S = S + S.T
        vals = np.zeros(n)
        vecs = np.zeros(n * n)
        _engine.check(lib.bug_la_eigh(n, np.ascontiguousarray(S).ctypes.data_as(_engine._c_double_p),
                                      vals.ctypes.data_as(_engine._c_double_p),
                                      vecs.ctypes.data_as(_engine._c_double_p)))
        assert np.allclose(vals, np.linalg.eigvalsh(S), atol=1e-12 * max(1, np.max(np.abs(S))))
        V = vecs.reshape(n, n)
        assert np.allclose(V @ np.diag(vals) @ V.T, S, atol=1e-11 * max(1, np.max(np.abs(S))))
        Hs = np.triu(A, -1)
        h = np.ascontiguousarray(Hs).view(np.float64)
        ev = np.zeros(2 * n)
        _engine.check(lib.bug_la_eigvals_hess(n, h.ctypes.data_as(_engine._c_double_p),
                                              ev.ctypes.data_as(_engine._c_double_p)))
        got = np.sort_complex(ev.view(np.complex128))
        want = np.sort_complex(np.linalg.eigvals(Hs))
        assert np.max(np.abs(got - want)) <= 1e-9 * max(1.0, np.max(np.abs(want)))


def test_krylov_weight_matches_oracle():
    """The native Krylov weight (nodes evaluated in blocks) against the oracle's node-by-node
    evaluation, on Hessenberg matrices from mild to stiff (the 2 x 4096-panel cap reached)."""
    import numpy as np

    from bondupdategalerkin_b200 import _engine, build
    from oracle import krylov as OK

    build.build()
    lib = _engine.load()
    rng = np.random.default_rng(11)
    for n, scale, tau, herm in [(6, 1.0, -0.05j, True), (20, 50.0, -0.05j, True),
                                (33, 1e4, 0.02, False), (64, 3e5, 0.02, False)]:
        A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
        if herm:
            A = A + A.conj().T
        H = np.ascontiguousarray(np.triu(A, -1) * scale / n)
        h = H.view(np.float64)
        for k in (1, n // 2, n - 1):
            for seed in (True, False):
                out = np.zeros(1)
                _engine.check(lib.bug_la_kry_weight(n, h.ctypes.data_as(_engine._c_double_p), k,
                                                    tau.real, tau.imag, int(seed),
                                                    out.ctypes.data_as(_engine._c_double_p)))
                want = OK.kry_weight(H, k, tau, state_seed=seed)
                assert abs(out[0] - want) <= 1e-9 * max(abs(want), 1e-300), (n, k, seed, out[0], want)


def test_tridiagonal_eigensolver_matches_lapack():
    """The Lanczos tridiagonal's eigen-decomposition (implicit QR with Wilkinson shifts) against
    LAPACK through numpy: eigenvalues to 1e-13 of the norm, eigenvectors orthonormal and
    reconstructing T, on random, graded, Lanczos-like (decaying off-diagonals, one exactly zero)
    and degenerate tridiagonals of size 1 to 64."""
    import numpy as np

    from bondupdategalerkin_b200 import _engine, build

    build.build()
    lib = _engine.load()
    rng = np.random.default_rng(21)
    cases = []
    for n in (1, 2, 3, 7, 30, 64):
        cases.append((rng.standard_normal(n), rng.standard_normal(max(n - 1, 0))))
        cases.append((rng.standard_normal(n) * 1e3, np.geomspace(1.0, 1e-14, max(n - 1, 0))))
    d = rng.standard_normal(12)
    e = rng.standard_normal(11)
    e[5] = 0.0
    cases.append((d, e))
    cases.append((np.ones(10), np.zeros(9)))                 # fully degenerate, already diagonal
    cases.append((np.zeros(8), np.ones(7)))                  # symmetric spectrum, zero diagonal
    for d, e in cases:
        n = len(d)
        T = np.diag(d) + np.diag(e, 1) + np.diag(e, -1)
        vals = np.zeros(n)
        vecs = np.zeros((n, n))
        dp, ep = np.ascontiguousarray(d, float), np.ascontiguousarray(e if n > 1 else np.zeros(1), float)
        _engine.check(lib.bug_la_eigh_tridiag(n, dp.ctypes.data_as(_engine._c_double_p),
                                              ep.ctypes.data_as(_engine._c_double_p),
                                              vals.ctypes.data_as(_engine._c_double_p),
                                              vecs.ctypes.data_as(_engine._c_double_p)))
        scale = max(np.abs(T).max(), 1e-300)
        want = np.linalg.eigvalsh(T)
        assert np.all(np.diff(vals) >= 0)
        assert np.max(np.abs(vals - want)) <= 1e-13 * scale, (n, np.max(np.abs(vals - want)))
        assert np.max(np.abs(vecs.T @ vecs - np.eye(n))) <= 1e-13
        assert np.max(np.abs(vecs @ np.diag(vals) @ vecs.T - T)) <= 1e-13 * scale


def _tridiag(lib, d, e):
    import numpy as np

    from bondupdategalerkin_b200 import _engine

    n = len(d)
    vals, vecs = np.zeros(n), np.zeros((n, n))
    dp = np.ascontiguousarray(d, float)
    ep = np.ascontiguousarray(e if n > 1 else [0.0], float)
    code = lib.bug_la_eigh_tridiag(n, dp.ctypes.data_as(_engine._c_double_p),
                                   ep.ctypes.data_as(_engine._c_double_p),
                                   vals.ctypes.data_as(_engine._c_double_p),
                                   vecs.ctypes.data_as(_engine._c_double_p))
    return code, vals, vecs


def test_tridiagonal_eigensolver_reference_case_and_non_finite_input():
    """The reference's own case for ``_tridiag_eigen`` (``test_krylov_weights.jl:105-116``): exact
    to 1e-12 on finite input; NaN or Inf is named (BUG_ENONFINITE, the entries counted) instead of
    surfacing as a convergence failure."""
    import numpy as np

    from bondupdategalerkin_b200 import _engine, build

    build.build()
    lib = _engine.load()
    d, e = [0.3, -1.2, 2.5, 0.0, 1e-9], [1.0, 1e-12, 0.7, 2.0]
    code, vals, vecs = _tridiag(lib, d, e)
    assert code == 0
    T = np.diag(d) + np.diag(e, 1) + np.diag(e, -1)
    assert np.linalg.norm(T @ vecs - vecs @ np.diag(vals)) < 1e-12
    assert np.linalg.norm(vecs.T @ vecs - np.eye(5)) < 1e-12
    enonfinite = [k for k, v in _engine.STATUS.items() if v == "BUG_ENONFINITE"][0]
    for d, e, counts in (([0.0, np.nan], [1.0], "1 of 2 alpha, 0 of 1 beta"),
                         ([0.0, 1.0], [np.inf], "0 of 2 alpha, 1 of 1 beta")):
        code, _, _ = _tridiag(lib, d, e)
        assert code == enonfinite
        msg = lib.bug_last_error().decode()
        assert "non-finite" in msg and counts in msg, msg


def test_krylov_weight_two_by_two_known_answer():
    """The native weight on the reference's 2 x 2 (``test_krylov_weights.jl:44-56``): H_1 = [2 pi],
    beta = 1, tau = -i gives |tau| beta int_0^1 |exp(-2 pi i s)| ds = 1."""
    import numpy as np

    from bondupdategalerkin_b200 import _engine, build

    build.build()
    lib = _engine.load()
    H = np.ascontiguousarray([[2 * np.pi, 0.0], [1.0, 0.0]], dtype=np.complex128)
    out = np.zeros(1)
    _engine.check(lib.bug_la_kry_weight(2, H.view(np.float64).ctypes.data_as(_engine._c_double_p),
                                        1, 0.0, -1.0, 1, out.ctypes.data_as(_engine._c_double_p)))
    assert abs(out[0] - 1.0) <= 1e-10


def test_projected_footprint_is_the_documented_bound():
    """The job server's admission size (``bug_projected_footprint``, host arithmetic: no device):
    state, two environment stacks, one bond's Krylov basis and probes (64 + 16 vectors) and the
    two-site work tensors at bond dimension maxdim, in complex FP64, doubled for temporaries; zero
    for a degenerate chain; monotone in every argument."""
    import ctypes

    from bondupdategalerkin_b200 import _engine

    lib = _engine.load()
    f = lib.bug_projected_footprint
    f.restype, f.argtypes = ctypes.c_int64, [ctypes.c_int] * 4
    for L, d, D, w in ((64, 2, 256, 5), (20, 2, 64, 12), (8, 4, 32, 3)):
        D2 = D * D
        want = 2 * 16 * (L * d * D2 + 2 * L * w * D2 + 80 * d * D2 + 4 * d * d * D2)
        assert f(L, d, D, w) == want
        assert f(L + 1, d, D, w) > want and f(L, d, D + 1, w) > want and f(L, d, D, w + 1) > want
    assert f(0, 2, 64, 5) == 0 and f(8, 2, 0, 5) == 0
    assert f(64, 2, 256, 5) < 2 ** 31  # the headline chain at maxdim 256: ~1.8 GiB of 180 GB


def test_status_codes_raise_the_reference_exception_kinds():
    """A refused argument raises a ValueError (the reference's ArgumentError), non-finite data an
    ArithmeticError, each still an EngineError carrying its status code."""
    import numpy as np
    import pytest

    from bondupdategalerkin_b200 import _engine

    lib = _engine.load()
    v = np.zeros(4)
    p = v.ctypes.data_as(_engine._c_double_p)
    with pytest.raises(ValueError) as e:
        _engine.check(lib.bug_la_eigh_tridiag(-1, p, p, p, p))
    assert isinstance(e.value, _engine.EngineError) and e.value.code == 1
    d = np.array([0.0, np.nan])
    with pytest.raises(ArithmeticError) as e:
        _engine.check(lib.bug_la_eigh_tridiag(2, d.ctypes.data_as(_engine._c_double_p), p, p, p))
    assert isinstance(e.value, _engine.EngineError) and e.value.code == 2


def test_smoke_fails_loudly_without_a_device():
    """No CPU fallback: the smoke check of the device path raises where there is no GPU."""
    import pytest
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    import sys

    sys.path.insert(0, ROOT)
    import __graft_entry__ as g

    with pytest.raises(Exception):
        g.smoke()
