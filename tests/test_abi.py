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

    assert set(declared()) == set(_engine.SIGNATURES)
    lib = _engine.load()
    assert lib.bug_version().decode().startswith("bug_b200")


def test_context_creation_fails_loudly_without_a_device():
    import pytest
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    from bondupdategalerkin_b200 import _engine

    with pytest.raises(_engine.EngineError):
        _engine.Context(0)
