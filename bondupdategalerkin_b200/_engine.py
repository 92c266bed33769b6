"""ctypes binding of ``libbug_b200.so`` (the C-ABI declared in ``include/bug_b200.h``).

The library is built in-tree (``bondupdategalerkin_b200/build.py``) and loaded from this package
directory. There is no fallback: if the library or a CUDA device is missing, ``context()`` raises.
"""

from __future__ import annotations

import ctypes
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libbug_b200.so")

_c_int_p = ctypes.POINTER(ctypes.c_int)
_c_double_p = ctypes.POINTER(ctypes.c_double)
_vp = ctypes.c_void_p

# name -> (restype, argtypes)
SIGNATURES = {
    "bug_last_error": (ctypes.c_char_p, []),
    "bug_version": (ctypes.c_char_p, []),
    "bug_ctx_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(_vp)]),
    "bug_ctx_destroy": (ctypes.c_int, [_vp]),
    "bug_ctx_synchronize": (ctypes.c_int, [_vp]),
    "bug_ctx_launches": (ctypes.c_int64, [_vp]),
    "bug_ctx_bytes_in_use": (ctypes.c_int64, [_vp]),
    "bug_ctx_stream": (_vp, [_vp]),
    "bug_ctx_set_profiling": (ctypes.c_int, [_vp, ctypes.c_int]),
    "bug_ctx_set_mixed": (ctypes.c_int, [_vp, ctypes.c_int]),
    "bug_batch_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp]),
    "bug_batch_context": (ctypes.c_int, [_vp, ctypes.c_int, _vp]),
    "bug_batch_launches": (ctypes.c_int64, [_vp]),
    "bug_batch_destroy": (ctypes.c_int, [_vp]),
    "bug_ctx_kernel_stats": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int64),
                                            _c_double_p, _c_double_p, _c_double_p]),
    "bug_ctx_reset_stats": (ctypes.c_int, [_vp]),
    "bug_ctx_host_stats": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_int64), _c_double_p,
                                          _c_double_p, _c_double_p]),
    "bug_tensor_create": (ctypes.c_int, [_vp, ctypes.c_int, _c_int_p, _c_int_p, _c_int_p, _c_int_p,
                                         ctypes.c_int, _c_int_p, ctypes.POINTER(_vp)]),
    "bug_tensor_upload": (ctypes.c_int, [_vp, _vp, _c_double_p, ctypes.c_int64]),
    "bug_tensor_download": (ctypes.c_int, [_vp, _vp, _c_double_p, ctypes.c_int64]),
    "bug_tensor_free": (ctypes.c_int, [_vp, _vp]),
    "bug_tensor_shape": (ctypes.c_int, [_vp, _c_int_p, _c_int_p, ctypes.POINTER(ctypes.c_int64), _c_int_p]),
    "bug_tensor_meta": (ctypes.c_int, [_vp, _c_int_p, _c_int_p, _c_int_p, _c_int_p, _c_int_p]),
    "bug_tensors_from_host": (ctypes.c_int, [_vp, ctypes.c_int, _c_int_p, ctypes.POINTER(ctypes.c_int64),
                                             _c_double_p, ctypes.POINTER(ctypes.c_int64),
                                             ctypes.POINTER(_vp)]),
    "bug_tensors_layout": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(_vp),
                                          ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64)]),
    "bug_tensors_to_host": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.POINTER(_vp), _c_int_p,
                                           ctypes.POINTER(ctypes.c_int64), _c_double_p,
                                           ctypes.POINTER(ctypes.c_int64)]),
    "bug_contract": (ctypes.c_int, [_vp, _vp, ctypes.c_int, _c_int_p, _vp, _c_int_p, ctypes.c_int,
                                    ctypes.c_int, ctypes.POINTER(_vp)]),
    "bug_svd": (ctypes.c_int, [_vp, _vp, ctypes.c_int, _c_int_p, ctypes.c_double, ctypes.c_int,
                               ctypes.POINTER(_vp), ctypes.POINTER(_vp), _c_double_p, _c_int_p,
                               ctypes.c_int, _c_int_p, _c_int_p]),
    "bug_thin_qr": (ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                   ctypes.POINTER(_vp)]),
    "bug_env_boundary": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.POINTER(_vp)]),
    "bug_env_step": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, _vp, ctypes.POINTER(_vp)]),
    "bug_apply_one_site": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, ctypes.POINTER(_vp)]),
    "bug_apply_zero_site": (ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.POINTER(_vp)]),
    "bug_sketch_stream": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                         ctypes.POINTER(_vp)]),
    "bug_perp": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, ctypes.POINTER(_vp)]),
    "bug_root_expv": (ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.c_double, ctypes.c_double,
                                     ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                     ctypes.POINTER(_vp), ctypes.POINTER(ctypes.c_int64),
                                     _c_double_p]),
    "bug_site_populations": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.POINTER(_vp), ctypes.c_int,
                                            _c_double_p, ctypes.c_int, _c_int_p]),
    "bug_observable_sz": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.POINTER(_vp), ctypes.c_int,
                                         _c_double_p]),
    "bug_apply_two_site": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, ctypes.POINTER(_vp)]),
    "bug_scale_leg": (ctypes.c_int, [_vp, _vp, ctypes.c_int, _c_double_p, ctypes.POINTER(_vp)]),
    "bug_norm2": (ctypes.c_int, [_vp, _vp, _c_double_p]),
    "bug_inner": (ctypes.c_int, [_vp, _vp, _vp, _c_double_p]),
    "bug_inner_many": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.POINTER(_vp), _vp, _c_double_p]),
    "bug_lincomb": (ctypes.c_int, [_vp, ctypes.c_int, _c_double_p, ctypes.POINTER(_vp), ctypes.POINTER(_vp)]),
    "bug_permute": (ctypes.c_int, [_vp, _vp, _c_int_p, ctypes.POINTER(_vp)]),
    "bug_conj": (ctypes.c_int, [_vp, _vp, ctypes.POINTER(_vp)]),
    "bug_flip_leg": (ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.POINTER(_vp)]),
    "bug_oplus": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.POINTER(_vp), ctypes.c_int, ctypes.POINTER(_vp)]),
    "bug_trim": (ctypes.c_int, [_vp, _vp, ctypes.c_int, _c_int_p, ctypes.POINTER(_vp)]),
    "bug_la_expm": (ctypes.c_int, [ctypes.c_int, _c_double_p, _c_double_p]),
    "bug_work_ceilings": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int64),
                                         ctypes.c_int64, ctypes.c_int64, ctypes.c_double,
                                         ctypes.c_int, ctypes.c_double,
                                         ctypes.POINTER(ctypes.c_int64)]),
    "bug_la_eigh": (ctypes.c_int, [ctypes.c_int, _c_double_p, _c_double_p, _c_double_p]),
    "bug_la_eigh_tridiag": (ctypes.c_int, [ctypes.c_int, _c_double_p, _c_double_p, _c_double_p,
                                           _c_double_p]),
    "bug_server_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int64, ctypes.POINTER(_vp)]),
    "bug_server_submit": (ctypes.c_int, [_vp, _vp, ctypes.POINTER(ctypes.c_int64)]),
    "bug_server_cancel": (ctypes.c_int, [_vp, ctypes.c_int64]),
    "bug_server_wait": (ctypes.c_int, [_vp, ctypes.c_int64, ctypes.c_double, _c_int_p]),
    "bug_server_job_stats": (ctypes.c_int, [_vp, ctypes.c_int64, _vp]),
    "bug_server_step_times": (ctypes.c_int, [_vp, ctypes.c_int64, _c_double_p, ctypes.c_int, _c_int_p]),
    "bug_server_destroy": (ctypes.c_int, [_vp]),
    "bug_server_launches": (ctypes.c_int64, [_vp]),
    "bug_server_job_error": (ctypes.c_int, [_vp, ctypes.c_int64, ctypes.c_char_p, ctypes.c_int]),
    "bug_projected_footprint": (ctypes.c_int64, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "bug_la_kry_weight": (ctypes.c_int, [ctypes.c_int, _c_double_p, ctypes.c_int, ctypes.c_double,
                                         ctypes.c_double, ctypes.c_int, _c_double_p]),
    "bug_la_eigvals_hess": (ctypes.c_int, [ctypes.c_int, _c_double_p, _c_double_p]),
    "bug_inner_noalloc": (ctypes.c_int, [_vp, _vp, ctypes.c_int64, _vp, _vp]),
}
# declared in native.py (structure arguments)
NATIVE_ONLY = ("bug_mps_step", "bug_tdvp2_step", "bug_step_batch")  # bound in native.py with their structs

FAMILIES = ("copy", "gemm", "svd", "dot", "lincomb", "scale", "mixed")
# Where each family runs: the SVD (and the pivoted QR) is its own kernel; every other family is a
# stage kind of stage_kernel, one launch per operation.
KERNEL_NAMES = {"copy": "stage_kernel (copy stage)", "gemm": "stage_kernel (gemm stage)",
                "svd": "jacobi_svd_kernel", "dot": "stage_kernel (dot stages)",
                "lincomb": "stage_kernel (lincomb stage)", "scale": "stage_kernel (scale stage)",
                "mixed": "tc_pack_kernel + tc_cgemm_kernel (3xTF32 tcgen05)"}

STATUS = {0: "BUG_OK", 1: "BUG_EINVAL", 2: "BUG_ENONFINITE", 3: "BUG_ENOMEM", 4: "BUG_ETIMEOUT",
          5: "BUG_EDEVICE", 6: "BUG_ENOTCONV"}


class EngineError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


# The status codes as the exceptions a caller of the reference catches: an ArgumentError or
# DimensionMismatch is a ValueError here, a non-finite or unconverged computation an
# ArithmeticError, an allocation failure a MemoryError. Each is still an EngineError.
class EngineArgumentError(EngineError, ValueError):
    """BUG_EINVAL: a bad argument, shape or arrow."""


class EngineNonFiniteError(EngineError, ArithmeticError):
    """BUG_ENONFINITE: non-finite data where the reference throws."""


class EngineMemoryError(EngineError, MemoryError):
    """BUG_ENOMEM: a device or host allocation failed."""


class EngineConvergenceError(EngineError, ArithmeticError):
    """BUG_ENOTCONV: an iterative kernel hit its iteration bound."""


_ERRORS = {1: EngineArgumentError, 2: EngineNonFiniteError, 3: EngineMemoryError,
           6: EngineConvergenceError}


_lib = None
_lock = threading.Lock()


def load(path: str = LIB_PATH) -> ctypes.CDLL:
    """Load the engine library and declare every exported signature. Raises if it is missing."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(path):
            raise FileNotFoundError(
                f"{path} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'`"
            )
        lib = ctypes.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def check(code: int) -> None:
    if code != 0:
        raise _ERRORS.get(code, EngineError)(code, load().bug_last_error().decode(errors="replace"))


class Context:
    """One engine context (device + stream + memory pool)."""

    def __init__(self, device: int = 0):
        lib = load()
        h = _vp()
        check(lib.bug_ctx_create(device, ctypes.byref(h)))
        self.h = h
        self.lib = lib
        self.device = device

    @classmethod
    def borrow(cls, h, device: int = 0, owner=None) -> "Context":
        """A context owned elsewhere (a batch's): usable for tensors, never destroyed here. It keeps
        `owner` alive, so tensors on it (which hold their context) outlive the owner's teardown."""
        c = cls.__new__(cls)
        c.h = h
        c.lib = load()
        c.device = device
        c._owner = owner
        return c

    def synchronize(self):
        check(self.lib.bug_ctx_synchronize(self.h))

    def launches(self) -> int:
        return int(self.lib.bug_ctx_launches(self.h))

    def bytes_in_use(self) -> int:
        return int(self.lib.bug_ctx_bytes_in_use(self.h))

    def stream(self) -> int:
        """The context's ``cudaStream_t`` as an integer (for ``torch.cuda.ExternalStream``)."""
        return int(self.lib.bug_ctx_stream(self.h) or 0)

    def set_profiling(self, on: bool) -> None:
        check(self.lib.bug_ctx_set_profiling(self.h, int(on)))

    def set_mixed(self, min_dim: int) -> None:
        """Tensor-core 3xTF32 contractions for output blocks with both extents >= min_dim (0: off)."""
        check(self.lib.bug_ctx_set_mixed(self.h, int(min_dim)))

    def reset_stats(self) -> None:
        check(self.lib.bug_ctx_reset_stats(self.h))

    def host_stats(self) -> dict:
        """Host accounting since the last reset: read-back waits (count, seconds), seconds inside
        kernel-launch calls and inside the stream-ordered allocator."""
        n, w, la, al = ctypes.c_int64(), ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        check(self.lib.bug_ctx_host_stats(self.h, ctypes.byref(n), ctypes.byref(w), ctypes.byref(la),
                                          ctypes.byref(al)))
        return dict(syncs=int(n.value), wait_s=w.value, launch_s=la.value, alloc_s=al.value)

    def kernel_stats(self) -> dict:
        """Per kernel family: launches, algorithmic flops and bytes, device ms (profiling only)."""
        out = {}
        for fam, name in enumerate(FAMILIES):
            n = ctypes.c_int64()
            f, b, ms = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
            check(self.lib.bug_ctx_kernel_stats(self.h, fam, ctypes.byref(n), ctypes.byref(f),
                                                ctypes.byref(b), ctypes.byref(ms)))
            out[name] = dict(launches=int(n.value), flops=f.value, bytes=b.value, ms=ms.value)
        return out


_ctx = {}
_default_device = [0]


def set_default_device(device: int) -> None:
    """Device used by ``context()`` when none is given (one process per GPU sets its own)."""
    _default_device[0] = int(device)


def context(device: int | None = None) -> Context:
    """The process-wide context of ``device`` (created on first use)."""
    device = _default_device[0] if device is None else device
    c = _ctx.get(device)
    if c is None:
        c = Context(device)
        _ctx[device] = c
    return c
