"""The native step: ``cbe_bug_step`` as ONE call into ``libbug_b200.so`` (``bug_mps_step``).

The sweep logic, ledger and every tensor operation run inside the library; Python only passes
handles, the keyword arguments and a callback through which the library draws the Gaussian probes
from the caller's seeded ``numpy.random.Generator`` (the same draw stream, in the same order, as
the Python host in ``step.py`` and the CPU oracle).
"""

from __future__ import annotations

import ctypes
from types import SimpleNamespace

import numpy as np

from . import _engine as E
from .options import check_step_options, resolve_krylov_recurrence
from .tensor import DT

MAX_SITES = 1024
UNMET_NAMES = {1: "sample", 2: "tail", 3: "krylov", 4: "trunc", 5: "projection", 6: "expv", 7: "closure"}


RNG_CTL_FN = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_int)
DRAW_FN = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_int64, ctypes.POINTER(ctypes.c_double))
RNG_FORK_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(DRAW_FN),
                               ctypes.POINTER(ctypes.c_void_p))


def fork_rng(rng):
    """The right half's own stream under ``parallel = true`` (``rngR = MersenneTwister(rand(rng,
    UInt64))``, ``bug_step.jl:225``, ``frontier_closure.jl:125``): a generator seeded by ONE draw
    of ``rng`` over the full unsigned 64-bit range."""
    seed = int(rng.integers(0, np.iinfo(np.uint64).max, dtype=np.uint64, endpoint=True))
    return np.random.default_rng(seed)


class StepParams(ctypes.Structure):
    _fields_ = [("tol_basis", ctypes.c_double), ("tol_trunc", ctypes.c_double),
                ("tol_expv", ctypes.c_double), ("tol_krylov", ctypes.c_double),
                ("order", ctypes.c_int), ("maxdim", ctypes.c_int), ("hermitian", ctypes.c_int),
                ("work_ceiling_rule", ctypes.c_int), ("bond_ceiling_factor", ctypes.c_double),
                ("root", ctypes.c_int), ("reorth", ctypes.c_int), ("truncate", ctypes.c_int),
                ("root_maxiter", ctypes.c_int), ("fixed_width", ctypes.c_int),
                ("tail_factor", ctypes.c_double), ("krylov_mode", ctypes.c_int),
                ("krylov_fixed_depth", ctypes.c_int), ("dd_mode", ctypes.c_int),
                ("holdout_width", ctypes.c_int), ("batch_blocks", ctypes.c_int),
                ("cap_selection", ctypes.c_int), ("acceptance_factor", ctypes.c_double),
                ("eshift", ctypes.c_double), ("root_report", ctypes.c_int),
                ("outside_residual", ctypes.c_int), ("rng_ctl", RNG_CTL_FN),
                ("rng_ctl_user", ctypes.c_void_p), ("closure_checks", ctypes.c_int),
                ("root_method", ctypes.c_int), ("root_noshift", ctypes.c_int),
                ("parallel", ctypes.c_int), ("rng_fork", RNG_FORK_FN),
                ("rng_fork_user", ctypes.c_void_p), ("exact", ctypes.c_int),
                ("fold_omega", ctypes.c_int), ("n_keep", ctypes.c_int),
                ("keep_sites", ctypes.POINTER(ctypes.c_void_p)),
                ("keep_tols", ctypes.POINTER(ctypes.c_double)), ("frames_only", ctypes.c_int),
                ("root_ceiling_factor", ctypes.c_double),
                ("frames_out", ctypes.POINTER(ctypes.c_void_p))]


class BondLog(ctypes.Structure):
    _fields_ = [("bond", ctypes.c_int), ("side", ctypes.c_int), ("sample", ctypes.c_double),
                ("tail", ctypes.c_double), ("krylov_c", ctypes.c_double), ("krylov_d", ctypes.c_double),
                ("n_probes", ctypes.c_int64), ("n_selected", ctypes.c_int64),
                ("n_krylov", ctypes.c_int64), ("n_h1", ctypes.c_int64), ("c_pass", ctypes.c_int),
                ("d_after_c", ctypes.c_int), ("workcap", ctypes.c_int), ("met", ctypes.c_int),
                ("unmet_mask", ctypes.c_int), ("width", ctypes.c_int), ("r_old", ctypes.c_int),
                ("r_final", ctypes.c_int), ("discarded", ctypes.c_double)]


class StepInfo(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("unmet_mask", ctypes.c_int),
                ("unmet_order", ctypes.c_int * 8), ("root_link", ctypes.c_int),
                ("root_rank", ctypes.c_int), ("root_frame_width", ctypes.c_int),
                ("discarded", ctypes.c_double), ("n_matvec", ctypes.c_int64),
                ("max_sample", ctypes.c_double), ("max_tail", ctypes.c_double),
                ("max_krylov", ctypes.c_double), ("max_krylov_c", ctypes.c_double),
                ("max_krylov_d", ctypes.c_double), ("ledger_discarded", ctypes.c_double),
                ("expv_err", ctypes.c_double), ("expv_iters", ctypes.c_int64),
                ("n_probes", ctypes.c_int64), ("n_selected", ctypes.c_int64),
                ("n_krylov", ctypes.c_int64), ("n_h1", ctypes.c_int64), ("n_c_pass", ctypes.c_int64),
                ("n_d_after_c", ctypes.c_int64), ("workcap_reached", ctypes.c_int),
                ("maxdim_reached", ctypes.c_int), ("proj_err", ctypes.c_double),
                ("r_old", ctypes.c_int64), ("r_aug", ctypes.c_int64), ("r_final", ctypes.c_int64),
                ("n_passes", ctypes.c_int64), ("n_closure_sweeps", ctypes.c_int64),
                ("defect", ctypes.c_double), ("n_root_frontier", ctypes.c_int64),
                ("n_h1_closure", ctypes.c_int64), ("n_compress", ctypes.c_int64),
                ("leak1", ctypes.c_double), ("expanded", ctypes.c_int * MAX_SITES),
                ("n_new", ctypes.c_int * MAX_SITES), ("workcap", ctypes.c_int * MAX_SITES),
                ("n_holdout", ctypes.c_int64), ("n_targeted", ctypes.c_int64),
                ("e_pre", ctypes.c_double), ("e_root", ctypes.c_double), ("resid", ctypes.c_double),
                ("resid_initial", ctypes.c_double), ("outside", ctypes.c_double),
                ("outside_left", ctypes.c_double), ("outside_right", ctypes.c_double),
                ("outside_passes", ctypes.c_int), ("outside_added", ctypes.c_int),
                ("n_h2_leak", ctypes.c_int64)]



_declared = [False]


def _lib():
    lib = E.load()
    if not _declared[0]:
        lib.bug_step_batch.restype = ctypes.c_int
        lib.bug_step_batch.argtypes = [
            ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.c_void_p,
            ctypes.POINTER(ctypes.c_int), ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
            ctypes.POINTER(ctypes.c_double), ctypes.POINTER(StepParams), DRAW_FN, ctypes.c_void_p,
            ctypes.POINTER(StepInfo), ctypes.POINTER(ctypes.c_int)]
        lib.bug_mps_step.restype = ctypes.c_int
        lib.bug_mps_step.argtypes = [
            ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_int),
            ctypes.POINTER(ctypes.c_void_p), ctypes.c_double, ctypes.c_double,
            ctypes.POINTER(StepParams), DRAW_FN, ctypes.c_void_p, ctypes.POINTER(StepInfo),
            ctypes.POINTER(BondLog), ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
        _declared[0] = True
    return lib


def step_params(L, *, tol_basis=None, tol_trunc=None, tol_expv=None, tol_krylov=None, order=1,
                maxdim=None, hermitian=True, expansion=None, root=None, reorth=True, truncate=True,
                work_ceiling_rule="bond", bond_ceiling_factor=None, root_ceiling_factor=1.2,
                root_maxiter=30, krylov_rank_tol=0.0, frontier_tol=0.0, fold_omega=None,
                closure_checks=False, exact=False):
    """The keyword arguments of ``cbe_bug_step!`` as the C-ABI's ``bug_step_params`` (checked the
    way the reference checks them, ``bug_step_stages.jl:15-142``)."""
    if L < 2:
        raise ValueError("cbe_bug_step needs at least two sites")
    if L - 1 > MAX_SITES:
        raise ValueError(f"at most {MAX_SITES + 1} sites")
    rules = {"bond": 0, "maxdim": 1, "bond_strict": 2, "frame_root": 3}
    if work_ceiling_rule not in rules:
        raise ValueError(f"work_ceiling_rule {work_ceiling_rule!r}")
    if frontier_tol or krylov_rank_tol:
        raise NotImplementedError("frontier_tol / krylov_rank_tol > 0")
    mode, width, tail_factor, kmode, fixed_depth = "rank_tail", 8, 0.10, "auto", 0
    holdout, batch, capsel, accept = 4, 1, "storage", 1.0
    if expansion is not None:
        mode, width = expansion.mode, expansion.fixed_width
        tail_factor, kmode = expansion.tail_factor, expansion.krylov_mode
        fixed_depth = expansion.krylov_fixed_depth
        holdout = getattr(expansion, "holdout_width", 4)
        batch = getattr(expansion, "batch_blocks", 1)
        capsel = getattr(expansion, "cap_selection", "storage")
        accept = getattr(expansion, "acceptance_factor", 1.0)
    if not 1 <= batch <= 8:
        raise ValueError("batch_blocks must lie in 1:8")
    if capsel not in ("storage", "svd"):
        raise ValueError("cap_selection must be :storage or :svd")
    if not 0 < accept <= 1:
        raise ValueError("acceptance_factor must lie in (0,1]")
    if holdout < 1:
        raise ValueError("holdout_width must be positive")
    resolve_krylov_recurrence(kmode, hermitian)  # refuses an unknown recurrence by name
    if mode not in ("rank_tail", "adaptive") and not exact:
        raise NotImplementedError(f"DD mode {mode!r}: :rank_tail and :adaptive are built")
    return StepParams(
        tol_basis=tol_basis or 0.0, tol_trunc=-1.0 if tol_trunc is None else tol_trunc,
        tol_expv=tol_expv or 0.0, tol_krylov=tol_krylov or 0.0, order=order,
        maxdim=maxdim or 0, hermitian=int(hermitian),
        work_ceiling_rule=rules[work_ceiling_rule], root_ceiling_factor=float(root_ceiling_factor),
        bond_ceiling_factor=-1.0 if bond_ceiling_factor is None else float(bond_ceiling_factor),
        root=root or 0, reorth=int(reorth), truncate=int(truncate), root_maxiter=root_maxiter,
        fixed_width=width, tail_factor=tail_factor,
        krylov_mode={"auto": 0, "lanczos": 1, "arnoldi": 2}[kmode], krylov_fixed_depth=fixed_depth,
        dd_mode=1 if mode == "adaptive" else 0, holdout_width=holdout, batch_blocks=batch,
        cap_selection=1 if capsel == "svd" else 0, acceptance_factor=accept,
        closure_checks=int(bool(closure_checks)), exact=int(bool(exact)),
        fold_omega=0 if fold_omega is None else (1 if fold_omega else 2))


def cbe_bug_step(psi, mpo, tau, *, tol_basis=None, tol_trunc=None, tol_expv=None, tol_root=None,
                 tol_krylov=None, order=1, closure_probe=0, maxdim=None, hermitian=True,
                 expansion=None, rng=None, root=None, reorth=True, truncate=True,
                 work_ceiling_rule="bond", bond_ceiling_factor=None, root_ceiling_factor=1.2,
                 root_maxiter=30, krylov_rank_tol=0.0, frontier_tol=0.0, fold_omega=None,
                 closure_checks=False, eshift=0.0, root_report=None, outside_residual=False,
                 root_method="exp", root_shift=True, frames_report=None, keep_states=(),
                 keep_tols=(), frames_only=False, exact=False, parallel=False, kls=None):
    """``cbe_bug_step!(psi, mpo, tau; ...)`` (``src/BUG/TimeEvolution/bug_step.jl:17-513``) on an
    HBM-resident state, in place. Returns the step info (``CBEBugSweepInfo`` fields). The
    generators are ``H - eshift``; a dict passed as ``root_report`` receives the root's energies
    and, with ``outside_residual``, the outside-Galerkin defect after its re-enrichment
    (``_report_root!``, ``bug_step_stages.jl:243-390``). Every keyword of the reference is taken;
    the options it refuses raise ``ValueError``, the ones not built here ``NotImplementedError``
    (``options.check_step_options``)."""
    L = len(psi)
    p, keep = _step_setup(psi, mpo, rng, tol_basis=tol_basis, tol_trunc=tol_trunc, tol_expv=tol_expv,
                          tol_root=tol_root, tol_krylov=tol_krylov, order=order,
                          closure_probe=closure_probe, maxdim=maxdim, hermitian=hermitian,
                          expansion=expansion, root=root, reorth=reorth, truncate=truncate,
                          work_ceiling_rule=work_ceiling_rule,
                          bond_ceiling_factor=bond_ceiling_factor,
                          root_ceiling_factor=root_ceiling_factor, root_maxiter=root_maxiter,
                          krylov_rank_tol=krylov_rank_tol, frontier_tol=frontier_tol,
                          fold_omega=fold_omega, closure_checks=closure_checks, eshift=eshift,
                          root_report=root_report, outside_residual=outside_residual,
                          root_method=root_method, root_shift=root_shift,
                          frames_report=frames_report, keep_states=keep_states, keep_tols=keep_tols,
                          frames_only=frames_only, exact=exact, parallel=parallel, kls=kls)
    rng = keep["rng"]

    @DRAW_FN
    def draw(user, n, out):
        x = rng.standard_normal(int(n))
        ctypes.memmove(out, x.ctypes.data, 8 * int(n))

    ctx = psi.tensors[0].ctx
    tau = complex(tau)
    arr = (ctypes.c_void_p * L)(*[t.h.value for t in psi.tensors])
    warr = (ctypes.c_void_p * L)(*[w.h.value for w in mpo.tensors])
    center = ctypes.c_int(psi.center)
    info = StepInfo()
    cap = 8 * L
    logs = (BondLog * cap)()
    nlog = ctypes.c_int()
    E.check(_lib().bug_mps_step(ctx.h, L, arr, ctypes.byref(center), warr, tau.real, tau.imag,
                                ctypes.byref(p), draw, None, ctypes.byref(info), logs, cap,
                                ctypes.byref(nlog)))
    _frames_report(ctx, keep, L)
    return _step_result(psi, ctx, arr, center, info, logs, min(nlog.value, cap), order, eshift,
                        root_report)


def _step_setup(psi, mpo, rng, *, tol_basis, tol_trunc, tol_expv, tol_root, tol_krylov, order,
                closure_probe, maxdim, hermitian, expansion, root, reorth, truncate,
                work_ceiling_rule, bond_ceiling_factor, root_ceiling_factor, root_maxiter,
                krylov_rank_tol, frontier_tol, fold_omega, closure_checks, eshift, root_report,
                outside_residual, root_method, root_shift, frames_report, keep_states, keep_tols,
                frames_only, exact, parallel, kls):
    """The step's keyword checks and its ``bug_step_params`` (with the generator save/restore
    callback); returns the struct and the objects that must outlive the call."""
    L = len(psi)
    tol_expv = check_step_options(
        L, len(mpo), root=root, parallel=parallel, kls=kls, tol_expv=tol_expv, tol_root=tol_root,
        order=order, work_ceiling_rule=work_ceiling_rule, bond_ceiling_factor=bond_ceiling_factor,
        root_ceiling_factor=root_ceiling_factor, frontier_tol=frontier_tol,
        krylov_rank_tol=krylov_rank_tol, closure_probe=closure_probe, keep_states=keep_states,
        keep_tols=keep_tols, frames_only=frames_only, frames_report=frames_report, exact=exact,
        root_report=root_report, truncate=truncate, outside_residual=outside_residual)
    if outside_residual and root_report is None:
        raise ValueError("outside_residual needs root_report")
    fold = (order > 1 and not exact) if fold_omega is None else bool(fold_omega)
    if outside_residual and not fold:
        raise NotImplementedError("the outside residual with the exact (unfolded) leak")
    p = step_params(L, tol_basis=tol_basis, tol_trunc=tol_trunc, tol_expv=tol_expv,
                    tol_krylov=tol_krylov, order=order, maxdim=maxdim, hermitian=hermitian,
                    expansion=expansion, root=root, reorth=reorth, truncate=truncate,
                    work_ceiling_rule=work_ceiling_rule, bond_ceiling_factor=bond_ceiling_factor,
                    root_ceiling_factor=root_ceiling_factor,
                    root_maxiter=root_maxiter, krylov_rank_tol=krylov_rank_tol,
                    frontier_tol=frontier_tol, fold_omega=fold_omega, closure_checks=closure_checks,
                    exact=exact)
    if rng is None:
        rng = np.random.default_rng(0x5EED)
    saved = []

    @RNG_CTL_FN
    def rng_ctl(user, op):
        if op == 0:
            saved.append(rng.bit_generator.state)
        else:
            rng.bit_generator.state = saved.pop()

    methods = {"exp": 0, "trapezoid": 1, "radau2": 2, "radau3": 3, "radau2_gmres": 4}
    if root_method not in methods:
        raise NotImplementedError(f"root_method {root_method!r}: {tuple(methods)} are built")
    p.root_method = methods[root_method]
    p.root_noshift = 0 if root_shift else 1
    forks = []  # the forked streams and their callbacks live until the step returns

    @RNG_FORK_FN
    def rng_fork(user, draw_out, user_out):
        sub = fork_rng(rng)

        @DRAW_FN
        def draw_sub(u, n, out):
            x = sub.standard_normal(int(n))
            ctypes.memmove(out, x.ctypes.data, 8 * int(n))

        forks.append((sub, draw_sub))
        draw_out[0] = draw_sub
        user_out[0] = None
        return 0

    p.parallel = int(parallel is True or parallel == "half_sweeps")
    p.rng_fork = rng_fork
    p.eshift = float(eshift)
    p.root_report = int(root_report is not None)
    p.outside_residual = int(bool(outside_residual))
    p.rng_ctl = rng_ctl
    held = {"rng": rng, "rng_ctl": rng_ctl, "saved": saved, "rng_fork": rng_fork, "forks": forks}
    if len(keep_states):
        # the kept states' site handles, state-major, and their tolerances (0: contained exactly)
        for k in keep_states:
            if len(k) != L:
                raise ValueError(f"a kept state has {len(k)} sites, the state has {L}")
        sites = (ctypes.c_void_p * (len(keep_states) * L))(
            *[t.h.value for k in keep_states for t in k.tensors])
        tols = [float(t) for t in keep_tols] if len(keep_tols) else [0.0] * len(keep_states)
        ctols = (ctypes.c_double * len(tols))(*tols)
        p.n_keep = len(keep_states)
        p.keep_sites = ctypes.cast(sites, ctypes.POINTER(ctypes.c_void_p))
        p.keep_tols = ctypes.cast(ctols, ctypes.POINTER(ctypes.c_double))
        held["keep"] = (sites, ctols, list(keep_states))
    p.frames_only = int(bool(frames_only))
    if frames_report is not None:
        slots = (ctypes.c_void_p * (2 * L))()
        p.frames_out = ctypes.cast(slots, ctypes.POINTER(ctypes.c_void_p))
        held["frames"] = (slots, frames_report, float(eshift))
    return p, held


def _frames_report(ctx, held, L):
    """Fills the caller's ``frames_report`` dict from the step's frame handles (the reference's
    ``KLFrames``, ``bug_step.jl:455-467``): left frames of bonds 1..root, right frames of bonds
    root..L-1, the root's environments."""
    if "frames" not in held:
        return
    slots, report, eshift = held["frames"]
    own = [None if not slots[i] else DT(ctx, ctypes.c_void_p(slots[i])) for i in range(2 * L)]
    left = {b: own[b - 1] for b in range(1, L) if own[b - 1] is not None}
    right = {b: own[L - 2 + b] for b in range(1, L) if own[L - 2 + b] is not None}
    report.update(left_frames=left, right_frames=right, root_link=max(left), lenv=own[2 * L - 2],
                  renv=own[2 * L - 1], eshift=eshift)


def _step_result(psi, ctx, arr, center, info, logs, nlog, order, eshift, root_report):
    """Installs the step's new site handles in ``psi`` and returns the step info dict."""
    L = len(psi)
    for i in range(L):
        if arr[i]:
            psi.tensors[i] = DT(ctx, ctypes.c_void_p(arr[i]))
    psi.center = center.value
    unmet = [UNMET_NAMES[c] for c in info.unmet_order if c]
    ledger = SimpleNamespace(
        unmet=unmet, tolerance_met=info.status == 0, expv_err=info.expv_err,
        expv_iters=info.expv_iters, discarded=info.ledger_discarded, max_sample=info.max_sample,
        max_tail=info.max_tail, max_krylov=info.max_krylov, max_krylov_c=info.max_krylov_c,
        max_krylov_d=info.max_krylov_d, n_probes=info.n_probes, n_selected=info.n_selected,
        n_holdout=info.n_holdout, n_targeted=info.n_targeted,
        n_krylov=info.n_krylov, n_h1=info.n_h1, n_c_pass=info.n_c_pass, n_d_after_c=info.n_d_after_c,
        workcap_reached=bool(info.workcap_reached), maxdim_reached=bool(info.maxdim_reached),
        proj_err=info.proj_err, r_old=info.r_old, r_aug=info.r_aug, r_final=info.r_final,
        order=order, n_passes=info.n_passes, n_closure_sweeps=info.n_closure_sweeps,
        defect=info.defect, n_root_frontier=info.n_root_frontier, n_h1_closure=info.n_h1_closure,
        n_h2_leak=info.n_h2_leak, n_compress=info.n_compress,
        bond_log=[{f: getattr(logs[i], f) for f, _ in BondLog._fields_} for i in range(nlog)]
        if logs is not None else [],
    )
    ledger.status = lambda: "met" if ledger.tolerance_met else "budget_unmet"
    if root_report is not None:
        root_report.update(
            eshift=float(eshift), e_pre=info.e_pre, e_root=info.e_root,
            resid_initial=info.resid_initial, outside_passes=info.outside_passes,
            outside_added=info.outside_added, outside=info.outside, outside_left=info.outside_left,
            outside_right=info.outside_right, resid=info.resid)
    return dict(
        expanded=list(info.expanded[:L - 1]), n_new=list(info.n_new[:L - 1]),
        root_link=info.root_link, root_rank=info.root_rank, err_pre=0.0, err_fnl=0.0,
        discarded=info.discarded, n_matvec=info.n_matvec, root_frame_width=info.root_frame_width,
        ledger=ledger, status="met" if info.status == 0 else "budget_unmet",
        bond_dims=psi.bond_dims(), workcap=list(info.workcap[:L - 1]),
    )


_STEP_DEFAULTS = dict(tol_basis=None, tol_trunc=None, tol_expv=None, tol_root=None, tol_krylov=None,
                      order=1, closure_probe=0, maxdim=None, hermitian=True, expansion=None,
                      root=None, reorth=True, truncate=True, work_ceiling_rule="bond",
                      bond_ceiling_factor=None, root_ceiling_factor=1.2, root_maxiter=30,
                      krylov_rank_tol=0.0, frontier_tol=0.0, fold_omega=None,
                      closure_checks=False, eshift=0.0, root_report=None, outside_residual=False,
                      root_method="exp", root_shift=True, frames_report=None, keep_states=(),
                      keep_tols=(), frames_only=False, exact=False, parallel=False, kls=None)


class Batch:
    """Chains stepped together (``bug_step_batch``): ``n`` engine contexts and one host thread per
    chain, so the chains' host work and kernels overlap; with ``combine`` the contexts share one
    stream and the small stages the chains queue between their read-backs are merged into shared
    launches (a thread-block cluster per chain). Build chain ``i``'s state and
    MPO on ``contexts[i]`` (``tensor.from_blocks(..., ctx)``); each chain's result is the same as
    its own ``cbe_bug_step``. The batch is torn down when the last reference to it or to a tensor
    on its contexts goes away (tensors hold their context, which holds the batch)."""

    class _Handle:
        def __init__(self, lib, h):
            self.lib, self.h = lib, h

        def __del__(self):
            if self.h:
                self.lib.bug_batch_destroy(self.h)
                self.h = None

    def __init__(self, n: int, device: int = 0, combine: bool = False):
        lib = _lib()
        h = ctypes.c_void_p()
        E.check(lib.bug_batch_create(int(device), int(n), int(bool(combine)), ctypes.byref(h)))
        self._handle = Batch._Handle(lib, h)
        self.h, self.n, self.lib = h, int(n), lib
        self.contexts = []
        for i in range(self.n):
            c = ctypes.c_void_p()
            E.check(lib.bug_batch_context(h, i, ctypes.byref(c)))
            self.contexts.append(E.Context.borrow(c, device, owner=self._handle))

    def launches(self) -> int:
        return int(self.lib.bug_batch_launches(self.h))

    def step(self, states, mpos, taus, rngs, **kw) -> list:
        """One ``cbe_bug_step`` of every chain (``states[i]``, ``mpos[i]``, ``taus[i]``, drawing
        from ``rngs[i]``), the same keywords for all; returns the per-chain info dicts."""
        n = len(states)
        if not (len(mpos) == len(taus) == len(rngs) == n) or n < 1 or n > self.n:
            raise ValueError("Batch.step: one state, MPO, tau and generator per chain")
        opts = dict(_STEP_DEFAULTS)
        unknown = set(kw) - set(opts)
        if unknown:
            raise TypeError(f"unknown keywords {sorted(unknown)}")
        opts.update(kw)
        params = (StepParams * n)()
        keeps = []
        for i in range(n):
            p, keep = _step_setup(states[i], mpos[i], rngs[i], **opts)
            params[i] = p
            keeps.append(keep)
        gens = [k["rng"] for k in keeps]

        @DRAW_FN
        def draw(user, count, out):
            x = gens[int(user or 0)].standard_normal(int(count))
            ctypes.memmove(out, x.ctypes.data, 8 * int(count))

        Ls = (ctypes.c_int * n)(*[len(s) for s in states])
        arrs = [(ctypes.c_void_p * len(s))(*[t.h.value for t in s.tensors]) for s in states]
        warrs = [(ctypes.c_void_p * len(m))(*[w.h.value for w in m.tensors]) for m in mpos]
        psi_io = (ctypes.c_void_p * n)(*[ctypes.cast(a, ctypes.c_void_p).value for a in arrs])
        mpo_p = (ctypes.c_void_p * n)(*[ctypes.cast(a, ctypes.c_void_p).value for a in warrs])
        centers = (ctypes.c_int * n)(*[s.center for s in states])
        tr = (ctypes.c_double * n)(*[complex(t).real for t in taus])
        ti = (ctypes.c_double * n)(*[complex(t).imag for t in taus])
        users = (ctypes.c_void_p * n)(*range(n))
        infos = (StepInfo * n)()
        status = (ctypes.c_int * n)()
        E.check(self.lib.bug_step_batch(self.h, n, Ls, ctypes.cast(psi_io, ctypes.c_void_p), centers,
                                        ctypes.cast(mpo_p, ctypes.c_void_p), tr, ti, params, draw,
                                        ctypes.cast(users, ctypes.c_void_p), infos, status))
        out = []
        for i in range(n):
            center = ctypes.c_int(centers[i])
            out.append(_step_result(states[i], states[i].tensors[0].ctx, arrs[i], center, infos[i],
                                    None, 0, opts["order"], opts["eshift"], opts["root_report"]))
        return out


# ── kernel-granular entry points (``bug_env_step`` ... ``bug_observable_sz``) ──────────────────


def _call(ctx, fn, *args):
    h = ctypes.c_void_p()
    E.check(getattr(ctx.lib, fn)(ctx.h, *args, ctypes.byref(h)))
    return DT(ctx, h) if h.value else None


def env_boundary(ctx, side: str, charge: int = 0) -> DT:
    """Chain-end environment: ``side`` "left" or "right" (the latter carrying the total charge)."""
    return _call(ctx, "bug_env_boundary", 0 if side == "left" else 1, int(charge))


def env_step(env: DT, A: DT, W: DT, side: str) -> DT:
    """``_mpo_left_step`` / ``_mpo_right_step`` (``mpo_environments.jl:65-108``)."""
    return _call(env.ctx, "bug_env_step", 0 if side == "left" else 1, env.h, A.h, W.h)


def apply_one_site(lenv: DT, W: DT, renv: DT, x: DT) -> DT:
    """``apply_one_site`` (``effective_operators.jl:27-64``)."""
    return _call(x.ctx, "bug_apply_one_site", lenv.h, W.h, renv.h, x.h)


def apply_zero_site(lgen: DT, rgen: DT, core: DT) -> DT:
    """``apply_zero_site`` (``effective_operators.jl:91-107``)."""
    return _call(core.ctx, "bug_apply_zero_site", lgen.h, rgen.h, core.h)


def sketch_stream(side: str, a: DT, b: DT, Wl: DT, Wr: DT, lenv: DT, renv: DT, probe: DT) -> DT:
    """``_stream_left`` / ``_stream_right`` (``mpo_environments.jl:409-481``): side "left" with
    ``a = U0 S0``, ``b = V0``; side "right" with ``a = U0``, ``b = S0 V0``."""
    return _call(probe.ctx, "bug_sketch_stream", 0 if side == "left" else 1, a.h, b.h, Wl.h, Wr.h,
                 lenv.h, renv.h, probe.h)


def perp(side: str, frame: DT, K: DT) -> DT:
    """``perp_component`` / ``perp_component_right`` (``sectors.jl:215-240``)."""
    return _call(K.ctx, "bug_perp", 0 if side == "left" else 1, frame.h, K.h)


def root_expv(lgen: DT, rgen: DT, core: DT, tau, hermitian=True, maxiter=30, reorth=True,
              tol_expv=1e-10):
    """``expv`` of the root (``root_methods.jl:359-402``): ``(exp(tau H0) core, H0 applications,
    accumulated tail estimate)``."""
    tau = complex(tau)
    ctx = core.ctx
    h = ctypes.c_void_p()
    iters, err = ctypes.c_int64(), ctypes.c_double()
    E.check(ctx.lib.bug_root_expv(ctx.h, lgen.h, rgen.h, core.h, tau.real, tau.imag, int(hermitian),
                                  int(maxiter), int(reorth), float(tol_expv), ctypes.byref(h),
                                  ctypes.byref(iters), ctypes.byref(err)))
    return DT(ctx, h), int(iters.value), float(err.value)


def _handles(psi):
    return (ctypes.c_void_p * len(psi.tensors))(*[t.h.value for t in psi.tensors])


def site_populations(psi) -> list:
    """Normalised local populations per site, the site leg's indices in leg order."""
    ctx = psi.tensors[0].ctx
    n = ctypes.c_int()
    E.check(ctx.lib.bug_site_populations(ctx.h, len(psi.tensors), _handles(psi), psi.center, None, 0,
                                         ctypes.byref(n)))
    buf = np.zeros(max(n.value, 1))
    E.check(ctx.lib.bug_site_populations(ctx.h, len(psi.tensors), _handles(psi), psi.center,
                                         buf.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), n.value,
                                         ctypes.byref(n)))
    out, k = [], 0
    for t in psi.tensors:
        d = sum(t.legs[1].sectors.values())
        out.append(buf[k:k + d].copy())
        k += d
    return out


def observable_sz(psi) -> np.ndarray:
    """``<S^z_j>`` for every site (``bug_observable_sz``)."""
    ctx = psi.tensors[0].ctx
    out = np.zeros(len(psi.tensors))
    E.check(ctx.lib.bug_observable_sz(ctx.h, len(psi.tensors), _handles(psi), psi.center,
                                      out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
    return out


def apply_two_site(lenv: DT, Wl: DT, Wr: DT, renv: DT, theta: DT) -> DT:
    """``apply_h_two_site`` (``mpo_environments.jl:316-344``) on a two-site tensor ``(l, s1, s2, r)``."""
    return _call(theta.ctx, "bug_apply_two_site", lenv.h, Wl.h, Wr.h, renv.h, theta.h)


# ── two-site TDVP baseline (``bug_tdvp2_step``) ───────────────────────────────────────────────


class TDVP2Params(ctypes.Structure):
    _fields_ = [("maxdim", ctypes.c_int), ("trunc_thresh", ctypes.c_double), ("maxiter", ctypes.c_int),
                ("tol", ctypes.c_double), ("hermitian", ctypes.c_int), ("conv_tol", ctypes.c_double),
                ("substeps", ctypes.c_int), ("weight_tol", ctypes.c_double), ("eshift", ctypes.c_double)]


class TDVP2Info(ctypes.Structure):
    _fields_ = [("max_bond", ctypes.c_int), ("theta_elements", ctypes.c_int64),
                ("discarded", ctypes.c_double), ("peak_elements", ctypes.c_int64),
                ("krylov_dims", ctypes.c_int64), ("cumulative", ctypes.c_double)]


def tdvp2_step(psi, mpo, tau, *, maxdim=200, trunc_thresh=1e-12, maxiter=30, tol=1e-15,
               hermitian=True, conv_tol=0.0, substeps=1, weight_tol=None, eshift=0.0,
               backward_report=None, backward_norms=None) -> dict:
    """``tdvp2_step!(psi, h, tau; ...)`` (``src/Baselines/TDVP/tdvp2.jl:229-297``): one symmetric
    two-site TDVP step on an HBM-resident state, in place. Returns the ``TDVP2Info`` fields. The
    backward-substep amplification reports (``backward_report``, ``backward_norms``) are not
    built and raise ``NotImplementedError`` when asked for."""
    L = len(psi)
    if L < 2:
        raise ValueError("tdvp2_step needs at least two sites")
    if len(mpo) != L:
        raise ValueError(f"chain has {len(mpo)} sites, state has {L}")
    if weight_tol is not None and weight_tol < 0:
        raise ValueError(f"weight_tol must be non-negative, got {weight_tol}")
    if backward_report is not None or backward_norms is not None:
        raise NotImplementedError("backward_report / backward_norms are not built")
    lib = E.load()
    lib.bug_tdvp2_step.restype = ctypes.c_int
    lib.bug_tdvp2_step.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p),
                                   ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_void_p),
                                   ctypes.c_double, ctypes.c_double, ctypes.POINTER(TDVP2Params),
                                   ctypes.POINTER(TDVP2Info)]
    p = TDVP2Params(maxdim=int(maxdim), trunc_thresh=float(trunc_thresh), maxiter=int(maxiter),
                    tol=float(tol), hermitian=int(hermitian), conv_tol=float(conv_tol),
                    substeps=int(substeps), weight_tol=-1.0 if weight_tol is None else float(weight_tol),
                    eshift=float(eshift))
    ctx = psi.tensors[0].ctx
    tau = complex(tau)
    arr = (ctypes.c_void_p * L)(*[t.h.value for t in psi.tensors])
    warr = (ctypes.c_void_p * L)(*[w.h.value for w in mpo.tensors])
    center = ctypes.c_int(psi.center)
    info = TDVP2Info()
    E.check(lib.bug_tdvp2_step(ctx.h, L, arr, ctypes.byref(center), warr, tau.real, tau.imag,
                               ctypes.byref(p), ctypes.byref(info)))
    for i in range(L):
        if arr[i]:
            psi.tensors[i] = DT(ctx, ctypes.c_void_p(arr[i]))
    psi.center = center.value
    return {f: getattr(info, f) for f, _ in TDVP2Info._fields_}
