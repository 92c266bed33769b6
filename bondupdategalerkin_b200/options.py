"""The keyword checks of ``cbe_bug_step!`` (``src/BUG/TimeEvolution/bug_step_stages.jl:40-142``).

Every keyword of the reference step is accepted under its own name. A value the reference refuses
raises ``ValueError`` (its ``ArgumentError`` / ``DimensionMismatch``) with the reference's reason,
in the reference's order; a valid value of an option this engine does not build raises
``NotImplementedError`` naming it. The checks are pure host logic, run before any device work.
"""

from __future__ import annotations

from dataclasses import dataclass

# the per-bond work ceiling's factor under `:bond` (basis_budget.jl:484-494): frames at most
# ceil(factor d D_b)
DEFAULT_BOND_CEILING_FACTOR = 1.2


@dataclass
class DDQRExpansion:
    """``DDQRExpansion`` defaults (``src/BUG/Randomised/cbe.jl:254-290``): the expansion settings
    the step passes to the native library (``bug_step_params``)."""

    mode: str = "rank_tail"
    fixed_width: int = 8
    fixed_rank: int = 0
    rank_initial_width: int = 4
    rank_floor: int = 0
    tail_factor: float = 0.10
    holdout_width: int = 4
    batch_blocks: int = 1
    cap_selection: str = "storage"
    acceptance_factor: float = 1.0
    krylov_mode: str = "auto"
    krylov_fixed_depth: int = 0

KLS_SCHEDULES = ("sequential", "kl_then_s", "concurrent")  # parallel_kls.jl:7
WORK_CEILING_RULES = ("maxdim", "bond", "bond_strict", "frame_root")
BUILT_WORK_CEILING_RULES = ("maxdim", "bond", "bond_strict", "frame_root")


def _parallel_mode(parallel):
    """``_resolve_parallel`` (``dd_cbe_expand.jl:428-433``): ``(mode name, runs in parallel)``."""
    if isinstance(parallel, bool):
        return ("half_sweeps" if parallel else "serial"), parallel
    if parallel == "serial":
        return "serial", False
    if parallel in ("half_sweeps", "full"):
        return parallel, True
    raise ValueError(f"parallel must be :serial, :half_sweeps, :full or a Bool, got {parallel!r}")


def check_step_options(L, mpo_len, *, root=None, parallel=False, kls=None, tol_expv=None,
                       tol_root=None, order=1, work_ceiling_rule="bond", bond_ceiling_factor=None,
                       root_ceiling_factor=1.2, frontier_tol=0.0, krylov_rank_tol=0.0,
                       closure_probe=0, keep_states=(), keep_tols=(), frames_only=False,
                       frames_report=None, exact=False, root_report=None, truncate=True,
                       outside_residual=False):
    """Check the options as ``_step_options`` does and return ``tol_expv`` (``tol_root`` is its
    other name)."""
    if mpo_len != L:
        raise ValueError(f"MPO has {mpo_len} sites, state has {L}")
    if L < 2:
        raise ValueError("cbe_bug_step needs at least two sites")
    root_link = (L // 2) if root is None else root  # _bug_root_link: the middle bond
    if not 1 <= root_link <= L - 1:
        raise ValueError(f"root must be a bond in 1:{L - 1}, got {root_link}")
    mode, _ = _parallel_mode(parallel)
    if mode == "full" and kls is None:
        kls = "concurrent"
    if tol_root is not None and tol_expv is not None:
        raise ValueError("tol_root and tol_expv name the same tolerance; pass one")
    if tol_root is not None:
        tol_expv = tol_root
    if order < 1:
        raise ValueError(f"order must be >= 1, got {order}")
    if bond_ceiling_factor is None:
        bond_ceiling_factor = DEFAULT_BOND_CEILING_FACTOR if work_ceiling_rule == "bond" else 0.0
    if frontier_tol < 0:
        raise ValueError(f"frontier_tol must be >= 0, got {frontier_tol}")
    if work_ceiling_rule not in WORK_CEILING_RULES:
        raise ValueError("work_ceiling_rule must be :maxdim, :bond, :bond_strict or :frame_root, "
                         f"got {work_ceiling_rule!r}")
    if not (bond_ceiling_factor == 0 or (bond_ceiling_factor > 1 and work_ceiling_rule in
                                         ("bond", "bond_strict", "frame_root"))):
        raise ValueError("bond_ceiling_factor must be 0, or > 1 with work_ceiling_rule = :bond, got "
                         f"{bond_ceiling_factor} with :{work_ceiling_rule}")
    if not root_ceiling_factor > 1:
        raise ValueError("root_ceiling_factor must exceed one")
    if work_ceiling_rule == "frame_root" and \
            root_ceiling_factor > (2.0 if bond_ceiling_factor == 0 else bond_ceiling_factor):
        raise ValueError("root_ceiling_factor must not exceed frame factor")
    if closure_probe < 0:
        raise ValueError(f"closure_probe must be a non-negative count, got {closure_probe}")
    keep_states, keep_tols = list(keep_states), list(keep_tols)
    if keep_tols and len(keep_tols) != len(keep_states):
        raise ValueError(f"keep_tols has {len(keep_tols)} entries for {len(keep_states)} keep_states")
    if any(t < 0 for t in keep_tols):
        raise ValueError(f"keep_tols must be >= 0, got {keep_tols}")
    if frames_only and (root_report is not None or kls is not None or truncate):
        raise ValueError("frames_only needs root_report = nothing, kls = nothing and truncate = false")
    if kls is not None:
        if kls not in KLS_SCHEDULES:
            raise ValueError(f"the K/L/S schedule must be one of {KLS_SCHEDULES}, got {kls!r}")
        if outside_residual:
            raise ValueError("the parallel K/L/S step does not combine with the outside-residual "
                             "re-enrichment")
    # bond_work_ceilings_strict refuses a factor of at most one (basis_budget.jl:506), which the
    # step's default factor 0 under :bond_strict is
    if work_ceiling_rule == "bond_strict" and not bond_ceiling_factor > 1:
        raise ValueError("strict bond factor must exceed 1")
    # valid, but not built here
    unbuilt = []
    if kls is not None:
        unbuilt.append(f"parallel = {parallel!r} / kls = {kls!r} (the parallel K/L/S step)")
    if work_ceiling_rule not in BUILT_WORK_CEILING_RULES:
        unbuilt.append(f"work_ceiling_rule = :{work_ceiling_rule}")
    if frontier_tol > 0 or krylov_rank_tol > 0:
        unbuilt.append("frontier_tol / krylov_rank_tol > 0")
    if closure_probe > 0:
        unbuilt.append("closure_probe > 0 (the frontier measurement of order-1 steps)")
    if unbuilt:
        raise NotImplementedError("not built: " + "; ".join(unbuilt))
    return tol_expv


KRYLOV_MODES = ("auto", "lanczos", "arnoldi")


def resolve_krylov_recurrence(mode, hermitian):
    """``resolve_krylov_recurrence`` (``src/BUG/Randomised/cbe.jl:299``): ``auto`` is Lanczos on a
    Hermitian step and Arnoldi otherwise, an explicit recurrence is kept, another name is refused."""
    if mode not in KRYLOV_MODES:
        raise ValueError(f"krylov_mode must be :auto, :lanczos or :arnoldi, got {mode!r}")
    if mode == "auto":
        return "lanczos" if hermitian else "arnoldi"
    return mode
