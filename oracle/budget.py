"""Tolerance budget, work ceilings and the step ledger of the CPU oracle.

TEST INFRASTRUCTURE (see ``oracle/blocks.py``). Restates
``src/BUG/Core/RankAdaptation/basis_budget.jl``: ``AdaptiveBudget`` (``:12-23``),
``basis_allocation`` (``:75-119``), ``indicator`` (``:128``), ``AdaptiveLedger`` (``:144-275``),
``_unmet!`` (``:284-288``), ``budget_status`` (``:298-299``), ``merge_ledger!`` (``:343-387``),
``_log_bond!`` (``:399-436``), ``work_ceiling`` (``:454-455``), ``bond_work_ceilings``
(``:484-494``), ``TOL_DEFAULTS`` (``:568``); and ``_tail_rank`` (``truncation.jl:262-278``).
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

TOL_DEFAULTS = dict(basis=1e-5, trunc=1e-7, expv=1e-10)
DEFAULT_BOND_CEILING_FACTOR = 1.2
ADAPTIVE_GROWTH = 1.2


@dataclass
class Budget:
    basis: float
    trunc: float
    expv: float

    def __post_init__(self):
        if not self.basis > 0:
            raise ValueError(f"tol_basis must be positive, got {self.basis}")
        if not self.trunc >= 0:
            raise ValueError(f"tol_trunc must be non-negative, got {self.trunc}")
        if not self.expv > 0:
            raise ValueError(f"tol_expv must be positive, got {self.expv}")


@dataclass
class Allocation:
    per_bond: float
    sample: float
    tail: float
    krylov: float
    scale: float
    rule: str = "rss"
    krylov_rank: float = 0.0


def basis_allocation(budget: Budget, nbonds: int, tau=0, nrm=1.0, nfront=1, rule="rss",
                     krylov=None, krylov_rank=0.0) -> Allocation:
    nb = max(nbonds, 1)
    nf = max(nfront, 1)
    if rule not in ("rss", "linear"):
        raise ValueError(f"rule must be rss or linear, got {rule}")
    kr = 1.0 if krylov is None else float(krylov) / budget.basis
    if not kr > 0:
        raise ValueError(f"tol_krylov must be positive, got {krylov}")
    if not krylov_rank >= 0:
        raise ValueError(f"krylov_rank_tol must be >= 0, got {krylov_rank}")
    rank_share = float(krylov_rank) / budget.basis
    at = abs(tau)
    scale = 1.0 if at == 0 else at / max(float(nrm), 2.220446049250313e-16)
    if rule == "linear":
        per_test = budget.basis / (2 * (nb + 1) * nf)
        return Allocation(2 * per_test, per_test, per_test, kr * per_test, scale, "linear",
                          rank_share * per_test)
    per_bond = budget.basis / math.sqrt(nb * nf)
    per_test = per_bond / math.sqrt(4)
    return Allocation(per_bond, per_test, per_test, kr * per_test, scale, "rss", rank_share * per_test)


def indicator(alloc: Allocation, resid: float) -> float:
    return alloc.scale * float(resid)


@dataclass
class Ledger:
    max_sample: float = 0.0
    max_sample_l: float = 0.0
    max_sample_r: float = 0.0
    max_tail: float = 0.0
    max_krylov: float = 0.0
    max_krylov_c: float = 0.0
    max_krylov_d: float = 0.0
    discarded: float = 0.0
    expv_err: float = 0.0
    n_probes: int = 0
    n_holdout: int = 0
    n_selected: int = 0
    n_krylov: int = 0
    n_h1: int = 0
    n_targeted: int = 0
    n_c_pass: int = 0
    n_d_after_c: int = 0
    workcap_reached: bool = False
    tolerance_met: bool = True
    maxdim_reached: bool = False
    proj_err: float = 0.0
    r_old: int = 0
    r_aug: int = 0
    r_final: int = 0
    expv_iters: int = 0
    unmet: list = field(default_factory=list)
    sample_log: list = field(default_factory=list)
    bond_log: list = field(default_factory=list)
    order: int = 1
    n_passes: int = 0
    n_closure_sweeps: int = 0
    leak: list = field(default_factory=list)
    defect: float = 0.0
    n_root_frontier: int = 0
    # the frontiers measured on the half-sweeps' frames before any closure enrichment
    # (basis_budget.jl:219-225): time-weighted leaks and scale-free ||(I - P) A F_j|| / ||F_j||
    leak_initial: list = field(default_factory=list)
    rho_initial: list = field(default_factory=list)
    n_h2_leak: int = 0
    n_h1_closure: int = 0
    closure_log: list = field(default_factory=list)
    n_compress: int = 0

    def unmet_(self, what: str):
        self.tolerance_met = False
        if what not in self.unmet:
            self.unmet.append(what)
        return self

    def status(self) -> str:
        return "met" if self.tolerance_met else "budget_unmet"

    def merge(self, o: "Ledger") -> "Ledger":
        self.max_sample = max(self.max_sample, o.max_sample)
        self.max_sample_l = max(self.max_sample_l, o.max_sample_l)
        self.max_sample_r = max(self.max_sample_r, o.max_sample_r)
        self.sample_log += o.sample_log
        self.max_tail = max(self.max_tail, o.max_tail)
        self.max_krylov = max(self.max_krylov, o.max_krylov)
        self.max_krylov_c = max(self.max_krylov_c, o.max_krylov_c)
        self.max_krylov_d = max(self.max_krylov_d, o.max_krylov_d)
        self.n_c_pass += o.n_c_pass
        self.n_d_after_c += o.n_d_after_c
        self.discarded = max(self.discarded, o.discarded)
        self.expv_err = max(self.expv_err, o.expv_err)
        self.n_probes += o.n_probes
        self.n_holdout += o.n_holdout
        self.n_selected += o.n_selected
        self.n_krylov += o.n_krylov
        self.n_h1 += o.n_h1
        self.n_targeted += o.n_targeted
        self.workcap_reached |= o.workcap_reached
        self.tolerance_met &= o.tolerance_met
        self.maxdim_reached |= o.maxdim_reached
        self.proj_err = max(self.proj_err, o.proj_err)
        self.r_old = max(self.r_old, o.r_old)
        self.r_aug = max(self.r_aug, o.r_aug)
        self.r_final = max(self.r_final, o.r_final)
        self.expv_iters += o.expv_iters
        for u in o.unmet:
            if u not in self.unmet:
                self.unmet.append(u)
        self.bond_log += o.bond_log
        self.order = max(self.order, o.order)
        self.n_passes += o.n_passes
        self.n_closure_sweeps += o.n_closure_sweeps
        self.leak += o.leak
        self.defect = max(self.defect, o.defect)
        self.n_root_frontier += o.n_root_frontier
        self.leak_initial += o.leak_initial
        self.rho_initial += o.rho_initial
        self.n_h2_leak += o.n_h2_leak
        self.n_h1_closure += o.n_h1_closure
        self.closure_log += o.closure_log
        self.n_compress += o.n_compress
        return self


def log_bond(ledger: Ledger, bl: Ledger, bond: int, side: str, width: int) -> Ledger:
    """Close one bond of a sweep into ``bl.bond_log`` and fold ``bl`` in (``basis_budget.jl:399-436``)."""
    final = {}
    for e in bl.sample_log:
        final[e["side"]] = e["sketch"]
    bl.bond_log.append(dict(
        bond=bond, side=side, sample=bl.max_sample, tail=bl.max_tail,
        krylov_c=bl.max_krylov_c, krylov_d=bl.max_krylov_d, n_probes=bl.n_probes,
        n_holdout=bl.n_holdout, n_selected=bl.n_selected, n_targeted=bl.n_targeted,
        n_krylov=bl.n_krylov, n_h1=bl.n_h1, c_pass=bl.n_c_pass > 0, d_after_c=bl.n_d_after_c > 0,
        workcap=bl.workcap_reached, met=bl.tolerance_met, unmet=list(bl.unmet), width=width,
        n_sectors=sum(len(v) for v in final.values()), probes_per_sector=final,
    ))
    return ledger.merge(bl)


def work_ceiling(maxdim: int, bond_rank: int, site_dim: int = 2) -> int:
    return max(site_dim * maxdim, site_dim * bond_rank, 1)


def _ceil9(x: float) -> int:
    return math.ceil(round(x, 9))


def bond_work_ceilings(bond_ranks, site_dim: int, maxdim: int, factor: float = 0.0):
    def ceiling_of(r):
        return _ceil9(factor * site_dim * r) if factor > 0 else 2 * site_dim * r

    return [max(min(ceiling_of(r), maxdim), 1) for r in bond_ranks]


def bond_work_ceilings_strict(bond_ranks, maxdim: int, factor: float = 1.2):
    """``bond_work_ceilings_strict`` (``basis_budget.jl:497-508``): ``ceil(f D_b)`` per bond,
    without the local dimension."""
    if not factor > 1:
        raise ValueError("strict bond factor must exceed 1")
    return [max(1, min(maxdim, _ceil9(factor * r))) for r in bond_ranks]


def bond_frame_root_ceilings(old_bonds, maxdim: int, root_bond: int, frame_factor: float = 2.0,
                             root_factor: float = 1.2):
    """``bond_frame_root_ceilings`` (``basis_budget.jl:511-545``): ``ceil(frame_factor D_b)``
    away from the root bond, ``ceil(root_factor D_root)`` at it."""
    if not 1 <= root_bond <= len(old_bonds):
        raise ValueError(f"root bond {root_bond} outside 1:{len(old_bonds)}")
    if not frame_factor > 1:
        raise ValueError("frame_factor must exceed 1")
    if not root_factor > 1:
        raise ValueError("root_factor must exceed 1")
    if root_factor > frame_factor:
        raise ValueError("root_factor cannot exceed frame_factor")
    if maxdim < 1:
        raise ValueError("maxdim must be positive")
    return [max(1, min(maxdim, _ceil9((root_factor if b + 1 == root_bond else frame_factor) * r)))
            for b, r in enumerate(old_bonds)]


def tail_rank(lst, scale: float, allowance: float, kmax: int, base: float = 0.0):
    """Test A: the smallest ``keep <= kmax`` whose scaled tail fits ``allowance``
    (``truncation.jl:262-278``)."""
    n = len(lst)
    kmax = min(kmax, n)
    if kmax <= 0:
        return 0, scale * math.sqrt(base + sum(float(s) ** 2 * float(d) for s, d, _, _ in lst))
    weights = [float(s) ** 2 * float(d) for s, d, _, _ in lst]
    tail = base + sum(weights[kmax:n])
    keep = kmax
    while keep > 0:
        trial = tail + weights[keep - 1]
        if not scale * math.sqrt(trial) <= allowance:
            break
        tail = trial
        keep -= 1
    return keep, scale * math.sqrt(tail)
