"""The rank-adaptive BUG step of the CPU oracle: ``cbe_bug_step``.

TEST INFRASTRUCTURE (see ``oracle/blocks.py``). Restates, in the reference's order:

* ``cbe_bug_step!`` (``src/BUG/TimeEvolution/bug_step.jl:17-513``) with ``_resolve_step_options``
  (``bug_step_stages.jl:15-142``), ``_close_root_frontiers!`` (``:172-240``), ``_step_info``
  (``:473-544``);
* the half-sweeps ``_half_left!`` / ``_half_right!`` (``src/BUG/Core/Sweeps/half_sweeps.jl:218-410``);
* ``_frame_from`` (``effective_operators.jl:201-220``), ``canonical!`` / ``move_left!`` /
  ``move_right!`` (``canonical_form.jl:317-361``);
* ``_krylov_enrich`` / ``_extend_frame`` / ``_record_krylov!`` (``krylov_enrichment.jl:135-307``);
* ``_overlap_left/right``, ``_projection_miss``, ``_project_root``, ``_projected_frontiers``,
  ``_frontier_mps`` (``krylov_closure_frames.jl:207-355``);
* ``_single_pass_closure!`` (``krylov_closure_loop.jl:203-281``), ``_frontier_sweep!``
  (``frontier_closure.jl:42-222``), ``_frontier_left/right`` and ``_polar_frame``
  (``frontier_sweeps.jl:20-354``), ``_frame_onto_left/right`` and ``_bond_action``
  (``krylov_frontier_bonds.jl:13-106``);
* ``truncate_recursive!`` / ``_budget_svd`` / ``_cut_divisor`` (``truncation.jl:49-158``) and
  ``_assemble_and_compress!`` (``diagnostics.jl:269-337``).

Scope: ``mode = :rank_tail`` DD-QR expansion, Lanczos/Arnoldi local Krylov with the sequential
rule, ``order >= 1`` with the single-pass or checked closure and the folded (sampled) or, with
``fold_omega = false``, exact frontier leaks; ``exact = true`` expands by the complete DD-projected
fused basis, ``keep_states`` are unioned into the frames, ``frames_only`` skips the root solve and
``frames_report`` (a dict) receives the frames, ``krylov_rank_tol`` ranks the local Krylov
directions and ``frontier_tol`` compresses each frontier before its sweep. The K/L/S schedules
raise.
"""

from __future__ import annotations

import copy
import math
import time
from dataclasses import dataclass, replace

import numpy as np

from . import blocks as B
from . import krylov as K
from .budget import (DEFAULT_BOND_CEILING_FACTOR, TOL_DEFAULTS, Budget, Ledger,
                     basis_allocation, bond_frame_root_ceilings, bond_work_ceilings,
                     bond_work_ceilings_strict, indicator, log_bond, tail_rank, work_ceiling)
from .cbe import (CBE_EPS, BondFrame, cap_to_local_room, dd_cbe_expand, exact_leak,
                  folded_closures, perp_left, perp_right, rank_cut, reortho, rows_from_u,
                  sampled_leak)
from .env import (ZeroSiteH, apply_one_site, left_boundary, left_env_stack, left_step,
                  right_boundary, right_env_stack, right_step, total_charge)

VOPS = K.VecOps()
FRONTIER_FLOOR = 1e-14


@dataclass
class DDQRExpansion:
    """``DDQRExpansion`` defaults (``src/BUG/Randomised/cbe.jl:254-290``)."""

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


# ── canonical form ───────────────────────────────────────────────────────────────────────────


def move_right(psi, site):
    res = B.svd(psi[site], (0, 1), cutoff=0.0)
    psi[site + 1] = B.contract(res.SVd(), (1,), psi[site + 1], (0,))
    psi[site] = res.U


def move_left(psi, site):
    res = B.svd(psi[site], (0,), cutoff=0.0)
    psi[site - 1] = B.contract(psi[site - 1], (2,), res.US(), (0,))
    psi[site] = res.Vd


def canonical(psi, site):
    if not 1 <= site <= len(psi):
        raise IndexError(site)
    while psi.center < site:
        move_right(psi, psi.center)
        psi.center += 1
    while psi.center > site:
        move_left(psi, psi.center)
        psi.center -= 1
    return psi


def frame_from(left, right) -> BondFrame:
    res_l = B.svd(left, (0, 1), cutoff=0.0)
    res_r = B.svd(right, (0,), cutoff=0.0)
    core = B.contract(res_l.SVd(), (1,), res_r.US(), (0,))
    return BondFrame(res_l.U, core, res_r.Vd, res_l.U.dim(2))


def frame_onto_left(left_isometry, carry, right) -> BondFrame:
    res_r = B.svd(right, (0,), cutoff=0.0)
    ov = B.contract(left_isometry, (0, 1), carry, (0, 1), conja=True)
    return BondFrame(left_isometry, B.contract(ov, (1,), res_r.US(), (0,)), res_r.Vd,
                     left_isometry.dim(2))


def frame_onto_right(left, carry, right_isometry) -> BondFrame:
    res_l = B.svd(left, (0, 1), cutoff=0.0)
    ov = B.contract(carry, (1, 2), right_isometry, (1, 2), conjb=True)
    return BondFrame(res_l.U, B.contract(res_l.SVd(), (1,), ov, (0,)), right_isometry,
                     right_isometry.dim(0))


def polar_frame(frame, side):
    if side == "left":
        res = B.svd(frame, (0, 1), cutoff=0.0)
        return B.contract(res.U, (2,), res.Vd, (0,))
    res = B.svd(frame, (0,), cutoff=0.0)
    return B.contract(res.U, (1,), res.Vd, (0,))


# ── local Krylov enrichment (Tests C/D) ─────────────────────────────────────────────────────


def extend_frame(frame, residual, direction, side, weight, allowance, room):
    legs = (0, 1) if side == "left" else (1, 2)
    nres = B.norm(residual)
    cut = rank_cut(0.0, B.norm(direction), nres)
    res = B.svd(residual, legs, cutoff=cut)
    nk = len(res.kept)
    keep, tail = tail_rank(res.kept, weight, allowance, min(nk, room), base=B.sq_weight(res.trunc))
    fits = tail <= allowance
    if keep == 0:
        return frame, 0, fits
    if keep < nk:
        res = B.svd(residual, legs, cutoff=cut, nkeep=keep)
    if side == "left":
        nb = reortho(frame, res.U, "left")
    else:
        nb = reortho(frame, rows_from_u(res.U), "right")
    nb = cap_to_local_room(frame, nb, side)
    if nb is None:
        return frame, 0, fits
    fl = 2 if side == "left" else 0
    return B.oplus([frame, nb], fl), nb.dim(fl), fits


def append_ranked(frame, cands, side, allowance, workcap):
    """``_append_ranked`` (``krylov_enrichment.jl:186-195``): one SVD of the collected weighted
    residuals' direct sum ranks their local directions, and the fewest top ones whose discarded
    tail fits ``allowance`` join the frame; ``fits = False`` when the work ceiling cut more."""
    if not cands:
        return frame, 0, True
    fl = 2 if side == "left" else 0
    room = workcap - frame.dim(fl) if workcap > 0 else 1 << 62
    block = cands[0] if len(cands) == 1 else B.oplus(cands, fl)
    if room <= 0:
        return frame, 0, B.norm(block) <= allowance
    return extend_frame(frame, block, block, side, 1.0, allowance, room)


def krylov_enrich(seed, applyH, start_frame, side, tau, alloc, workcap=0, amp=1.0,
                  state_seed=True, recurrence="arnoldi", fixed_depth=0):
    """``_krylov_enrich`` (``krylov_enrichment.jl:213-292``): Tests C/D on each Krylov direction,
    appending in chain order, or with ``alloc.krylov_rank > 0`` collecting every direction above
    the allowance against the start frame and ranking them at the end (:func:`append_ranked`)."""
    perp = perp_left if side == "left" else perp_right
    fl = 2 if side == "left" else 0
    allow = alloc.krylov
    ranked = alloc.krylov_rank > 0
    cands = []
    st = dict(frame=start_frame, eta_c=0.0, eta_d=0.0, added=0, added_d=0, nd=0)

    def score(direction, weight, first):
        residual = perp(st["frame"], direction)
        eta = weight * B.norm(residual)
        if first:
            st["eta_c"] = eta
        else:
            st["eta_d"] = max(st["eta_d"], eta)
        if not eta > allow:
            return True
        if ranked:  # the frame stays the start frame: every candidate against the same frame
            cands.append(B.scale(residual, weight))
            if not first:
                st["nd"] += 1
            return True
        room = workcap - st["frame"].dim(fl) if workcap > 0 else 1 << 62
        if room <= 0:
            return False
        st["frame"], nadd, fits = extend_frame(st["frame"], residual, direction, side, weight,
                                               allow, room)
        st["added"] += nadd
        if not first:
            st["added_d"] += nadd
        return fits

    kb = K.krylov_basis(VOPS, seed, applyH, tau, alloc.krylov, score, amp=amp,
                        state_seed=state_seed, recurrence=recurrence, fixed_depth=fixed_depth)
    capped = kb["capped"]
    if ranked:
        st["frame"], st["added"], fits = append_ranked(start_frame, cands, side,
                                                       alloc.krylov_rank, workcap)
        st["added_d"] = st["added"] if st["nd"] > 0 else 0
        capped = capped or not fits
    stats = dict(eta_c=st["eta_c"], eta_d=st["eta_d"], added=st["added"], n_h1=kb["n_h1"],
                 d_after_c=st["eta_c"] <= alloc.krylov and st["added_d"] > 0, capped=capped,
                 met=kb["closed"] and not capped)
    return st["frame"], stats


def record_krylov(ledger, st, alloc):
    ledger.max_krylov_c = max(ledger.max_krylov_c, st["eta_c"])
    ledger.max_krylov_d = max(ledger.max_krylov_d, st["eta_d"])
    ledger.max_krylov = max(ledger.max_krylov, st["eta_c"], st["eta_d"])
    ledger.n_krylov += st["added"]
    ledger.n_h1 += st["n_h1"]
    if st["eta_c"] <= alloc.krylov:
        ledger.n_c_pass += 1
    if st["d_after_c"]:
        ledger.n_d_after_c += 1
    if st["capped"]:
        ledger.workcap_reached = True
    if not st["met"]:
        ledger.unmet_("krylov")


# ── half-sweeps ──────────────────────────────────────────────────────────────────────────────


@dataclass
class Ctx:
    mpo: object
    tau: complex
    root_link: int
    alloc: object
    expansion: DDQRExpansion
    recurrence: str
    wcap: list
    rng: object
    eshift: float = 0.0  # the generators are H - eshift (shift_h, effective_operators.jl:110-129)
    parallel: bool = False  # parallel = true: right halves draw from a stream forked off `rng`
    exact: bool = False  # exact = true: DD expansions sketch the complete fused basis, no draws
    fold: bool = True  # fold_omega: frontier leaks sampled from folded closures, else exact
    keep_states: tuple = ()  # MPS the frames must contain (keep_states)
    keep_tols: tuple = ()  # per kept state: 0 contained exactly, > 0 admitted at that tolerance
    cap_keep: bool = False  # work_ceiling_rule = :bond: admitted states fill frames to the ceiling
    frontier_tol: float = 0.0  # > 0: each frontier compressed to its own rank before its sweep


def fork_rng(rng):
    """The right half-sweep's own stream under ``parallel = true``: a generator seeded by ONE 64-bit
    draw from ``rng`` (``MersenneTwister(rand(rng, UInt64))``, ``bug_step.jl:225`` and
    ``frontier_closure.jl:125``); here numpy's default generator seeded by ``rng.integers`` over the
    full unsigned 64-bit range."""
    seed = int(rng.integers(0, np.iinfo(np.uint64).max, dtype=np.uint64, endpoint=True))
    return np.random.default_rng(seed)


def shifted(y, x, s):
    """``(H - s) x`` from ``y = H x`` (``shift_h``); ``s = 0`` returns ``y`` itself."""
    return y if s == 0.0 else B.add(y, x, 1.0, -s)


@dataclass
class HalfAcc:
    nmv: int = 0
    peak: int = 0


def cap_at(wcap, bond):
    return wcap if isinstance(wcap, int) else wcap[bond - 1]


def expand(cx: Ctx, fr, bond, lch, rch, side, ledger):
    return dd_cbe_expand(fr, cx.mpo, bond, lch, rch, side, cx.alloc, ledger, cap_at(cx.wcap, bond),
                         cx.rng, fixed_width=cx.expansion.fixed_width,
                         tail_factor=cx.expansion.tail_factor, mode=cx.expansion.mode,
                         holdout_width=cx.expansion.holdout_width,
                         batch_blocks=cx.expansion.batch_blocks,
                         cap_selection=cx.expansion.cap_selection,
                         acceptance_factor=cx.expansion.acceptance_factor, exact=cx.exact)


UNION_KEEP = 0.5  # ``_UNION_KEEP`` (half_sweeps.jl:127)


def union_fresh(frame, cand, side, tol=0.0, room=None):
    """``_union_fresh`` (``half_sweeps.jl:143-176``): orthonormal directions of ``cand`` outside
    ``frame`` that survive a second projection, at most ``room`` of them (the strongest), or
    ``None``. ``tol = 0`` admits every direction above the numerical floor (``cand`` is contained
    exactly); ``tol > 0`` only those carrying more than about ``tol |cand|``."""
    if room is not None and room <= 0:
        return None
    left = side == "left"
    perp = perp_left if left else perp_right
    legs = (0, 1) if left else (1, 2)

    def orient(U):
        return U if left else rows_from_u(U)

    res = perp(frame, cand)
    nres, ncand = B.norm(res), B.norm(cand)
    if nres <= CBE_EPS * max(ncand, 1.0) or nres <= tol * ncand:
        return None
    first_cut = max(rank_cut(0.0, ncand, nres), tol * ncand / nres)
    basis = orient(B.svd(B.scale(res, 1.0 / nres), legs, cutoff=first_cut).U)
    res = perp(frame, basis)
    fac = B.svd(res, legs, cutoff=1e-13)
    smax = max((sv for sv, *_ in fac.kept), default=0.0)
    if smax < UNION_KEEP:
        return None
    return orient(B.svd(res, legs, cutoff=UNION_KEEP / smax, nkeep=room).U)


def union_kept(frame, cands, side, cx: Ctx, bond):
    """Every kept state's carried site tensor unioned into ``frame`` in turn (``_union_left`` /
    ``_union_right``, ``half_sweeps.jl:184-204``, the loops at ``:281-297`` and ``:385-398``);
    under the per-bond ceiling a tolerance-admitted state fills the frame only up to the bond's
    work ceiling (``_keep_room``, ``:179-181``)."""
    fl = 2 if side == "left" else 0
    for cand, tol in zip(cands, cx.keep_tols):
        room = cap_at(cx.wcap, bond) - frame.dim(fl) if cx.cap_keep and tol > 0 else None
        fresh = union_fresh(frame, cand, side, tol, room)
        if fresh is not None:
            frame = B.oplus([frame, fresh], fl)
    return frame


def half_left(psiL, left_frames, expanded, nn, acc, hledger, cx: Ctx):
    mpo, root = cx.mpo, cx.root_link
    canonical(psiL, 1)
    rstack = right_env_stack(psiL, mpo, downto=3)
    lch = left_boundary()
    lroot = lch
    carry = None
    kcar = [None] * len(cx.keep_states)  # each kept state's carry (b_i, link)
    for bond in range(1, root + 1):
        carried = psiL[bond] if carry is None else B.contract(carry, (1,), psiL[bond], (0,))
        fr = frame_from(carried, psiL[bond + 1])
        bl = Ledger()
        ex = expand(cx, fr, bond, lch, rstack[bond + 2], "left", bl)
        nn[bond - 1] = ex.n_new_l
        rp = B.contract(psiL[bond + 1], (1, 2), ex.V_ex, (1, 2), conjb=True)
        Kex = B.contract(carried, (2,), rp, (0,))
        rch1 = right_step(rstack[bond + 2], ex.V_ex, mpo[bond + 1])
        W = mpo[bond]

        def applyH(v, lch=lch, W=W, rch1=rch1):
            acc.nmv += 1
            return shifted(apply_one_site(lch, W, rch1, v), v, cx.eshift)

        Wk, st = krylov_enrich(Kex, applyH, ex.U_ex, "left", cx.tau, cx.alloc,
                               workcap=cap_at(cx.wcap, bond), recurrence=cx.recurrence,
                               fixed_depth=cx.expansion.krylov_fixed_depth)
        record_krylov(bl, st, cx.alloc)
        if cx.keep_states:
            kx = [k[bond] if c is None else B.contract(c, (1,), k[bond], (0,))
                  for k, c in zip(cx.keep_states, kcar)]
            Wk = union_kept(Wk, kx, "left", cx, bond)
            kcar = [B.contract(Wk, (0, 1), x, (0, 1), conja=True) for x in kx]
        left_frames[bond] = Wk
        expanded[bond - 1] = Wk.dim(2)
        log_bond(hledger, bl, bond, "left", expanded[bond - 1])
        carry = B.contract(Wk, (0, 1), carried, (0, 1), conja=True)
        if bond == root:
            lroot = lch
        if bond < root:
            lch = left_step(lch, Wk, mpo[bond])
    return lroot


def half_right(psiR, right_frames, expanded, nn, acc, hledger, cx: Ctx):
    mpo, root = cx.mpo, cx.root_link
    L = len(psiR)
    canonical(psiR, L)
    lstack = left_env_stack(psiR, mpo, upto=L - 2)
    rch = right_boundary(total_charge(psiR))
    rroot = rch
    carry = None
    kcar = [None] * len(cx.keep_states)  # each kept state's carry (link, b_j)
    for bond in range(L - 1, root - 1, -1):
        carried = psiR[bond + 1] if carry is None else B.contract(psiR[bond + 1], (2,), carry, (0,))
        fr = frame_from(psiR[bond], carried)
        bl = Ledger()
        ex = expand(cx, fr, bond, lstack[bond], rch, "right", bl)
        nn[bond - 1] = ex.n_new_r
        lp = B.contract(ex.U_ex, (0, 1), psiR[bond], (0, 1), conja=True)
        Bex = B.contract(lp, (1,), carried, (0,))
        lch1 = left_step(lstack[bond], ex.U_ex, mpo[bond])
        W = mpo[bond + 1]

        def applyH(v, lch1=lch1, W=W, rch=rch):
            acc.nmv += 1
            return shifted(apply_one_site(lch1, W, rch, v), v, cx.eshift)

        Zk, st = krylov_enrich(Bex, applyH, ex.V_ex, "right", cx.tau, cx.alloc,
                               workcap=cap_at(cx.wcap, bond), recurrence=cx.recurrence,
                               fixed_depth=cx.expansion.krylov_fixed_depth)
        record_krylov(bl, st, cx.alloc)
        if cx.keep_states:
            kx = [k[bond + 1] if c is None else B.contract(k[bond + 1], (2,), c, (0,))
                  for k, c in zip(cx.keep_states, kcar)]
            Zk = union_kept(Zk, kx, "right", cx, bond)
            kcar = [B.contract(x, (1, 2), Zk, (1, 2), conjb=True) for x in kx]
        right_frames[bond] = Zk
        if bond != root:
            expanded[bond - 1] = Zk.dim(0)
        log_bond(hledger, bl, bond, "right", Zk.dim(0))
        carry = B.contract(carried, (1, 2), Zk, (1, 2), conjb=True)
        if bond == root:
            rroot = rch
        if bond > root:
            rch = right_step(rch, Zk, mpo[bond + 1])
    return rroot, carry


# ── overlaps and projections ─────────────────────────────────────────────────────────────────


def overlap_left(psi, left_frames, root):
    AL = None
    for site in range(1, root + 1):
        carried = psi[site] if AL is None else B.contract(AL, (1,), psi[site], (0,))
        AL = B.contract(left_frames[site], (0, 1), carried, (0, 1), conja=True)
    return AL


def overlap_right(psi, right_frames, root):
    AR = None
    for bond in range(len(psi) - 1, root - 1, -1):
        carried = psi[bond + 1] if AR is None else B.contract(psi[bond + 1], (2,), AR, (0,))
        AR = B.contract(carried, (1, 2), right_frames[bond], (1, 2), conjb=True)
    return AR


def projection_miss(psi, left_frames, right_frames, root):
    L = len(psi)
    rf = [None] * (L + 2)
    for site in range(L, 1, -1):
        carried = psi[L] if site == L else B.contract(psi[site], (2,), rf[site + 1], (0,))
        res = B.svd(carried, (0,), cutoff=0.0)
        rf[site] = res.US()
    miss2 = 0.0
    AL = None
    for site in range(1, root + 1):
        carried = psi[site] if AL is None else B.contract(AL, (1,), psi[site], (0,))
        outside = perp_left(left_frames[site], carried)
        miss2 += B.norm(B.contract(outside, (2,), rf[site + 1], (0,))) ** 2
        AL = B.contract(left_frames[site], (0, 1), carried, (0, 1), conja=True)
    lf = [None] * (L + 1)
    res = B.svd(AL, (0,), cutoff=0.0)
    lf[root] = res.SVd()
    for bond in range(root + 1, L):
        res = B.svd(B.contract(lf[bond - 1], (1,), psi[bond], (0,)), (0, 1), cutoff=0.0)
        lf[bond] = res.SVd()
    AR = None
    for bond in range(L - 1, root - 1, -1):
        carried = psi[bond + 1] if AR is None else B.contract(psi[bond + 1], (2,), AR, (0,))
        outside = perp_right(right_frames[bond], carried)
        miss2 += B.norm(B.contract(lf[bond], (1,), outside, (0,))) ** 2
        AR = B.contract(carried, (1, 2), right_frames[bond], (1, 2), conjb=True)
    return math.sqrt(miss2)


# ── the order-p closure (single pass) ────────────────────────────────────────────────────────


@dataclass
class KLFrames:
    left_frames: dict
    right_frames: dict
    root_link: int
    lenv: object
    renv: object
    gen: int = 0
    eshift: float = 0.0


def root_generator(mpo, fr: KLFrames):
    """``B = P H P - eshift`` at the root (``_root_generator``, ``krylov_closure_frames.jl:291-303``)."""
    return ZeroSiteH(mpo, fr.root_link, fr.lenv, fr.renv, fr.left_frames[fr.root_link],
                     fr.right_frames[fr.root_link], eshift=fr.eshift)


def project_root(psi, fr: KLFrames):
    return B.contract(overlap_left(psi, fr.left_frames, fr.root_link), (1,),
                      overlap_right(psi, fr.right_frames, fr.root_link), (0,))


def frontier_mps(psi, fr: KLFrames, core):
    from .models import MPS

    L, root = len(psi), fr.root_link
    ts = [fr.left_frames[s] for s in range(1, root)]
    ts.append(B.contract(fr.left_frames[root], (2,), core, (0,)))
    ts += [fr.right_frames[b] for b in range(root, L)]
    return MPS(ts, root)


def bond_action(fr2: BondFrame, mpo, bond, lch, rch, side, rng, fold=True):
    """``_bond_action`` (``krylov_frontier_bonds.jl:80-100``): with ``fold = true`` the sampled
    leak of the folded closures, with ``fold = false`` the exact leak of the formed two-site
    action (one two-site application, no draws)."""
    if not fold:
        return exact_leak(fr2, mpo, bond, lch, rch, side)
    skl, skr = folded_closures(fr2, mpo, bond, lch, rch)
    grown = fr2.U0.dim(2) if side == "left" else fr2.V0.dim(0)
    count = max(8, -(-grown // 4))
    return sampled_leak(fr2, skl, skr, side, count, rng)


def frontier_left(Fm, mpo, fr: KLFrames, cx: Ctx, amp, enrich, gen):
    root, L = fr.root_link, len(Fm)
    canonical(Fm, 1)
    rstack = right_env_stack(Fm, mpo, downto=3)
    lch = left_boundary()
    lenv = lch
    carry = Pm = None
    Wn = {}
    lg = Ledger()
    leak = [0.0] * (root + 1)
    out = dict(added=0, nskip=0, n_h1=0, n_h2=0)
    if not enrich:
        chain = {}
        ch = left_boundary()
        for bond in range(1, root + 1):
            chain[bond] = ch
            if bond < root:
                ch = left_step(ch, fr.left_frames[bond], mpo[bond])
    for bond in range(1, root + 1):
        if not enrich:
            lch = chain[bond]
        old = fr.left_frames[bond] if Pm is None else B.contract(Pm, (1,), fr.left_frames[bond], (0,))
        site_core = Fm[bond] if carry is None else B.contract(carry, (1,), Fm[bond], (0,))
        tsf = frame_onto_left(old, site_core, Fm[bond + 1])
        rch = rstack[bond + 2]
        leak[bond] = bond_action(tsf, mpo, bond, lch, rch, "left", cx.rng, cx.fold)
        out["n_h2"] += 0 if cx.fold else 1
        bl = Ledger()
        quiet = indicator(cx.alloc, leak[bond]) <= cx.alloc.per_bond
        if enrich and not quiet:
            ex = expand(cx, tsf, bond, lch, rch, "left", bl)
            rp = B.contract(Fm[bond + 1], (1, 2), ex.V_ex, (1, 2), conjb=True)
            Kex = B.contract(site_core, (2,), rp, (0,))
            rch1 = right_step(rch, ex.V_ex, mpo[bond + 1])
            W = mpo[bond]

            def applyH(v, lch=lch, W=W, rch1=rch1):
                out["n_h1"] += 1
                return shifted(apply_one_site(lch, W, rch1, v), v, cx.eshift)

            Wi, st = krylov_enrich(Kex, applyH, ex.U_ex, "left", cx.tau, cx.alloc,
                                   workcap=cap_at(cx.wcap, bond), amp=amp, state_seed=False,
                                   recurrence=cx.recurrence,
                                   fixed_depth=cx.expansion.krylov_fixed_depth)
            record_krylov(bl, st, cx.alloc)
        else:
            out["nskip"] += 1
            Wi = old
        Wn[bond] = polar_frame(Wi, "left") if enrich else old
        out["added"] += Wn[bond].dim(2) - old.dim(2)
        log_bond(lg, bl, bond, "left", Wn[bond].dim(2))
        if enrich:
            Pm = B.contract(Wn[bond], (0, 1), old, (0, 1), conja=True)
        carry = B.contract(Wn[bond], (0, 1), site_core, (0, 1), conja=True)
        if bond == root:
            lenv = lch
        if enrich and bond < root:
            lch = left_step(lch, Wn[bond], mpo[bond])
    return dict(frames=Wn, env=lenv, ledger=lg, leak=leak[1:], added=out["added"],
                n_h1=out["n_h1"], n_h2=out["n_h2"])


def frontier_right(Fm, mpo, fr: KLFrames, cx: Ctx, amp, enrich, gen):
    root, L = fr.root_link, len(Fm)
    canonical(Fm, L)
    lstack = left_env_stack(Fm, mpo, upto=L - 2)
    rch = right_boundary(total_charge(Fm))
    renv = rch
    carry = Pm = None
    Zn = {}
    lg = Ledger()
    leak = [0.0] * L
    out = dict(added=0, nskip=0, n_h1=0, n_h2=0)
    if not enrich:
        chain = {}
        ch = right_boundary(total_charge(Fm))
        for bond in range(L - 1, root - 1, -1):
            chain[bond] = ch
            if bond > root:
                ch = right_step(ch, fr.right_frames[bond], mpo[bond + 1])
    for bond in range(L - 1, root - 1, -1):
        if not enrich:
            rch = chain[bond]
        old = fr.right_frames[bond] if Pm is None else B.contract(fr.right_frames[bond], (2,), Pm, (0,))
        site_core = Fm[bond + 1] if carry is None else B.contract(Fm[bond + 1], (2,), carry, (0,))
        tsf = frame_onto_right(Fm[bond], site_core, old)
        lch = lstack[bond]
        leak[bond] = bond_action(tsf, mpo, bond, lch, rch, "right", cx.rng, cx.fold)
        out["n_h2"] += 0 if cx.fold else 1
        bl = Ledger()
        quiet = indicator(cx.alloc, leak[bond]) <= cx.alloc.per_bond
        if enrich and not quiet:
            ex = expand(cx, tsf, bond, lch, rch, "right", bl)
            lp = B.contract(ex.U_ex, (0, 1), Fm[bond], (0, 1), conja=True)
            Bex = B.contract(lp, (1,), site_core, (0,))
            lch1 = left_step(lch, ex.U_ex, mpo[bond])
            W = mpo[bond + 1]

            def applyH(v, lch1=lch1, W=W, rch=rch):
                out["n_h1"] += 1
                return shifted(apply_one_site(lch1, W, rch, v), v, cx.eshift)

            Zj, st = krylov_enrich(Bex, applyH, ex.V_ex, "right", cx.tau, cx.alloc,
                                   workcap=cap_at(cx.wcap, bond), amp=amp, state_seed=False,
                                   recurrence=cx.recurrence,
                                   fixed_depth=cx.expansion.krylov_fixed_depth)
            record_krylov(bl, st, cx.alloc)
        else:
            out["nskip"] += 1
            Zj = old
        Zn[bond] = polar_frame(Zj, "right") if enrich else old
        out["added"] += Zn[bond].dim(0) - old.dim(0)
        log_bond(lg, bl, bond, "right", Zn[bond].dim(0))
        if enrich:
            Pm = B.contract(old, (1, 2), Zn[bond], (1, 2), conjb=True)
        carry = B.contract(site_core, (1, 2), Zn[bond], (1, 2), conjb=True)
        if bond == root:
            renv = rch
        if enrich and bond > root:
            rch = right_step(rch, Zn[bond], mpo[bond + 1])
    return dict(frames=Zn, env=renv, ledger=lg, leak=[leak[b] for b in range(root, L)],
                added=out["added"], n_h1=out["n_h1"], n_h2=out["n_h2"])


def frontier_sweep(fr: KLFrames, psi, mpo, core, degree, cx: Ctx, nrm, enrich=True):
    nF = B.norm(core)
    if nF <= FRONTIER_FLOOR * max(nrm, K.np.finfo(float).eps):
        return dict(added=0, leak=0.0, met=True, capped=False, ledger=Ledger())
    Fm = frontier_mps(psi, fr, core)
    if cx.frontier_tol > 0:
        # frontier_tol > 0 (frontier_closure.jl:102-120): the frontier, written in the frames with
        # frame-wide bonds, is compressed to its own rank at that weight tolerance (no rank cap:
        # the widest frame); its Schmidt vectors stay in the frames' span
        L = len(Fm)
        width = max(max(fr.left_frames[b].dim(2) for b in range(1, fr.root_link + 1)),
                    max(fr.right_frames[b].dim(0) for b in range(fr.root_link, L)))
        truncate_recursive(Fm, fr.root_link, width, cx.frontier_tol, [0.0] * (L - 1))
    FmR = Fm.copy()
    gen = fr.gen + 1
    amp = nF / max(nrm, np.finfo(float).eps)
    # parallel: the right half draws from its own stream, forked here (frontier_closure.jl:125-145);
    # the halves are independent, so running them one after the other gives the concurrent result
    cxR = replace(cx, rng=fork_rng(cx.rng)) if cx.parallel else cx
    rl = frontier_left(Fm, mpo, fr, cx, amp, enrich, gen)
    rr = frontier_right(FmR, mpo, fr, cxR, amp, enrich, gen)
    lg = Ledger()
    lg.merge(rl["ledger"])
    lg.merge(rr["ledger"])
    lL = math.sqrt(sum(x * x for x in rl["leak"]))
    lR = math.sqrt(sum(x * x for x in rr["leak"]))
    leak = indicator(cx.alloc, math.sqrt(lL * lL + lR * lR))
    if enrich:
        met = lg.tolerance_met
    else:
        met = all(indicator(cx.alloc, x) <= cx.alloc.per_bond for x in rl["leak"] + rr["leak"])
    added = rl["added"] + rr["added"]
    if enrich and added > 0:
        for b in range(1, fr.root_link + 1):
            fr.left_frames[b] = rl["frames"][b]
        for b in range(fr.root_link, len(psi)):
            fr.right_frames[b] = rr["frames"][b]
        fr.lenv, fr.renv, fr.gen = rl["env"], rr["env"], gen
    lg.n_closure_sweeps = 1
    lg.n_h1_closure = rl["n_h1"] + rr["n_h1"]
    lg.n_h2_leak = rl["n_h2"] + rr["n_h2"]
    return dict(added=added, leak=leak, met=met, capped=enrich and lg.workcap_reached, ledger=lg,
                leaks_left=rl["leak"], leaks_right=rr["leak"])


def single_pass_closure(fr: KLFrames, psi, mpo, root_start, cx: Ctx, order, nrm, ledger):
    lg = Ledger(order=order)
    state = dict(nroot=0, root=root_start, op=root_generator(mpo, fr))

    def applyB(v):
        state["nroot"] += 1
        return state["op"].apply(v)

    leak = [float("nan")] * order
    met = True
    for degree in range(1, order):
        F = state["root"]
        for d in range(1, degree + 1):
            F = B.scale(applyB(F), cx.tau / d)
        sr = frontier_sweep(fr, psi, mpo, F, degree, cx, nrm, enrich=True)
        lg.merge(sr["ledger"])
        leak[degree] = sr["leak"]
        met &= sr["met"]
        if sr["added"] > 0:
            state["op"] = root_generator(mpo, fr)
            state["root"] = project_root(psi, fr)
    lg.n_passes = 1
    lg.leak = leak
    lg.defect = sum(leak[d] / (d + 1) for d in range(order) if not math.isnan(leak[d]))
    lg.n_root_frontier = state["nroot"]
    if not met:
        lg.unmet_("closure")
    ledger.merge(lg)
    return dict(root_start=state["root"], n_h1=lg.n_h1_closure, n_root=state["nroot"])


def projected_frontiers(applyB, root, tau, count):
    """``_projected_frontiers`` (``krylov_closure_frames.jl:315-323``): ``F_j = (tau / j) B F_{j-1}``."""
    out, F = [], root
    for d in range(1, count + 1):
        F = B.scale(applyB(F), tau / d)
        out.append(F)
    return out


def closure_loop(frontier, sweep, order, maxpass, include_zero=False):
    """``_closure_loop!`` (``frontier_closure.jl:370-409``): pass 1 sweeps the initial degrees,
    later passes ``1..order-1``; converged when a pass adds nothing and meets every share; a pass
    with a share unmet and a sweep at the work ceiling stops capped."""
    later = list(range(1, order))
    initial = list(range(order)) if include_zero else later
    if not initial:
        return dict(passes=0, converged=True, exhausted=False, capped=False)
    ok0 = True
    for p in range(1, maxpass + 1):
        grew, allmet, capped = False, True, False
        for degree in (initial if p == 1 else later):
            r = sweep(frontier(degree), degree, p)
            grew |= r["added"] > 0
            allmet &= r["met"]
            capped |= r["capped"]
            if degree == 0:
                ok0 = r["met"]
        if not grew or not later:
            return dict(passes=p, converged=allmet and ok0, exhausted=False, capped=False)
        if capped and not allmet:
            return dict(passes=p, converged=False, exhausted=False, capped=True)
    return dict(passes=maxpass, converged=False, exhausted=True, capped=False)


def measure_frontiers(fr: KLFrames, psi, mpo, root_start, cx: Ctx, count, nrm):
    """``_measure_frontiers`` (``frontier_closure.jl:289-359``, serial): frontiers 0..count-1 of
    the root generator, each swept without enrichment on the frames as they stand; their leaks
    and scale-free ``||(I - P) A F_j|| / ||F_j||`` go to the ledger's ``leak_initial`` /
    ``rho_initial``. The frames are not touched."""
    state = dict(nroot=0)
    op = root_generator(mpo, fr)

    def applyB(v):
        state["nroot"] += 1
        return op.apply(v)

    cores = [root_start]
    if count > 1:
        cores += projected_frontiers(applyB, root_start, cx.tau, count - 1)
    lg = Ledger()
    leak, rho, met, met0 = [0.0] * count, [0.0] * count, True, True
    for d, core in enumerate(cores):
        sw = frontier_sweep(fr, psi, mpo, core, d, cx, nrm, enrich=False)
        lg.merge(sw["ledger"])
        nF = B.norm(core)
        raw = math.sqrt(sum(x * x for x in sw.get("leaks_left", ())) +
                        sum(x * x for x in sw.get("leaks_right", ())))
        leak[d] = sw["leak"]
        rho[d] = raw / nF if nF > 0 else 0.0
        if d >= 1:
            met &= sw["met"]
        else:
            met0 = sw["met"]
    lg.leak_initial, lg.rho_initial = leak, rho
    lg.n_root_frontier = state["nroot"]
    return dict(leak=leak, rho=rho, met=met, met0=met0, ledger=lg, n_root=state["nroot"])


def checked_closure(fr: KLFrames, psi, mpo, root_start, cx: Ctx, order, nrm, ledger):
    """``_krylov_closure!`` with ``checks = true`` (``krylov_closure_loop.jl:18-194``, serial,
    ``include_zero = false``): measure every frontier on the incoming frames first
    (``_measure_frontiers``, ``frontier_closure.jl:289-359``) and leave them untouched if all
    close; otherwise run the closure loop and measure degree 0 on the final frames."""
    lg = Ledger(order=order)
    state = dict(nroot=0, root=root_start, op=root_generator(mpo, fr))

    def applyB(v):
        state["nroot"] += 1
        return state["op"].apply(v)

    # the frontiers measured on the incoming frames (leak_initial / rho_initial)
    probe = measure_frontiers(fr, psi, mpo, root_start, cx, order, nrm)
    state["nroot"] += probe["n_root"]
    probe["ledger"].n_root_frontier = 0  # counted once, with the closure's, below
    lg.merge(probe["ledger"])
    final_leak = dict(enumerate(probe["leak"]))
    met, met0 = probe["met"], probe["met0"]
    gen0 = fr.gen
    if met:
        res = dict(passes=0, converged=True)
    else:
        state["op"] = root_generator(mpo, fr)

        def frontier(degree):
            if degree == 0:
                return state["root"]
            return projected_frontiers(applyB, state["root"], cx.tau, degree)[degree - 1]

        def sweep(F, degree, pass_):
            sw = frontier_sweep(fr, psi, mpo, F, degree, cx, nrm, enrich=True)
            lg.merge(sw["ledger"])
            final_leak[degree] = sw["leak"]
            if sw["added"] > 0:
                state["op"] = root_generator(mpo, fr)
                state["root"] = project_root(psi, fr)
            return sw

        res = closure_loop(frontier, sweep, order, closure_maxpass(order))
        if fr.gen != gen0:
            sw = frontier_sweep(fr, psi, mpo, frontier(0), 0, cx, nrm, enrich=False)
            lg.merge(sw["ledger"])
            final_leak[0] = sw["leak"]
    lg.n_passes = res["passes"]
    lg.leak = [final_leak[d] for d in range(order)]
    lg.defect = sum(lg.leak[d] / (d + 1) for d in range(order))
    lg.n_root_frontier = state["nroot"]
    if not res["converged"]:
        lg.unmet_("closure")
    ledger.merge(lg)
    return dict(root_start=state["root"], n_h1=lg.n_h1_closure, n_root=state["nroot"])


# ── compression ──────────────────────────────────────────────────────────────────────────────


def cut_divisor(L, root):
    return math.sqrt(root - 1) + math.sqrt(L - root)


def budget_svd(tensor, split, maxdim, share_of):
    res = B.svd(tensor, split, cutoff=0.0, nkeep=maxdim)
    share = share_of(B.sq_weight(res.kept) + B.sq_weight(res.trunc))
    nk = len(res.kept)
    keep, tail = tail_rank(res.kept, 1.0, share, nk, base=B.sq_weight(res.trunc))
    capped = tail > share and len(res.trunc) > 0
    keep = max(keep, 1)
    if keep < nk:
        res = B.svd(tensor, split, cutoff=0.0, nkeep=keep)
    return res, capped


def truncate_recursive(psi, root, maxdim, weight_tol, bond_weights):
    L = len(psi)
    st = dict(worst=0.0, nrm2=-1.0, capped=False)
    cum = [0.0, 0.0]
    sdiv = cut_divisor(L, root)

    def share_of(total):
        if st["nrm2"] < 0:
            st["nrm2"] = total
        return weight_tol * math.sqrt(max(st["nrm2"], 0.0)) / sdiv if sdiv > 0 else 0.0

    def cut(t, split):
        res, cc = budget_svd(t, split, maxdim, share_of)
        st["capped"] |= cc
        return res

    def account(res, side, bond):
        st["worst"] = max(st["worst"], B.trunc_weight(res))
        cum[side] += B.sq_weight(res.trunc)
        bond_weights[bond - 1] = B.sq_weight(res.trunc)
        if st["nrm2"] < 0:
            st["nrm2"] = B.sq_weight(res.kept) + B.sq_weight(res.trunc)

    for site in range(root, 1, -1):
        res = cut(psi[site], (0,))
        account(res, 0, site - 1)
        psi[site] = res.Vd
        psi[site - 1] = B.contract(psi[site - 1], (2,), res.US(), (0,))
        psi.center = site - 1
    canonical(psi, root)
    for site in range(root, L):
        res = cut(psi[site], (0, 1))
        account(res, 1, site)
        psi[site] = res.U
        psi[site + 1] = B.contract(res.SVd(), (1,), psi[site + 1], (0,))
        psi.center = site + 1
    nrm2 = st["nrm2"]
    cumulative = (math.sqrt(cum[0]) + math.sqrt(cum[1])) / math.sqrt(nrm2) if nrm2 > 0 else 0.0
    for i in range(len(bond_weights)):
        bond_weights[i] = math.sqrt(bond_weights[i] / nrm2) if nrm2 > 0 else 0.0
    return st["worst"], cumulative, st["capped"]


def assemble_and_compress(psi, left_frames, right_frames, root, res, ledger, bwts, bd0, maxdim,
                          tol_trunc, truncate):
    L = len(psi)
    discarded = B.trunc_weight(res)
    for site in range(1, root):
        psi[site] = left_frames[site]
    psi[root] = B.contract(left_frames[root], (2,), res.U, (0,))
    psi[root + 1] = B.contract(res.SVd(), (1,), right_frames[root], (0,))
    for bond in range(root + 1, L):
        psi[bond + 1] = right_frames[bond]
    psi.center = root + 1
    root_rank = psi[root].dim(2)
    if truncate:
        wtr, cumw, capped = truncate_recursive(psi, root + 1, maxdim, tol_trunc, bwts)
        discarded = max(discarded, wtr)
        ledger.n_compress += 1
        ledger.discarded = cumw
        ledger.maxdim_reached = capped
        if cumw > tol_trunc * (1 + 1e-8):
            ledger.unmet_("trunc")
    bd1 = psi.bond_dims()
    ledger.r_final = max(bd1) if bd1 else 0
    for e in ledger.bond_log:
        e.update(r_old=bd0[e["bond"] - 1], r_final=bd1[e["bond"] - 1], discarded=bwts[e["bond"] - 1])
    return root_rank, discarded


# ── the step ─────────────────────────────────────────────────────────────────────────────────


def bug_root_link(L):
    return max(1, min(L - 1, L // 2))


def local_dim(psi):
    return max(psi[s].dim(1) for s in range(1, len(psi) + 1))


def closure_maxpass(order):
    return 2 * order + 2  # _closure_maxpass, krylov_closure_frames.jl:12


def complement_action(psi, mpo, fr: KLFrames, core, cx: Ctx):
    """``estimate_global_complement_action`` (``frontier_closure.jl:238-277``, ``nsample = 0``): the
    per-bond two-site misses of a non-enriching frontier sweep of ``core`` on the frames ``fr``,
    measured with a copy of the step's generator so its stream is left untouched."""
    rng = np.random.default_rng()
    rng.bit_generator.state = cx.rng.bit_generator.state
    L = len(psi)
    alloc = basis_allocation(Budget(1.0, 0.0, 1.0), L - 1)  # scale 1: raw norms
    mcx = Ctx(cx.mpo, 0j, cx.root_link, alloc, cx.expansion, cx.recurrence, cx.wcap, rng, cx.eshift)
    frames = KLFrames(dict(fr.left_frames), dict(fr.right_frames), fr.root_link, fr.lenv, fr.renv,
                      fr.gen, fr.eshift)
    sw = frontier_sweep(frames, psi, mpo, core, 0, mcx, max(B.norm(core), np.finfo(float).eps),
                        enrich=False)
    pl, pr = sw.get("leaks_left", []), sw.get("leaks_right", [])
    left = math.sqrt(sum(x * x for x in pl))
    right = math.sqrt(sum(x * x for x in pr))
    return dict(left=left, right=right, bound=math.sqrt(left * left + right * right),
                per_left=list(pl), per_right=list(pr))


def report_root(report, psi, mpo, left_frames, right_frames, root_link, lenv_root, renv_root,
                root_operator, root_start, root_result, solve_with, *, cx, nrm, ledger, expanded,
                outside_residual, tol_basis, order):
    """``_report_root!`` (``bug_step_stages.jl:243-390``): the Rayleigh-quotient energies before and
    after the root solve and, with ``outside_residual``, the defect ``|tau| ||(I - P) H psi_1|| /
    ||psi_1||``; while it fails ``tol_basis`` the frames are re-enriched by the evolved state's own
    frontier sweep and the root re-solved (at most ``2 order + 2`` passes)."""
    state = dict(op=root_operator, lenv=lenv_root, renv=renv_root, rep=None)

    def rayleigh(v):
        n2 = B.norm(v) ** 2
        if not n2 > 0:
            return float("nan")
        return B.inner(v, state["op"].apply(v)).real / n2 + cx.eshift

    def frames():
        return KLFrames(left_frames, right_frames, root_link, state["lenv"], state["renv"], 0, cx.eshift)

    def outside_of(v):
        return complement_action(psi, mpo, frames(), v, cx)

    def residual_of(action, v):
        if action is None:
            return float("nan")
        return abs(cx.tau) * action["bound"] / max(B.norm(v), np.finfo(float).eps)

    e_pre = rayleigh(root_start)
    outside = outside_of(root_result) if outside_residual else None
    initial = residual_of(outside, root_result)
    passes = added = 0
    if outside_residual:
        while not (residual_of(outside, root_result) <= tol_basis) and passes < closure_maxpass(order):
            fr = frames()
            passes += 1
            sw = frontier_sweep(fr, psi, mpo, root_result, 0, cx, nrm, enrich=True)
            ledger.merge(sw["ledger"])
            if sw["added"] == 0:
                break
            added += sw["added"]
            state["lenv"], state["renv"] = fr.lenv, fr.renv
            root_start = project_root(psi, fr)
            state["op"] = root_generator(mpo, fr)
            root_result, state["rep"] = solve_with(state["op"], root_start)
            outside = outside_of(root_result)
            if sw["capped"]:
                break
        if added > 0:
            L = len(psi)
            for b in range(1, root_link):
                expanded[b - 1] = left_frames[b].dim(2)
            for b in range(root_link + 1, L):
                expanded[b - 1] = right_frames[b].dim(0)
            ledger.r_aug = max(max(expanded, default=0), right_frames[root_link].dim(0))
    e_root = rayleigh(root_result)
    rn = max(B.norm(root_result), np.finfo(float).eps)
    nan = float("nan")
    report.update(
        eshift=cx.eshift, e_pre=e_pre, e_root=e_root, n_root=None, resid_initial=initial,
        outside_passes=passes, outside_added=added,
        outside=nan if outside is None else outside["bound"] / rn,
        outside_left=nan if outside is None else outside["left"] / rn,
        outside_right=nan if outside is None else outside["right"] / rn,
        per_left=[] if outside is None else [x / rn for x in outside["per_left"]],
        per_right=[] if outside is None else [x / rn for x in outside["per_right"]],
        resid=nan if outside is None else abs(cx.tau) * outside["bound"] / rn,
    )
    return dict(root_start=root_start, root_result=root_result, lenv=state["lenv"],
                renv=state["renv"], rep=state["rep"])


KLS_SCHEDULES = ("sequential", "kl_then_s", "concurrent")  # parallel_kls.jl:7


def step_options(L, mpo_len, root, parallel, kls, tol_expv, tol_root, order, work_ceiling_rule,
                 bond_ceiling_factor, root_ceiling_factor, frontier_tol, krylov_rank_tol,
                 closure_probe, keep_states, keep_tols, frames_only, frames_report, exact,
                 root_report, truncate, outside_residual):
    """``_step_options`` (``bug_step_stages.jl:40-142``): the reference's refusals (``ValueError``)
    in its order, then the options this restatement leaves out (``NotImplementedError``). Returns
    ``(root_link, tol_expv)``."""
    if mpo_len != L:
        raise ValueError(f"MPO has {mpo_len} sites, state has {L}")
    if L < 2:
        raise ValueError("cbe_bug_step needs at least two sites")
    root_link = bug_root_link(L) if root is None else root
    if not 1 <= root_link <= L - 1:
        raise ValueError(f"root must be a bond in 1:{L - 1}, got {root_link}")
    if isinstance(parallel, bool):
        mode, run_parallel = ("half_sweeps" if parallel else "serial"), parallel
    elif parallel in ("serial", "half_sweeps", "full"):
        mode, run_parallel = parallel, parallel != "serial"
    else:
        raise ValueError(f"parallel must be :serial, :half_sweeps, :full or a Bool, got {parallel!r}")
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
    if work_ceiling_rule not in ("maxdim", "bond", "bond_strict", "frame_root"):
        raise ValueError(f"work_ceiling_rule must be :maxdim, :bond, :bond_strict or :frame_root, "
                         f"got {work_ceiling_rule!r}")
    if not (bond_ceiling_factor == 0 or (bond_ceiling_factor > 1 and work_ceiling_rule != "maxdim")):
        raise ValueError("bond_ceiling_factor must be 0, or > 1 with work_ceiling_rule = bond")
    if not root_ceiling_factor > 1:
        raise ValueError("root_ceiling_factor must exceed one")
    frame_factor = 2.0 if bond_ceiling_factor == 0 else bond_ceiling_factor
    if work_ceiling_rule == "frame_root" and root_ceiling_factor > frame_factor:
        raise ValueError("root_ceiling_factor must not exceed frame factor")
    if closure_probe < 0:
        raise ValueError(f"closure_probe must be a non-negative count, got {closure_probe}")
    if len(keep_tols) and len(keep_tols) != len(keep_states):
        raise ValueError(f"keep_tols has {len(keep_tols)} entries for {len(keep_states)} keep_states")
    if any(t < 0 for t in keep_tols):
        raise ValueError(f"keep_tols must be >= 0, got {list(keep_tols)}")
    if frames_only and (root_report is not None or kls is not None or truncate):
        raise ValueError("frames_only needs root_report = nothing, kls = nothing and truncate = false")
    if kls is not None and kls not in KLS_SCHEDULES:
        raise ValueError(f"the K/L/S schedule must be one of {KLS_SCHEDULES}, got {kls!r}")
    if kls is not None and outside_residual:
        raise ValueError("the parallel K/L/S step does not combine with the outside-residual "
                         "re-enrichment")
    if kls is not None:
        raise NotImplementedError("the parallel K/L/S step (parallel = :full, kls) is not restated")
    if work_ceiling_rule == "bond_strict" and not bond_ceiling_factor > 1:
        raise ValueError("strict bond factor must exceed 1")
    return root_link, tol_expv


def cbe_bug_step(psi, mpo, tau, *, tol_basis=None, tol_trunc=None, tol_expv=None, tol_root=None,
                 tol_krylov=None, order=1, closure_probe=0, maxdim=None, hermitian=True,
                 expansion=None, rng=None, root=None, reorth=True, truncate=True,
                 work_ceiling_rule="bond", bond_ceiling_factor=None, root_ceiling_factor=1.2,
                 root_maxiter=K.ROOT_MAXITER, krylov_rank_tol=0.0, frontier_tol=0.0,
                 fold_omega=None, closure_checks=False, eshift=0.0, root_report=None,
                 outside_residual=False, root_method="exp", root_shift=True, frames_report=None,
                 keep_states=(), keep_tols=(), frames_only=False, exact=False, parallel=False,
                 kls=None):
    """One rank-adaptive BUG step in place; returns the step info dict
    (``bug_step.jl:17-513``). The generators are ``H - eshift``; with ``root_report`` (a dict) the
    root's energies and, with ``outside_residual``, the outside-Galerkin defect and its
    re-enrichment are filled in (``_report_root!``, ``bug_step_stages.jl:243-390``)."""
    tau = complex(tau)
    L = len(psi)
    root_link, tol_expv = step_options(
        L, len(mpo), root, parallel, kls, tol_expv, tol_root, order, work_ceiling_rule,
        bond_ceiling_factor, root_ceiling_factor, frontier_tol, krylov_rank_tol, closure_probe,
        keep_states, keep_tols, frames_only, frames_report, exact, root_report, truncate,
        outside_residual)
    budget = Budget(TOL_DEFAULTS["basis"] if tol_basis is None else tol_basis,
                    TOL_DEFAULTS["trunc"] if tol_trunc is None else tol_trunc,
                    TOL_DEFAULTS["expv"] if tol_expv is None else tol_expv)
    if order < 1:
        raise ValueError(f"order must be >= 1, got {order}")
    if bond_ceiling_factor is None:
        bond_ceiling_factor = DEFAULT_BOND_CEILING_FACTOR if work_ceiling_rule == "bond" else 0.0
    # bug_step_stages.jl:67: the folded closures are the default above order 1 unless exact
    fold = (order > 1 and not exact) if fold_omega is None else bool(fold_omega)
    if outside_residual and root_report is None:
        raise ValueError("outside_residual needs root_report")
    if outside_residual and not fold:
        raise NotImplementedError("the outside residual with the exact (unfolded) leak is not restated")
    eshift = float(eshift)
    maxdim = 128 if maxdim is None else maxdim
    bond_ranks = psi.bond_dims()
    # the work ceilings from the bonds before the step (bug_step_stages.jl:114-129)
    if work_ceiling_rule == "bond":
        wcap = bond_work_ceilings(bond_ranks, local_dim(psi), maxdim, factor=bond_ceiling_factor)
    elif work_ceiling_rule == "bond_strict":
        wcap = bond_work_ceilings_strict(bond_ranks, maxdim, factor=bond_ceiling_factor)
    elif work_ceiling_rule == "frame_root":
        wcap = bond_frame_root_ceilings(
            bond_ranks, maxdim, root_link, root_factor=root_ceiling_factor,
            frame_factor=2.0 if bond_ceiling_factor == 0 else bond_ceiling_factor)
    else:
        wcap = work_ceiling(maxdim, max(bond_ranks, default=0), local_dim(psi))
    expansion = DDQRExpansion() if expansion is None else expansion
    recurrence = expansion.krylov_mode
    if recurrence not in ("auto", "lanczos", "arnoldi"):  # resolve_krylov_recurrence refuses it
        raise ValueError(f"krylov_mode must be :auto, :lanczos or :arnoldi, got {recurrence!r}")
    if recurrence == "auto":
        recurrence = "lanczos" if hermitian else "arnoldi"
    if rng is None:
        rng = np.random.default_rng(0x5EED)

    t0 = time.perf_counter()
    nrm = B.norm(psi[psi.center]) if 1 <= psi.center <= L else 1.0
    alloc = basis_allocation(budget, L - 1, tau=tau, nrm=nrm, nfront=order, rule="linear",
                             krylov=tol_krylov, krylov_rank=krylov_rank_tol)
    ledger = Ledger(order=order)
    bd0 = psi.bond_dims()
    ledger.r_old = max(bd0, default=0)
    bwts = [0.0] * (L - 1)
    expanded = [0] * (L - 1)
    nL = [0] * (L - 1)
    nR = [0] * (L - 1)
    accL, accR = HalfAcc(), HalfAcc()
    run_parallel = parallel is True or parallel == "half_sweeps"
    ktols = tuple(float(t) for t in keep_tols) if len(keep_tols) else (0.0,) * len(keep_states)
    cx = Ctx(mpo, tau, root_link, alloc, expansion, recurrence, wcap, rng, eshift, run_parallel,
             bool(exact), fold, tuple(keep_states), ktols, work_ceiling_rule != "maxdim",
             float(frontier_tol))
    # parallel = true: the right half-sweep's stream is forked off the step's before either half
    # runs (bug_step.jl:222-268)
    cxR = replace(cx, rng=fork_rng(rng)) if run_parallel else cx
    ledgerL, ledgerR = Ledger(), Ledger()
    left_frames, right_frames = {}, {}
    psiL = psi.copy()
    psiR = psi
    lenv_root = half_left(psiL, left_frames, expanded, nL, accL, ledgerL, cx)
    renv_root, AR = half_right(psiR, right_frames, expanded, nR, accR, ledgerR, cxR)
    ledger.merge(ledgerL)
    ledger.merge(ledgerR)
    n_new = nL[: root_link - 1] + nR[root_link - 1:]
    AL = overlap_left(psi, left_frames, root_link)
    root_start = B.contract(AL, (1,), AR, (0,))
    nclose = 0
    fr = KLFrames(left_frames, right_frames, root_link, lenv_root, renv_root, 0, eshift)
    if order > 1:
        closure = checked_closure if closure_checks else single_pass_closure
        cl = closure(fr, psi, mpo, root_start, cx, order, nrm, ledger)
        for b in range(1, root_link):
            expanded[b - 1] = left_frames[b].dim(2)
        for b in range(root_link + 1, L):
            expanded[b - 1] = right_frames[b].dim(0)
        lenv_root, renv_root, root_start = fr.lenv, fr.renv, cl["root_start"]
        nclose = cl["n_h1"] + cl["n_root"]
    elif closure_probe > 0:
        # a measurement only (bug_step_stages.jl:221-236): a copied generator and untouched
        # frames, so the step itself stays bit-identical
        probe = measure_frontiers(fr, psi, mpo, root_start, replace(cx, rng=copy.deepcopy(rng)),
                                  closure_probe, nrm)
        ledger.merge(probe["ledger"])
    npsi = B.norm(psi[psi.center])
    ledger.r_aug = max(max(expanded, default=0), right_frames[root_link].dim(0))
    ledger.proj_err = projection_miss(psi, left_frames, right_frames, root_link) / npsi if npsi > 0 else 0.0
    if ledger.proj_err > budget.basis:
        ledger.unmet_("projection")
    gen = ZeroSiteH(mpo, root_link, lenv_root, renv_root, left_frames[root_link],
                    right_frames[root_link], eshift=eshift)
    nroot = [0]

    def solve_with(op, start):
        def apply_root(v):
            nroot[0] += 1
            return op.apply(v)

        return K.expv(VOPS, apply_root, tau, start, hermitian=hermitian, maxiter=root_maxiter,
                      tol=1e-15, reorth=reorth, conv_tol=budget.expv, substeps=0,
                      root_method=root_method, rational_shift=root_shift)

    # frames_only: the caller solves its own root on these frames, so the start is carried
    # (bug_step.jl:381-382) and no expv report is read
    root_result, rep = (root_start, None) if frames_only else solve_with(gen, root_start)
    if root_report is not None:
        rr = report_root(root_report, psi, mpo, left_frames, right_frames, root_link, lenv_root,
                         renv_root, gen, root_start, root_result, solve_with, cx=cx, nrm=nrm,
                         ledger=ledger, expanded=expanded, outside_residual=outside_residual,
                         tol_basis=budget.basis, order=order)
        root_start, root_result = rr["root_start"], rr["root_result"]
        if rr["rep"] is not None:
            rep = rr["rep"]
    if rep is not None:
        ledger.expv_err = rep[2]
        ledger.expv_iters = rep[0]
        if rep[2] > budget.expv * (1 + 1e-8):
            ledger.unmet_("expv")
    if frames_report is not None:  # the KLFrames the step integrated in (bug_step.jl:455-467)
        frames_report.update(left_frames=dict(left_frames), right_frames=dict(right_frames),
                             root_link=root_link, lenv=lenv_root, renv=renv_root,
                             eshift=float(eshift))
    res = B.svd(root_result, (0,), cutoff=0.0)
    expanded[root_link - 1] = left_frames[root_link].dim(2)
    root_frame_width = right_frames[root_link].dim(0)
    root_rank, discarded = assemble_and_compress(psi, left_frames, right_frames, root_link, res,
                                                 ledger, bwts, bd0, maxdim, budget.trunc, truncate)
    return dict(
        expanded=expanded, n_new=n_new, root_link=root_link, root_rank=root_rank,
        err_pre=0.0, err_fnl=0.0, discarded=discarded,
        n_matvec=accL.nmv + accR.nmv + nroot[0] + nclose, root_frame_width=root_frame_width,
        ledger=ledger, status=ledger.status(), seconds=time.perf_counter() - t0,
        bond_dims=psi.bond_dims(), start_ranks=bd0, workcap=wcap,
        record=dict(policy="dd_qr_streamed", qr_backend="householder",
                    closure="dd_qr_streamed" if order > 1 else "none", order=order,
                    parallel_mode="half_sweeps" if run_parallel else "serial", r_old=max(bd0, default=0),
                    r_aug=max(max(expanded, default=0), root_frame_width),
                    r_final=max(psi.bond_dims(), default=0), maxdim=maxdim,
                    workcap=max(wcap) if isinstance(wcap, list) else wcap,
                    n_root=nroot[0], rule=alloc.rule),
    )
