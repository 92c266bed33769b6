"""DD-QR controlled bond expansion of the CPU oracle (``mode = :rank_tail``).

TEST INFRASTRUCTURE (see ``oracle/blocks.py``). Restates:

* ``perp_component`` / ``perp_component_right`` (``src/BUG/Core/TensorNetworks/sectors.jl:215-240``);
* ``_rank_cut`` (``src/BUG/Core/RankAdaptation/truncation.jl:194-195``), ``_reortho_left/right``
  (``:374-394``), ``_cap_to_local_room`` (``:332-351``), ``_frame_sector_dims`` (``:297-322``);
* ``_alloc_columns`` (``src/BUG/Randomised/cbe.jl:188-195``), ``_dd_probe`` (``dd_cbe.jl:132-161``),
  ``sector_graded_sketch(...; comp_ratio = nothing)`` (``sketch.jl:14-54``), ``_sample_residual``
  (``sketch.jl:141-180``), ``sampled_leak`` (``cbe.jl:355-391``), ``_fold_sketch_closures``
  (``cbe.jl:62-144``);
* ``dd_cbe_expand`` with its default ``tail_dd`` branch (``dd_cbe_expand.jl:19-301,383-419``),
  the incremental controller and the deterministic ``exact = true`` branch (the complete fused
  basis, ``_dd_probe(...; exact = true)``, and the one-pass certified range, ``:346-360``);
* ``_bond_action`` with ``fold = false``: the exact two-site leak (``krylov_frontier_bonds.jl:37-100``).

A right frame's bond leg is incoming; an SVD over ``(site, link_r)`` returns that leg outgoing, so
the orthonormal rows are re-expressed on an incoming leg (:func:`rows_from_u`) before they join a
right frame -- the U(1) label of a leg depends on its arrow (``sectors.jl:193-206``).
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import blocks as B
from .budget import ADAPTIVE_GROWTH, indicator
from .env import stream_left, stream_right

EPS = 2.220446049250313e-16
CBE_EPS = 100 * EPS
REORTH_KEEP = 1 / math.sqrt(2)


def perp_left(U: B.BT, K: B.BT) -> B.BT:
    """``K - U (U^dag K)`` over the ``(link, site)`` legs."""
    ov = B.contract(U, (0, 1), K, (0, 1), conja=True)
    proj = B.contract(U, (2,), ov, (0,))
    return B.sub(K, proj)


def perp_right(V: B.BT, K: B.BT) -> B.BT:
    """``K - (K V^dag) V`` over the ``(site, link)`` legs."""
    ov = B.contract(K, (1, 2), V, (1, 2), conjb=True)
    proj = B.contract(ov, (1,), V, (0,))
    return B.sub(K, proj)


def flip_leg(t: B.BT, leg: int) -> B.BT:
    """The same tensor on a leg of opposite arrow: labels negated, arrow reversed."""
    legs = list(t.legs)
    legs[leg] = B.Leg(-t.legs[leg].dir, {-q: d for q, d in t.legs[leg].sectors.items()})
    blocks = {}
    for k, v in t.blocks.items():
        k2 = list(k)
        k2[leg] = -k2[leg]
        blocks[tuple(k2)] = v
    return B.BT(legs, blocks)


def rows_from_u(U: B.BT) -> B.BT:
    """``U`` = (site, link, new:+1) of an SVD over a right frame's legs -> rows ``(new:-1, site,
    link)`` spanning the same space (``permutedims(U, (3, 1, 2))``)."""
    return flip_leg(B.permute(U, (2, 0, 1)), 0)


def rank_cut(stol: float, sketch_norm: float, outside_norm: float) -> float:
    return stol if stol > 0 else CBE_EPS * max(sketch_norm, outside_norm) / outside_norm


def reortho(frame, block, side):
    """``orth(perp(block))`` or ``None`` (``truncation.jl:374-394``)."""
    if block is None:
        return None
    perp = perp_left if side == "left" else perp_right
    outside = perp(frame, block)
    if B.norm(outside) <= CBE_EPS * max(B.norm(block), 1.0):
        return None
    if side == "left":
        return B.svd(outside, (0, 1), cutoff=1e-14).U
    return rows_from_u(B.svd(outside, (1, 2), cutoff=1e-14).U)


def fused_dims(frame, side):
    """``(dfull, dT)``: per charge of the frame's local space, its dimension and the frame's
    width there (``truncation.jl:297-322``)."""
    if side == "left":
        fs = B.fused_sectors(frame.legs[0], frame.legs[1], +1)
        la, lb, bl = frame.legs[0], frame.legs[1], frame.legs[2]
    else:
        fs = B.fused_sectors(frame.legs[1], frame.legs[2], -1)
        la, lb, bl = frame.legs[1], frame.legs[2], frame.legs[0]
    dfull = {c: sum(la.sectors[a] * lb.sectors[b] for a, b in pairs) for c, pairs in fs.items()}
    dT = {c: bl.sectors.get(c, 0) for c in dfull}
    for c, w in dT.items():
        if w > dfull[c]:
            raise RuntimeError(f"frame holds {w} directions in sector {c}, local space {dfull[c]}")
    return dfull, dT


def cap_to_local_room(frame, cand, side):
    if cand is None:
        return None
    fl = 2 if side == "left" else 0
    dfull, dT = fused_dims(frame, side)
    counts = {}
    over = False
    for c, lw in dfull.items():
        du = cand.legs[fl].sectors.get(c, 0)
        if du == 0:
            continue
        counts[c] = min(du, lw - dT[c])
        over |= counts[c] < du
    if not over:
        return cand
    return B.trim_per_sector(cand, fl, counts)


def alloc_columns(dims: dict, budget: int) -> dict:
    tot = sum(dims.values())
    if tot == 0 or budget <= 0:
        return {q: 0 for q in dims}
    return {q: min(d, math.ceil(d / tot * budget)) for q, d in dims.items()}


def boost_columns(cols: dict, boost: dict, cap: dict) -> dict:
    """``_boost!`` (``cbe.jl:206-216``): raise targeted sectors' columns, capped by ``cap``;
    returns what did not fit."""
    left = {}
    for q, extra in boost.items():
        if q not in cap:
            continue
        have = cols.get(q, 0)
        add = min(max(extra, 0), max(cap[q] - have, 0))
        cols[q] = have + add
        if extra > add:
            left[q] = extra - add
    return left


def dd_probe(opp, oside, width, rng, boost=None):
    """Sector-graded Gaussian probe in ``opp``'s discarded space (``dd_cbe.jl:132-161``)."""
    dfull, dT = fused_dims(opp, oside)
    dC = {c: max(dfull[c] - dT[c], 0) for c in dfull}
    if sum(dC.values()) == 0:
        return None
    cols = alloc_columns(dC, width)
    if boost:
        boost_columns(cols, boost, dC)
    if oside == "left":
        om = B.gaussian_fused(rng, opp.legs[0], opp.legs[1], cols, new_first=False)
    else:
        om = B.gaussian_fused(rng, opp.legs[1], opp.legs[2], cols, new_first=True)
    if om is None:
        return None
    projected = (perp_left if oside == "left" else perp_right)(opp, om)
    return projected if B.norm(projected) > 0 else None


def dd_probe_exact(opp, oside):
    """``_dd_probe(...; exact = true)`` (``dd_cbe.jl:140-161``): the complete fused basis of
    ``opp``'s two local legs with ``opp`` projected out; ``None`` when there is no discarded space
    or nothing survives the projection. Draws nothing."""
    dfull, dT = fused_dims(opp, oside)
    if sum(max(dfull[c] - dT[c], 0) for c in dfull) == 0:
        return None
    if oside == "left":
        om = B.identity_fused(opp.legs[0], opp.legs[1], new_first=False)
    else:
        om = B.identity_fused(opp.legs[1], opp.legs[2], new_first=True)
    if om is None:
        return None
    projected = (perp_left if oside == "left" else perp_right)(opp, om)
    return projected if B.norm(projected) > 0 else None


def graded_sketch(frame, side, npre, rng):
    """``sector_graded_sketch(frame, side, npre; comp_ratio = nothing)`` (``sketch.jl:14-54``)."""
    dfull, _ = fused_dims(frame, side)
    cols = alloc_columns(dfull, npre)
    if side == "left":
        r = B.gaussian_fused(rng, frame.legs[0], frame.legs[1], cols, new_first=False)
    else:
        r = B.gaussian_fused(rng, frame.legs[1], frame.legs[2], cols, new_first=True)
    if r is None:
        return None
    return r if B.norm(r) > 0 else None


def sample_residual(basis, project, sketch, Om, wleg, side):
    """Test B with ``nh = 1`` and fixed probe ``Om`` (``sketch.jl:141-180``):
    ``(est, per_sector, cols)``."""
    per, cols = {}, {}
    if Om is None:
        return 0.0, per, cols
    for q, d in Om.legs[wleg].sectors.items():
        if d > 0:
            cols[q] = d
    if not cols:
        return 0.0, per, cols
    sketched = sketch(Om)
    if sketched is None:
        return 0.0, per, cols
    residual = project(sketched)
    if B.norm(residual) <= CBE_EPS:
        return 0.0, per, cols
    if basis is not None:
        off = perp_left(basis, residual) if side == "left" else perp_right(basis, residual)
        residual = project(off)
    rleg = 2 if side == "left" else 0
    for q, d in residual.legs[rleg].sectors.items():
        nq = cols.get(q, 0)
        if not nq > 0:
            raise RuntimeError(f"Test B: residual sector {q} has no holdout column")
        rq = B.trim_per_sector(residual, rleg, {q: d}) if len(residual.legs[rleg].sectors) > 1 else residual
        per[q] = (B.norm(rq) ** 2 if rq is not None else 0.0) / nq
    return math.sqrt(sum(per.values())), per, cols


# ── the :adaptive controller: sectorwise thin pivoted QR, DD select, the incremental sketch ────

REORTH_KEEP = 1.0 / math.sqrt(2.0)  # ``_REORTH_KEEP`` (dd_cbe.jl:273)
DD_HOLDOUT = 4                      # ``_DD_HOLDOUT`` (dd_cbe_controller.jl:12)


PIVOT_TIE = 1e-10  # near-equal squared column norms (relative) count as a pivot tie


def pivoted_qr(A: np.ndarray):
    """Column-pivoted Householder QR of ``A`` (m x n), thin: ``(Q, |R_kk|)`` with Q's columns
    scaled so that R_kk >= 0. LAPACK geqp3's factorisation (``qr(A, ColumnNorm())`` in Julia):
    step k moves the remaining column of largest norm over rows k.. to position k and zeroes it
    below the diagonal with a zlarfg reflector H = I - tau v v^H (v_k = 1, beta real), applying H^H
    to the columns right of it. Two rules are this restatement's: the remaining norms are
    recomputed at every step (geqp3 downdates them), and columns whose squared norm is within
    ``PIVOT_TIE`` of the largest count as tied, the lowest index winning. Without the tie rule
    the order of columns of (numerically) equal norm -- every column in ``_dd_select``'s second
    pass, whose input is orthonormal columns projected once more -- is decided by rounding, in
    LAPACK as well, and so are the subsets a capped controller keeps."""
    A = np.array(A, dtype=np.complex128, copy=True)
    m, n = A.shape
    kq = min(m, n)
    taus = np.zeros(kq, dtype=np.complex128)
    betas = np.zeros(kq)
    for k in range(kq):
        nrm2 = np.sum(A[k:, k:].real ** 2 + A[k:, k:].imag ** 2, axis=0)
        top = nrm2.max()
        p = k + int(np.argmax(nrm2 >= top * (1.0 - PIVOT_TIE)))
        if p != k:
            A[:, [k, p]] = A[:, [p, k]]
        alpha = A[k, k]
        xn2 = float(np.sum(A[k + 1:, k].real ** 2 + A[k + 1:, k].imag ** 2))
        if xn2 == 0.0 and alpha.imag == 0.0:
            beta, tau = alpha.real, 0.0j
        else:
            nrm = math.sqrt(alpha.real ** 2 + alpha.imag ** 2 + xn2)
            beta = -nrm if alpha.real >= 0.0 else nrm
            tau = complex((beta - alpha.real) / beta, -alpha.imag / beta)
            A[k + 1:, k] *= 1.0 / (alpha - beta)
        taus[k], betas[k] = tau, beta
        if tau != 0:
            v = np.concatenate([[1.0 + 0j], A[k + 1:, k]])
            w = v.conj() @ A[k:, k + 1:]
            A[k:, k + 1:] -= np.conj(tau) * np.outer(v, w)
    Q = np.eye(m, kq, dtype=np.complex128)
    for k in reversed(range(kq)):
        if taus[k] == 0:
            continue
        v = np.concatenate([[1.0 + 0j], A[k + 1:, k]])
        Q[k:, :] -= taus[k] * np.outer(v, v.conj() @ Q[k:, :])
    Q *= np.where(betas < 0.0, -1.0, 1.0)[None, :]
    return Q, np.abs(betas)


def thin_qr(sketch: B.BT, fl: int, ref_dir: int, thr: float):
    """Orthonormal basis of the span of ``sketch``'s leg-``fl`` columns by column-pivoted
    Householder QR per charge sector of leg ``fl`` (``_thin_qr``, ``dd_cbe.jl:184-259``; the
    factorisation of :func:`pivoted_qr`). A direction is kept when its pivot ``|R_kk|`` exceeds
    ``thr``. The new leg has the arrow ``ref_dir`` (``align_charge``); each kept column's phase
    makes ``R_kk`` real positive (the gauge both implementations fix)."""
    others = [i for i in range(sketch.rank) if i != fl]
    ydir = sketch.legs[fl].dir
    groups = {}
    for key in sorted(sketch.blocks):
        groups.setdefault(key[fl], []).append(key)
    out_blocks, space = {}, {}
    for charge in sorted(groups):
        keys = groups[charge]
        mats = [sketch.blocks[k].transpose(others + [fl]).reshape(-1, sketch.blocks[k].shape[fl])
                for k in keys]
        stacked = np.vstack(mats)
        if stacked.shape[0] == 0:
            continue
        Q, rdiag = pivoted_qr(stacked)
        kept = int(np.count_nonzero(rdiag > thr))
        if kept == 0:
            continue
        Qm = Q[:, :kept]
        qn = charge if ydir == ref_dir else -charge
        space[qn] = kept
        row = 0
        for k, M in zip(keys, mats):
            nr = M.shape[0]
            shp = [sketch.blocks[k].shape[i] for i in others] + [kept]
            blk = Qm[row:row + nr].reshape(shp)
            row += nr
            inv = np.argsort(others + [fl])
            nk = list(k)
            nk[fl] = qn
            out_blocks[tuple(nk)] = np.ascontiguousarray(blk.transpose(inv))
    if not space:
        return None
    legs = list(sketch.legs)
    legs[fl] = B.Leg(ref_dir, dict(sorted(space.items())))
    return B.BT(legs, out_blocks)


def dd_select(frame, sketch, side):
    """``_dd_select`` (``dd_cbe.jl:290-321``): ``P^D sketch``, a first QR at the floor
    ``CBE_EPS max(|sketch|, |projected|)``, then a QR of ``P^D`` of the first pass keeping
    pivots ``>= REORTH_KEEP`` ("twice is enough")."""
    left = side == "left"
    fl = 2 if left else 0
    perp = perp_left if left else perp_right
    projected = perp(frame, sketch)
    nz, ny = B.norm(sketch), B.norm(projected)
    if ny <= CBE_EPS * max(nz, 1.0):
        return None
    ref_dir = frame.legs[fl].dir
    first = thin_qr(projected, fl, ref_dir, CBE_EPS * max(nz, ny))
    if first is None:
        return None
    return thin_qr(perp(frame, first), fl, ref_dir, REORTH_KEEP)


def target_sectors(boost: dict, per: dict, Om, wleg: int, alloc) -> int:
    """``_target_sectors!`` (``sketch.jl:188-201``)."""
    if not per:
        return 0
    have = {} if Om is None else dict(Om.legs[wleg].sectors)
    share = alloc.sample ** 2 / len(per)
    n = 0
    for q, r2 in per.items():
        if not alloc.scale ** 2 * r2 > share:
            continue
        boost[q] = boost.get(q, 0) + max(have.get(q, 0), 1)
        n += 1
    return n


def record_sample(ledger, side, ind, per, hcols, sketch, wleg, alloc):
    """``_record_sample!`` (``sketch.jl:215-258``)."""
    ledger.max_sample = max(ledger.max_sample, ind)
    if side == "left":
        ledger.max_sample_l = max(ledger.max_sample_l, ind)
    else:
        ledger.max_sample_r = max(ledger.max_sample_r, ind)
    tot = sum(per.values())
    relunc = 0.5 * math.sqrt(sum(r2 ** 2 / hcols[q] for q, r2 in per.items())) / tot if tot > 0 else 0.0
    ledger.sample_log.append(dict(side=side, est=ind, relunc=relunc,
                                  per={q: alloc.scale * math.sqrt(r2) for q, r2 in per.items()},
                                  holdout=dict(hcols),
                                  sketch={} if sketch is None else dict(sketch.legs[wleg].sectors)))


def dd_controller(frame, side, draw, sketch, project, initial_width, wcap, ncap, alloc, ledger,
                  holdout_width=DD_HOLDOUT, batch_blocks=1, cap_selection="storage",
                  acceptance_factor=1.0):
    """``_dd_controller`` (``dd_cbe_controller.jl:26-212``, no audit): grows the DD basis block by
    block until an independent holdout finds the rest within ``acceptance_factor * alloc.sample``.
    Returns ``(basis, status)``.

    As in the reference, streaming a block (probe or holdout) sets the controller's ``width`` to
    that block's column count: the reference's ``stream`` closure assigns the enclosing ``width``
    (``dd_cbe_controller.jl:108-118``), so a widening doubles the last streamed block's width."""
    if not 0 < acceptance_factor <= 1:
        raise ValueError("acceptance_factor must lie in (0,1]")
    if not 1 <= batch_blocks <= 8:
        raise ValueError("batch_blocks must lie in 1:8")
    if cap_selection not in ("storage", "svd"):
        raise ValueError("cap_selection must be :storage or :svd")
    left = side == "left"
    fl, wleg = (2, 0) if left else (0, 2)
    st = dict(aug=frame, basis=None, count=0, streamed=0, discovered=0, width=0)
    boost = {}

    def absorb(sketched):
        nb = dd_select(st["aug"], sketched, side)
        if nb is None:
            return 0
        current = 0 if st["basis"] is None else st["basis"].dim(fl)
        room = ncap - current
        if room <= 0:
            return 0
        if nb.dim(fl) > room:
            if cap_selection == "svd":
                # the strongest sampled directions across sectors: an SVD of the thin projected
                # sketch (dd_cbe_controller.jl:67-96)
                off = (perp_left if left else perp_right)(st["aug"], sketched)
                noff = B.norm(off)
                fac = B.svd(off, (0, 1) if left else (1, 2), cutoff=rank_cut(0.0, noff, noff),
                            nkeep=room)
                if not fac.kept:
                    nb = None
                elif left:
                    nb = reortho(st["aug"], fac.U, "left")
                else:
                    nb = reortho(st["aug"], rows_from_u(fac.U), "right")
            else:
                nb = B.trim_total(nb, fl, room)
            if nb is None:
                return 0
        st["basis"] = nb if st["basis"] is None else B.oplus([st["basis"], nb], fl)
        st["aug"] = B.oplus([st["aug"], nb], fl)
        return nb.dim(fl)

    def stream(Om, field):
        w = Om.dim(wleg)
        st["width"] = w
        st["streamed"] += w
        if field == "n_probes":
            st["discovered"] += w
        if ledger is not None:
            setattr(ledger, field, getattr(ledger, field) + w)
        return sketch(Om)

    def fresh(columns):
        Om = draw(columns, None)
        return None if Om is None else (Om, stream(Om, "n_holdout"))

    def resid(check):
        return sample_residual(st["basis"], project, lambda _: check[1], check[0], wleg, side)

    def newsector():
        b = st["basis"]
        return b is not None and any(frame.legs[fl].sectors.get(q, 0) == 0
                                     for q in b.legs[fl].sectors)

    def remaining():
        return ncap - (0 if st["basis"] is None else st["basis"].dim(fl))

    if cap_selection == "svd":
        st["width"] = min(max(max(initial_width, ncap + min(4, ncap)), 1), max(wcap, 1))
    else:
        st["width"] = min(max(initial_width, 1), max(min(wcap, ncap), 1))
    last = draw(st["width"], None)
    if last is None:
        return None, "empty"
    st["count"] += absorb(stream(last, "n_probes"))
    check = fresh(holdout_width)
    escalated = False
    while True:
        if check is None:
            return st["basis"], "met"
        est, per, hcols = resid(check)
        ind = indicator(alloc, est)
        ok = ind <= acceptance_factor * alloc.sample
        if ok and not escalated and (ind > alloc.sample / 2 or newsector()):
            escalated = True
            wide = fresh(2 * holdout_width)
            if wide is not None:
                check = wide
                continue
        capped = st["discovered"] >= wcap or st["count"] >= ncap
        if ok or capped:
            if ledger is not None:
                record_sample(ledger, side, ind, per, hcols, last, wleg, alloc)
            if ok:
                return st["basis"], "met"
            if ledger is not None:
                ledger.unmet_("sample")
                ledger.workcap_reached = True
            return st["basis"], "work_limited"
        nt = target_sectors(boost, per, check[0], wleg, alloc)
        if ledger is not None:
            ledger.n_targeted += nt
        if batch_blocks == 1:
            next_check = fresh(holdout_width)
            added = absorb(check[1])
            if nt == 0:
                st["width"] = min(2 * st["width"], wcap)
            if remaining() > 0:
                blk = draw(min(st["width"], max(remaining() + 2, 1)), boost if boost else None)
                if blk is not None:
                    last = blk
                    added += absorb(stream(blk, "n_probes"))
            check = next_check
        else:
            # the failed holdout is absorbed, then up to batch_blocks targeted blocks before
            # the next holdout is drawn (dd_cbe_controller.jl:186-202)
            added = absorb(check[1])
            for _ in range(batch_blocks):
                if remaining() <= 0:
                    break
                if nt == 0:
                    st["width"] = min(2 * st["width"], wcap)
                blk = draw(min(st["width"], max(remaining() + 2, 1)), boost if boost else None)
                if blk is None:
                    break
                last = blk
                added += absorb(stream(blk, "n_probes"))
            check = fresh(holdout_width)
        st["count"] += added
        if added == 0:
            if ledger is not None:
                record_sample(ledger, side, ind, per, hcols, last, wleg, alloc)
                ledger.unmet_("sample")
            return st["basis"], "basis_limited"


@dataclass
class BondFrame:
    U0: B.BT
    S0: B.BT
    V0: B.BT
    old_rank: int


def frame_theta(fr: BondFrame) -> B.BT:
    return B.contract(B.contract(fr.U0, (2,), fr.S0, (0,)), (2,), fr.V0, (0,))


def folded_closures(fr: BondFrame, mpo, bond, lenv, renv):
    """``_fold_sketch_closures`` (``cbe.jl:62-132``): ``(skl, skr)`` with the projection applied."""
    Wl, Wr = mpo[bond], mpo[bond + 1]
    theta = frame_theta(fr)

    def skl(Om):
        t = B.contract(Om, (2,), renv, (0,), conja=True)
        rc = B.contract(t, (1, 2), Wr, (2, 3))                  # (g, ket_r, w_mid, s_ket_r)
        tc = B.contract(theta, (2, 3), rc, (3, 1))               # (l, s_l, g, w_mid)
        wm = B.contract(tc, (1, 3), Wl, (1, 3))                  # (l, g, w_l, s_bra_l)
        t = B.contract(wm, (0, 2), lenv, (2, 1))                 # (g, s_bra_l, bra)
        return perp_left(fr.U0, B.permute(t, (2, 1, 0)))

    def skr(Om):
        t = B.contract(Om, (0,), lenv, (0,), conja=True)         # (s_bra_l, g, w, ket_l)
        cap = B.permute(B.contract(t, (0, 2), Wl, (2, 0)), (1, 0, 2, 3))  # (ket_l, g, s_ket_l, w_mid)
        tc = B.contract(theta, (0, 1), cap, (0, 2))              # (s_r, r, g, w_mid)
        wm = B.contract(tc, (0, 3), Wr, (1, 0))                  # (r, g, s_bra_r, w_r)
        t = B.contract(wm, (0, 3), renv, (2, 1))                 # (g, s_bra_r, bra_r)
        return perp_right(fr.V0, t)

    return skl, skr


def exact_leak(fr: BondFrame, mpo, bond, lenv, renv, side) -> float:
    """``_bond_action`` with ``fold = false`` (``krylov_frontier_bonds.jl:94-99``): the two-site
    action ``X = H Theta_F`` formed once and the exact leak ``||(I - U0 U0^dag) X||``
    (``_left_leak``) or ``||X (I - V0^dag V0)||`` (``_right_leak``) of the frame's prescribed
    isometry. Draws nothing."""
    from .tdvp import apply_two_site

    X = apply_two_site(lenv, mpo[bond], mpo[bond + 1], renv, frame_theta(fr))  # (l, s1, s2, r)
    if side == "left":
        return B.norm(perp_left(fr.U0, X))
    ov = B.contract(X, (2, 3), fr.V0, (1, 2), conjb=True)  # (l, s1, bond)
    return B.norm(B.sub(X, B.contract(ov, (2,), fr.V0, (0,))))


def sampled_leak(fr: BondFrame, skl, skr, side, column_count, rng) -> float:
    """``sampled_leak`` (``cbe.jl:355-391``)."""
    if side == "left":
        Om = graded_sketch(fr.V0, "right", column_count, rng)
        return sample_residual(None, lambda s: perp_left(fr.U0, s), skl, Om, 0, "left")[0]
    Om = graded_sketch(fr.U0, "left", column_count, rng)
    return sample_residual(None, lambda s: perp_right(fr.V0, s), skr, Om, 2, "right")[0]


@dataclass
class Expansion:
    U_ex: B.BT
    V_ex: B.BT
    n_new_l: int
    n_new_r: int
    err_pre: float = 0.0
    err_fnl: float = 0.0


def dd_cbe_expand(fr: BondFrame, mpo, bond, lenv, renv, side, alloc, ledger, workcap, rng,
                  fixed_width=8, tail_factor=0.10, mode="rank_tail", holdout_width=DD_HOLDOUT,
                  batch_blocks=1, cap_selection="storage", acceptance_factor=1.0,
                  exact=False) -> Expansion:
    """Grow one frame of the bond by the DD-projected sketch (``dd_cbe_expand.jl:19-419``): rank
    by tail bisection (``:rank_tail``, ``tail_dd``) or by the incremental controller
    (``:adaptive``, ``_dd_controller``). ``exact = true`` (the deterministic reference) sketches
    the complete DD-projected fused basis once and keeps what ``_dd_select``'s QR admits: the
    ``_certified_range`` call with no allocation (``dd_cbe_expand.jl:346-360``), whose
    ``_range_find`` stops after one pass because its width cap is its start width
    (``dd_cbe_expand.jl:91``, ``sketch.jl:119-132``); the mode is then not consulted."""
    if mode not in ("rank_tail", "adaptive") and not exact:
        raise NotImplementedError(f"DD mode {mode!r}: only :rank_tail and :adaptive are restated")
    if mode == "rank_tail" and fixed_width < 1:
        raise ValueError("rank_tail requires positive fixed_width")
    if not 0 < tail_factor <= 1:
        raise ValueError("tail_factor must lie in (0,1]")
    left = side == "left"
    U0, V0 = fr.U0, fr.V0
    old_rank = fr.old_rank
    frame, opp = (U0, V0) if left else (V0, U0)
    oside = "right" if left else "left"
    fl, wleg = (2, 0) if left else (0, 2)
    none = Expansion(U0, V0, 0, 0)
    full_self = U0.dim(0) * U0.dim(1) if left else V0.dim(1) * V0.dim(2)
    full_opp = V0.dim(1) * V0.dim(2) if left else U0.dim(0) * U0.dim(1)
    cap = full_self - old_rank
    wbind = False
    if alloc is not None and workcap > 0:
        wk = max(workcap - old_rank, 0)
        wbind = wk < cap
        cap = min(cap, wk)
    if cap <= 0:
        return none
    if left:
        core = B.contract(U0, (2,), fr.S0, (0,))

        def sketch(Om):
            return stream_left(core, V0, mpo, bond, lenv, renv, Om)

        def project(b):
            return perp_left(U0, b)
    else:
        core = B.contract(fr.S0, (1,), V0, (0,))

        def sketch(Om):
            return stream_right(U0, core, mpo, bond, lenv, renv, Om)

        def project(b):
            return perp_right(V0, b)

    directions, direction_count = None, 0
    if exact:
        Om = dd_probe_exact(opp, oside)
        if Om is not None:
            directions = dd_select(frame, sketch(Om), side)
            direction_count = 0 if directions is None else directions.dim(fl)
        Om = None
    elif mode == "adaptive":
        dmax = max(U0.dim(0), old_rank, V0.dim(2))
        initial_width = math.ceil(1.2 * max(math.ceil(ADAPTIVE_GROWTH * dmax) - old_rank, 1))
        wcap = full_opp
        if alloc is not None and workcap > 0:
            wcap = min(wcap, workcap)
        directions, _ = dd_controller(frame, side, lambda w, bst: dd_probe(opp, oside, w, rng, bst),
                                      sketch, project, initial_width, wcap, cap, alloc, ledger,
                                      holdout_width, batch_blocks, cap_selection, acceptance_factor)
        direction_count = 0 if directions is None else directions.dim(fl)
        Om = None
    else:  # tail_dd
        Om = dd_probe(opp, oside, min(fixed_width, full_opp), rng)
    if Om is not None:
        if ledger is not None:
            ledger.n_probes += Om.dim(wleg)
        Y = project(sketch(Om))
        nY = B.norm(Y)
        if not nY <= CBE_EPS:
            legs = (0, 1) if left else (1, 2)
            rmax = min(cap, Om.dim(wleg))
            cache = {}

            def candidate(k):
                if k <= 0:
                    return None
                if k in cache:
                    return cache[k]
                fac = B.svd(Y, legs, cutoff=rank_cut(0.0, nY, nY), nkeep=k)
                if not fac.kept:
                    res = None
                elif left:
                    res = reortho(frame, fac.U, "left")
                else:
                    res = reortho(frame, rows_from_u(fac.U), "right")
                cache[k] = res
                return res

            limit = tail_factor * alloc.sample

            def metric(k):
                est = sample_residual(candidate(k), project, lambda _: Y, Om, wleg, side)[0]
                return indicator(alloc, est)

            if metric(0) <= limit:
                directions, direction_count = None, 0
            else:
                hi = rmax
                if metric(hi) > limit:
                    directions, direction_count = candidate(hi), hi
                else:
                    lo = 0
                    while hi - lo > 1:
                        k = (hi + lo) // 2
                        if metric(k) <= limit:
                            hi = k
                        else:
                            lo = k
                    Bk = candidate(hi)
                    directions, direction_count = Bk, (0 if Bk is None else Bk.dim(fl))
    if directions is None:
        return none
    if direction_count > cap:
        directions = B.trim_total(directions, fl, cap)
        if directions is None:
            return none
    if ledger is not None and wbind and direction_count >= cap:
        ledger.workcap_reached = True
    directions = cap_to_local_room(frame, directions, side)
    if directions is None:
        return none
    nq = directions.dim(fl)
    if ledger is not None:
        ledger.n_selected += nq
    grown = B.oplus([frame, directions], fl)
    if left:
        return Expansion(grown, V0, nq, 0)
    return Expansion(U0, grown, 0, nq)
