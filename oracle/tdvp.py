"""CPU restatement of the two-site TDVP baseline (test infrastructure: the checker of the device
``bug_tdvp2_step``, never part of the product).

Follows ``src/Baselines/TDVP/tdvp2.jl``: ``tdvp2_step!`` (``:229-297``), the bond update
``_tdvp2_bond!`` (``:39-136``) and the backward one-site half-step ``_tdvp2_backward`` (``:145-173``),
with the two-site action ``apply_h_two_site`` (``src/BUG/Core/Environments/mpo_environments.jl:316-344``)
written over explicit dimension-1 chain-end environments instead of the reference's ``nothing``
ends. The optional backward-amplification reports (``backward_report``, ``backward_norms``) are not
restated.
"""

from __future__ import annotations

import math

from . import blocks as B
from . import krylov as K
from .env import apply_one_site, left_boundary, left_env_stack, left_step, right_boundary
from .env import right_env_stack, right_step, total_charge
from .step import VOPS, bug_root_link, budget_svd, canonical, cut_divisor


def apply_two_site(lenv, Wl, Wr, renv, theta):
    """``H Theta`` for a two-site tensor ``(l, s1, s2, r)`` (``apply_h_two_site``)."""
    t = B.contract(lenv, (2,), theta, (0,))      # (bra_l, w, s1, s2, r)
    t = B.contract(t, (1, 2), Wl, (0, 1))        # (bra_l, s2, r, s1_bra, w_mid)
    t = B.contract(t, (4, 1), Wr, (0, 1))        # (bra_l, r, s1_bra, s2_bra, w_r)
    return B.contract(t, (4, 1), renv, (1, 2))   # (bra_l, s1_bra, s2_bra, bra_r)


def _elements(t) -> int:
    return sum(int(v.size) for v in t.blocks.values())


def _expv(apply, tau, vector, kw):
    out, rep = K.expv(VOPS, apply, tau, vector, hermitian=kw["hermitian"], maxiter=kw["maxiter"],
                      tol=kw["tol"], conv_tol=kw["conv_tol"], substeps=kw["substeps"])
    return out, rep


def tdvp2_step(psi, mpo, tau, maxdim=200, trunc_thresh=1e-12, maxiter=30, tol=1e-15,
               hermitian=True, conv_tol=0.0, substeps=1, weight_tol=None, eshift=0.0,
               backward_report=None, backward_norms=None):
    """One symmetric two-site TDVP step of ``tau`` in place (``tdvp2_step!``); returns the
    ``TDVP2Info`` fields as a dict."""
    L = len(psi)
    if L < 2:
        raise ValueError("tdvp2_step needs at least two sites")
    if len(mpo) != L:
        raise ValueError(f"chain has {len(mpo)} sites, state has {L}")
    if weight_tol is not None and weight_tol < 0:
        raise ValueError("weight_tol must be non-negative")
    if backward_report is not None or backward_norms is not None:
        raise NotImplementedError("backward_report / backward_norms are not restated")
    tau = complex(tau)
    half = tau / 2
    eshift = float(eshift)
    wdiv = cut_divisor(L, bug_root_link(L) + 1)
    kw = dict(hermitian=hermitian, maxiter=maxiter, tol=tol, conv_tol=conv_tol, substeps=substeps)
    acc = dict(apps=0, theta=0, worst=0.0, peak=0, w=[0.0, 0.0], tot=0.0)

    def stored():
        return sum(_elements(psi[s]) for s in range(1, L + 1))

    def shifted(apply):
        if eshift == 0.0:
            return apply
        return lambda x: B.add(apply(x), x, 1.0, -eshift)

    def counted(apply):
        def f(x):
            acc["apps"] += 1
            return apply(x)
        return f

    def backward(lch, W, rch, M):
        op = counted(shifted(lambda x: apply_one_site(lch, W, rch, x)))
        return _expv(op, -half, M, kw)[0]

    def bond(i, right, lch, rch, sweep):
        theta = B.contract(psi[i], (2,), psi[i + 1], (0,))
        acc["theta"] = max(acc["theta"], _elements(theta))
        acc["peak"] = max(acc["peak"], stored() + _elements(theta))
        h2 = counted(shifted(lambda x: apply_two_site(lch, mpo[i], mpo[i + 1], rch, x)))
        theta = _expv(h2, half, theta, kw)[0]
        if weight_tol is None:
            res = B.svd(theta, (0, 1), cutoff=max(trunc_thresh, 1e-14), nkeep=maxdim)
        else:
            res = budget_svd(theta, (0, 1), maxdim, lambda n2: weight_tol * math.sqrt(n2) / wdiv)[0]
        acc["worst"] = max(acc["worst"], B.trunc_weight(res))
        acc["w"][sweep] += B.sq_weight(res.trunc)
        acc["tot"] = max(acc["tot"], B.sq_weight(res.kept) + B.sq_weight(res.trunc))
        if right:
            psi[i] = res.U
            lnext = left_step(lch, psi[i], mpo[i])
            M = res.SVd()
            if i < L - 1:
                M = backward(lnext, mpo[i + 1], rch, M)
            psi[i + 1] = M
            psi.center = i + 1
            return lnext
        psi[i + 1] = res.Vd
        rnext = right_step(rch, psi[i + 1], mpo[i + 1])
        M = res.US()
        if i > 1:
            M = backward(lch, mpo[i], rnext, M)
        psi[i] = M
        psi.center = i
        return rnext

    canonical(psi, 1)
    rstack = right_env_stack(psi, mpo, downto=3)
    lch = left_boundary()
    for i in range(1, L):
        lch = bond(i, True, lch, rstack[i + 2], 0)
    lstack = left_env_stack(psi, mpo, upto=L - 2)
    rch = right_boundary(total_charge(psi))
    for i in range(L - 1, 0, -1):
        canonical(psi, i)
        rch = bond(i, False, lstack[i], rch, 1)
    cum = (math.sqrt(acc["w"][0]) + math.sqrt(acc["w"][1])) / math.sqrt(acc["tot"]) if acc["tot"] > 0 else 0.0
    return dict(max_bond=max(psi.bond_dims(), default=0), theta_elements=acc["theta"],
                discarded=acc["worst"], peak_elements=acc["peak"], krylov_dims=acc["apps"],
                cumulative=cum)
