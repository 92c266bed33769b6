"""MPO environments and effective operators of the CPU oracle.

TEST INFRASTRUCTURE (see ``oracle/blocks.py``). Restates ``src/BUG/Core/Environments/``:

* ``left_step`` / ``right_step``: ``_mpo_left_step`` / ``_mpo_right_step``
  (``mpo_environments.jl:65-108``) with the same contraction order. The chain ends are explicit
  dimension-1 environments (value 1) instead of ``nothing``; the MPO's boundary legs have
  dimension 1, so the arithmetic is the same.
* ``apply_one_site`` (``effective_operators.jl:39-64``), ``zero_site_h`` / ``apply_zero_site``
  (``:91-107``).
* ``stream_left`` / ``stream_right`` (``mpo_environments.jl:409-481``): the two-site action on a
  thin probe, ``Theta`` never formed.

Environment layouts: left ``(bra:-1, w:+1, ket:+1)``, right ``(bra:+1, w:-1, ket:-1)``.
"""

from __future__ import annotations

import numpy as np

from .blocks import BT, Leg, conj, contract, permute


def left_boundary() -> BT:
    return BT([Leg(-1, {0: 1}), Leg(+1, {0: 1}), Leg(+1, {0: 1})],
              {(0, 0, 0): np.ones((1, 1, 1), dtype=np.complex128)})


def right_boundary(total_charge: int) -> BT:
    q = int(total_charge)
    return BT([Leg(+1, {q: 1}), Leg(-1, {0: 1}), Leg(-1, {q: 1})],
              {(q, 0, q): np.ones((1, 1, 1), dtype=np.complex128)})


def total_charge(psi) -> int:
    (q, d), = psi[len(psi)].legs[2].sectors.items()
    return q


def left_step(E: BT, A: BT, W: BT, B: BT | None = None) -> BT:
    """E' = B^dag (E A W) on the next link (``mpo_environments.jl:65-82``)."""
    B = A if B is None else B
    t = contract(E, (2,), A, (0,))            # (bra, w, s, l_r)
    t = contract(t, (1, 2), W, (0, 1))        # (bra, l_r, s_bra, w_r)
    t = contract(t, (0, 2), B, (0, 1), conjb=True)  # (l_r, w_r, l_r')
    return permute(t, (2, 1, 0))


def right_step(R: BT, A: BT, W: BT) -> BT:
    """Mirror push through site ``A`` (``mpo_environments.jl:93-108``)."""
    t = contract(A, (2,), R, (2,))            # (l_l, s, bra, w)
    t = contract(t, (1, 3), W, (1, 3))        # (l_l, bra, w_l, s_bra)
    t = contract(t, (1, 3), A, (2, 1), conjb=True)  # (l_l, w_l, l_l')
    return permute(t, (2, 1, 0))


def right_env_stack(psi, mpo, downto: int):
    """``right_env_stack(psi, mpo; downto)`` (``mpo_environments.jl:161-175``): entry ``i`` (1-based
    link) is the environment of sites ``>= i``."""
    L = len(psi)
    envs = [None] * (L + 2)
    cur = right_boundary(total_charge(psi))
    envs[L + 1] = cur
    for site in range(L, downto - 1, -1):
        cur = right_step(cur, psi[site], mpo[site])
        envs[site] = cur
    return envs


def left_env_stack(psi, mpo, upto: int):
    """``left_env_stack(psi, mpo; upto)`` (``mpo_environments.jl:141-154``)."""
    L = len(psi)
    envs = [None] * (L + 2)
    cur = left_boundary()
    envs[1] = cur
    for site in range(1, upto + 1):
        cur = left_step(cur, psi[site], mpo[site])
        envs[site + 1] = cur
    return envs


def apply_one_site(Lenv: BT, W: BT, Renv: BT, x: BT) -> BT:
    """``H_eff x`` for a site tensor (``effective_operators.jl:39-64``)."""
    t = contract(Lenv, (2,), x, (0,))         # (bra_l, w, s, l_r)
    t = contract(t, (1, 2), W, (0, 1))        # (bra_l, l_r, s_bra, w_r)
    return contract(t, (3, 1), Renv, (1, 2))  # (bra_l, s_bra, bra_r)


class ZeroSiteH:
    """``H0 S = sum_w L[w] S R[w]`` through the expanded frames (``effective_operators.jl:78-107``)."""

    def __init__(self, mpo, bond, lenv, renv, U_ex, V_ex, eshift=0.0):
        self.l = left_step(lenv, U_ex, mpo[bond])
        self.r = right_step(renv, V_ex, mpo[bond + 1])
        self.eshift = float(eshift)  # applies H0 - eshift (shift_h)

    def apply(self, core: BT) -> BT:
        t = contract(self.l, (2,), core, (0,))     # (bra_l, w, b_r)
        y = contract(t, (1, 2), self.r, (1, 2))    # (bra_l, bra_r)
        if self.eshift == 0.0:
            return y
        from .blocks import add

        return add(y, core, 1.0, -self.eshift)


def stream_left(left_amplitude: BT, right_isometry: BT, mpo, bond, lenv, renv, Om: BT) -> BT:
    """``X Om`` for a probe in ``V0``'s layout ``(g, s_r, l_r)``; returns ``(l_l, s_l, g)``
    (``mpo_environments.jl:409-440``)."""
    Wl, Wr = mpo[bond], mpo[bond + 1]
    t = contract(Om, (2,), renv, (0,), conja=True)          # (g, s_bra_r, w, ket_r)
    rc = contract(t, (1, 2), Wr, (2, 3))                     # (g, ket_r, w_mid, s_ket_r)
    bp = contract(right_isometry, (1, 2), rc, (3, 1))        # (bond, g, w_mid)
    sp = contract(left_amplitude, (2,), bp, (0,))            # (l_l, s_l, g, w_mid)
    wm = contract(sp, (1, 3), Wl, (1, 3))                    # (l_l, g, w_l, s_bra_l)
    t = contract(wm, (0, 2), lenv, (2, 1))                   # (g, s_bra_l, bra)
    return permute(t, (2, 1, 0))


def stream_right(left_isometry: BT, right_amplitude: BT, mpo, bond, lenv, renv, Om: BT) -> BT:
    """``X^dag Om`` as rows for a probe in ``U0``'s layout ``(l_l, s_l, g)``; returns
    ``(g, s_r, l_r)`` (``mpo_environments.jl:449-481``)."""
    Wl, Wr = mpo[bond], mpo[bond + 1]
    t = contract(Om, (0,), lenv, (0,), conja=True)           # (s_bra_l, g, w, ket_l)
    gf = contract(t, (0, 2), Wl, (2, 0))                     # (g, ket_l, s_ket_l, w_mid)
    lc = permute(gf, (1, 0, 2, 3))                           # (ket_l, g, s_ket_l, w_mid)
    bp = contract(left_isometry, (0, 1), lc, (0, 2))         # (bond, g, w_mid)
    sp = contract(right_amplitude, (0,), bp, (0,))           # (s_r, l_r, g, w_mid)
    wm = contract(sp, (0, 3), Wr, (1, 0))                    # (l_r, g, s_bra_r, w_r)
    return contract(wm, (0, 3), renv, (2, 1))                # (g, s_bra_r, bra_r)
