"""Input builders and containers on device: spin-1/2 local space, product states, the XXZ MPO.

States and operators are assembled on the host block by block (they are tiny: bond dimension 1
states, MPO blocks of size <= 5x2x2x5) and uploaded once; from then on they live in HBM. They
follow:

* ``local_space`` / ``SECTOR_UP`` / ``SECTOR_DOWN`` (``src/QMB/Tooling/local_spaces.jl:14-39``):
  U(1) charge ``2 S^z`` (up +1, down -1); under ``:none`` one sector of dimension 2, up first.
* ``product_state`` / ``domain_wall_state`` / ``neel_state``
  (``src/QMB/Tooling/initial_states.jl:15-80,137,145``): bond dimension 1, centre at site L.
* ``xxz_mpo`` = ``mpo_from_terms(xxz_chain(L; J, delta))`` (``src/QMB/Models/ClosedSystem/xxz.jl:15-62``,
  ``src/BUG/Core/TensorNetworks/mpo.jl:208-254``): automaton states ``id, S+ open, S- open,
  (Sz open), done``; the XY term is ``(J/2)(S+S- + S-S+)``, the closing half carries the
  coefficient; site 1 keeps the ``id`` row, site L the ``done`` column.

Arrow conventions: an MPS site tensor is ``(link_l:-1, site:-1, link_r:+1)``; an MPO tensor is
``(w_l:-1, s_in:+1, s_out:-1, w_r:+1)`` with ``H = sum W[.., s_in, s_out, ..] |s_out><s_in|``.
"""

from __future__ import annotations

import numpy as np

from .tensor import Leg, from_blocks

SP = np.array([[0, 1], [0, 0]], dtype=np.complex128)  # <out|S+|in>, basis (up, down)
SM = np.array([[0, 0], [1, 0]], dtype=np.complex128)
SZ = np.array([[0.5, 0], [0, -0.5]], dtype=np.complex128)
ID = np.eye(2, dtype=np.complex128)


class LocalSpace:
    """Spin-1/2 site: ``state(i) -> (charge, index)`` for basis state ``i`` (0 = up, 1 = down)."""

    def __init__(self, symmetry: str):
        if symmetry not in ("U1", "none"):
            raise ValueError(f"symmetry must be 'U1' or 'none', got {symmetry!r}")
        self.symmetry = symmetry
        if symmetry == "U1":
            self.states = [(+1, 0), (-1, 0)]
            self.leg_sectors = {-1: 1, +1: 1}
        else:
            self.states = [(0, 0), (0, 1)]
            self.leg_sectors = {0: 2}

    def site_leg(self, dir: int) -> Leg:
        return Leg(dir, self.leg_sectors)

    def op_charge(self, op: np.ndarray) -> int:
        """Charge ``q_out - q_in`` an operator transfers (0 under ``:none``)."""
        qs = set()
        for i in range(2):
            for o in range(2):
                if op[o, i] != 0:
                    qs.add(self.states[o][0] - self.states[i][0])
        if len(qs) > 1:
            raise ValueError("operator does not have a definite charge")
        return qs.pop() if qs else 0


class MPS:
    """``tensors[i]``: ``(link_l, site, link_r)``; ``center`` is the orthogonality centre (1-based,
    as in ``symmetric_mps.jl:44-47``)."""

    def __init__(self, tensors, center: int):
        self.tensors = list(tensors)
        self.center = int(center)

    def __len__(self):
        return len(self.tensors)

    def __getitem__(self, i):  # 1-based
        return self.tensors[i - 1]

    def __setitem__(self, i, t):
        self.tensors[i - 1] = t

    def copy(self) -> "MPS":
        return MPS(self.tensors, self.center)

    def bond_dims(self):
        return [self[b].dim(2) for b in range(1, len(self))]


class MPO:
    def __init__(self, tensors):
        self.tensors = list(tensors)

    def __len__(self):
        return len(self.tensors)

    def __getitem__(self, i):  # 1-based
        return self.tensors[i - 1]


def product_state(spins, symmetry: str = "U1") -> MPS:
    """``spins``: sequence of ``'up'``/``'down'``. Bond dimension 1, centre at L."""
    ls = LocalSpace(symmetry)
    tensors = []
    ql = 0
    for s in spins:
        i = {"up": 0, "down": 1}[s]
        qs, idx = ls.states[i]
        qr = ql + qs
        blk = np.zeros((1, ls.leg_sectors[qs], 1), dtype=np.complex128)
        blk[0, idx, 0] = 1.0
        t = from_blocks([Leg(-1, {ql: 1}), ls.site_leg(-1), Leg(+1, {qr: 1})], {(ql, qs, qr): blk})
        tensors.append(t)
        ql = qr
    return MPS(tensors, len(tensors))


def domain_wall_state(L: int, symmetry: str = "U1") -> MPS:
    return product_state(["up" if i < L // 2 else "down" for i in range(L)], symmetry)


def neel_state(L: int, symmetry: str = "U1") -> MPS:
    return product_state(["up" if i % 2 == 0 else "down" for i in range(L)], symmetry)


def _op_blocks(ls: LocalSpace, op: np.ndarray):
    """Non-zero entries of a 2x2 operator as ``(q_in, i_in, q_out, i_out, value)``."""
    out = []
    for i in range(2):
        for o in range(2):
            if op[o, i] != 0:
                qi, ii = ls.states[i]
                qo, io = ls.states[o]
                out.append((qi, ii, qo, io, op[o, i]))
    return out


def mpo_from_entries(L: int, ls: LocalSpace, wstates, entries_of_site) -> MPO:
    """Build an MPO from automaton entries.

    ``wstates``: list of ``(name, charge)``; each state's position inside its charge sector is
    its order among the states of that charge. ``entries_of_site(site)`` yields
    ``(row_state, col_state, op2x2, coeff)``; site 1 keeps row ``wstates[0]`` only and site L
    column ``wstates[-1]`` only."""
    charge = {n: q for n, q in wstates}
    pos = {}
    count = {}
    for n, q in wstates:
        pos[n] = count.get(q, 0)
        count[q] = pos[n] + 1
    first, last = wstates[0][0], wstates[-1][0]
    tensors = []
    for site in range(1, L + 1):
        rows = [first] if site == 1 else [n for n, _ in wstates]
        cols = [last] if site == L else [n for n, _ in wstates]
        rsec, csec = {}, {}
        rpos, cpos = {}, {}
        for n in rows:
            q = charge[n]
            rpos[n] = rsec.get(q, 0)
            rsec[q] = rpos[n] + 1
        for n in cols:
            q = charge[n]
            cpos[n] = csec.get(q, 0)
            csec[q] = cpos[n] + 1
        legs = [Leg(-1, rsec), ls.site_leg(+1), ls.site_leg(-1), Leg(+1, csec)]
        blocks = {}
        for r, c, op, coeff in entries_of_site(site):
            if r not in rpos or c not in cpos:
                continue
            for qi, ii, qo, io, v in _op_blocks(ls, op):
                key = (charge[r], qi, qo, charge[c])
                assert -key[0] + key[1] - key[2] + key[3] == 0, (r, c, key)
                if key not in blocks:
                    blocks[key] = np.zeros(
                        (rsec[key[0]], ls.leg_sectors[qi], ls.leg_sectors[qo], csec[key[3]]),
                        dtype=np.complex128,
                    )
                blocks[key][rpos[r], ii, io, cpos[c]] += coeff * v
        tensors.append(from_blocks(legs, blocks))
    return MPO(tensors)


def xxz_mpo(L: int, J: float = 1.0, delta: float = 1.0, symmetry: str = "U1") -> MPO:
    """``H = J sum_i (Sx Sx + Sy Sy + delta Sz Sz)`` on an open chain (``xxz.jl:15-62``)."""
    if L < 2:
        raise ValueError("xxz_mpo needs at least two sites")
    ls = LocalSpace(symmetry)
    u1 = symmetry == "U1"
    wstates = [("id", 0), ("p", 2 if u1 else 0), ("m", -2 if u1 else 0)]
    if delta != 0.0:
        wstates.append(("z", 0))
    wstates.append(("done", 0))

    def entries(site):
        out = [("id", "id", ID, 1.0), ("done", "done", ID, 1.0)]
        out += [("id", "p", SP, 1.0), ("p", "done", SM, 0.5 * J)]
        out += [("id", "m", SM, 1.0), ("m", "done", SP, 0.5 * J)]
        if delta != 0.0:
            out += [("id", "z", SZ, 1.0), ("z", "done", SZ, J * delta)]
        if site == L:
            out = [e for e in out if not (e[0] == "id" and e[1] == "id")]
        if site == 1:
            out = [e for e in out if not (e[0] == "done")]
        return out

    return mpo_from_entries(L, ls, wstates, entries)


def move_right(psi, site):
    """``move_right!`` (``canonical_form.jl:10-54``): site = U, S Vd absorbed into site + 1."""
    from . import tensor as B

    res = B.svd(psi[site], (0, 1), cutoff=0.0)
    psi[site + 1] = B.contract(res.SVd(), (1,), psi[site + 1], (0,))
    psi[site] = res.U


def move_left(psi, site):
    """``move_left!``: site = Vd, U S absorbed into site - 1."""
    from . import tensor as B

    res = B.svd(psi[site], (0,), cutoff=0.0)
    psi[site - 1] = B.contract(psi[site - 1], (2,), res.US(), (0,))
    psi[site] = res.Vd


def canonical(psi, site):
    """``canonical!(psi, site)``: gauge moves (block SVDs on the device) to centre ``site``."""
    if not 1 <= site <= len(psi):
        raise IndexError(site)
    while psi.center < site:
        move_right(psi, psi.center)
        psi.center += 1
    while psi.center > site:
        move_left(psi, psi.center)
        psi.center -= 1
    return psi


def sz_profile(psi) -> np.ndarray:
    """``<S^z_j>`` for every site of a normalised or unnormalised state
    (``magnetisation`` -> ``site_expval``, ``src/QMB/Observables/bond_observables.jl:15``,
    ``local_observables.jl:11-24``): the centre is moved to each site in turn and the site's
    weight read off, which is exact because every other tensor is then an isometry."""
    from .tensor import to_blocks

    phi = psi.copy()
    ls_sym = "U1" if len(phi[1].legs[1].sectors) == 2 else "none"
    ls = LocalSpace(ls_sym)
    out = []
    canonical(phi, 1)
    for j in range(1, len(phi) + 1):
        if j > 1:
            canonical(phi, j)
        legs, blocks = to_blocks(phi[j])
        n2 = sum(float(np.vdot(b, b).real) for b in blocks.values())
        acc = 0.0
        for (ql, qs, qr), blk in blocks.items():
            for idx in range(blk.shape[1]):
                st = ls.states.index((qs, idx))
                acc += float(np.vdot(blk[:, idx, :], blk[:, idx, :]).real) * SZ[st, st].real
        out.append(acc / n2)
    return np.array(out)
