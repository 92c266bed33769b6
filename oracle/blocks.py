"""Block-sparse U(1) tensors for the CPU oracle (numpy, complex128).

TEST INFRASTRUCTURE. This package is the CPU restatement that the parity tests, ``smoke()`` and
the CPU-baseline leg of ``bench.py`` check the CUDA engine against; nothing in the product imports
it. It restates the semantics of the reference's block-sparse container and kernels
(``deps/Telum/src/contract.jl``, ``deps/Telum/src/svd.jl``) for abelian symmetries only.

Conventions (this module's own, equivalent to Telum's for U(1) and ``:none``):

* A tensor is a list of legs and a dict of dense blocks. A leg has an arrow ``dir`` (+1 outgoing,
  -1 incoming) and an ordered map ``charge -> dimension``. A block is keyed by one charge per leg
  and exists only when the charges balance: ``sum_i dir_i * q_i == 0``. Absent blocks are zero.
* ``:none`` is the one-sector case: every charge is 0.
* Charge conservation in an MPS site tensor ``(link_l, site, link_r)`` has arrows ``(-1,-1,+1)``,
  so ``q_r = q_l + q_s`` and a link carries the total charge to its left.

The SVD follows Telum's selection (``deps/Telum/src/svd.jl:1825-1921``): per-sector LAPACK SVD,
keep ``sigma > cutoff * sigma_max``, a stable descending sort over all sectors, then ``Nkeep``.
Sectors are visited in ascending charge order, which fixes how ties across sectors are broken.
The phase of every singular pair is fixed by the rule in :func:`_fix_phases` so that two
implementations that agree to roundoff also agree on the link bases that randomised probes are
drawn in.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

#: weights of the phase-fixing functional, ``c_i = 1 / (i + golden ratio)``
_PHI = (1.0 + 5.0 ** 0.5) / 2.0


class Leg:
    """One tensor leg: an arrow and an ordered ``charge -> dim`` map (ascending charge)."""

    __slots__ = ("dir", "sectors")

    def __init__(self, dir: int, sectors):
        self.dir = int(dir)
        self.sectors = {int(q): int(d) for q, d in sorted(dict(sectors).items()) if int(d) > 0}

    def dim(self) -> int:
        return sum(self.sectors.values())

    def flip(self) -> "Leg":
        return Leg(-self.dir, self.sectors)

    def same_space(self, other: "Leg") -> bool:
        return self.sectors == other.sectors

    def __repr__(self):
        return f"Leg({self.dir:+d}, {self.sectors})"


def merge_legs(a: Leg, b: Leg) -> Leg:
    """The union of two legs' sectors (dimensions must agree where both have a sector)."""
    if a.dir != b.dir:
        raise ValueError(f"leg arrows differ: {a} vs {b}")
    out = dict(a.sectors)
    for q, d in b.sectors.items():
        if q in out and out[q] != d:
            raise ValueError(f"sector {q} has dimension {out[q]} vs {d}")
        out[q] = d
    return Leg(a.dir, out)


class BT:
    """A block-sparse tensor: ``legs`` and ``blocks`` (charge tuple -> complex128 ndarray)."""

    __slots__ = ("legs", "blocks")

    def __init__(self, legs, blocks=None):
        self.legs = list(legs)
        self.blocks = {} if blocks is None else dict(blocks)

    @property
    def rank(self) -> int:
        return len(self.legs)

    def dim(self, leg: int) -> int:
        return self.legs[leg].dim()

    def copy(self) -> "BT":
        return BT(self.legs, {k: v.copy() for k, v in self.blocks.items()})

    def elements(self) -> int:
        return sum(v.size for v in self.blocks.values())

    def __repr__(self):
        return f"BT(legs={self.legs}, nblocks={len(self.blocks)})"


def check(t: BT) -> BT:
    """Assert the charge rule and the block shapes (debug helper for tests)."""
    for key, blk in t.blocks.items():
        assert len(key) == t.rank
        assert sum(l.dir * q for l, q in zip(t.legs, key)) == 0, (key, t.legs)
        assert blk.shape == tuple(l.sectors[q] for l, q in zip(t.legs, key)), (key, blk.shape)
    return t


# ── elementwise algebra ──────────────────────────────────────────────────────────────────────


def norm(t: BT) -> float:
    """Frobenius norm over every stored block (``tlarray/algebra.jl:69-105``)."""
    s = 0.0
    for k in sorted(t.blocks):
        b = t.blocks[k]
        s += float(np.vdot(b, b).real)
    return math.sqrt(s)


def inner(a: BT, b: BT) -> complex:
    """``<a|b>`` over matching blocks; zero when none match (``symmetric_mps.jl:83-93``)."""
    s = 0.0 + 0.0j
    for k in sorted(a.blocks):
        if k in b.blocks:
            s += complex(np.vdot(a.blocks[k], b.blocks[k]))
    return s


def scale(t: BT, s) -> BT:
    return BT(t.legs, {k: s * v for k, v in t.blocks.items()})


def add(a: BT, b: BT, alpha=1.0, beta=1.0) -> BT:
    """``alpha*a + beta*b`` on the union of the two block sets."""
    legs = [merge_legs(x, y) for x, y in zip(a.legs, b.legs)]
    out = {}
    for k, v in a.blocks.items():
        out[k] = alpha * v
    for k, v in b.blocks.items():
        if k in out:
            out[k] = out[k] + beta * v
        else:
            out[k] = beta * v
    return BT(legs, out)


def sub(a: BT, b: BT) -> BT:
    return add(a, b, 1.0, -1.0)


def conj(t: BT) -> BT:
    """Complex conjugate with every arrow flipped (Telum's ``t'``)."""
    return BT([l.flip() for l in t.legs], {k: np.conj(v) for k, v in t.blocks.items()})


def permute(t: BT, perm) -> BT:
    perm = tuple(perm)
    return BT(
        [t.legs[p] for p in perm],
        {tuple(k[p] for p in perm): np.ascontiguousarray(v.transpose(perm)) for k, v in t.blocks.items()},
    )


# ── contraction ──────────────────────────────────────────────────────────────────────────────


def contract(a: BT, ia, b: BT, ib, conja: bool = False, conjb: bool = False) -> BT:
    """Contract legs ``ia`` of ``a`` with legs ``ib`` of ``b`` (``contract.jl:2686-2691``).

    Paired legs must carry opposite arrows (after the optional conjugations). The result keeps
    ``a``'s free legs in order, then ``b``'s. Every matching block pair is one dense contraction
    (``contract.jl:952-1005`` does the same per pair with zgemm); the abelian w-matrix is 1
    (``contract.jl:2277``).
    """
    ia, ib = tuple(ia), tuple(ib)
    if conja:
        a = conj(a)
    if conjb:
        b = conj(b)
    for x, y in zip(ia, ib):
        la, lb = a.legs[x], b.legs[y]
        if la.dir != -lb.dir:
            raise ValueError(f"contract: arrows must oppose, leg {x} {la} vs leg {y} {lb}")
    fa = [i for i in range(a.rank) if i not in ia]
    fb = [i for i in range(b.rank) if i not in ib]
    legs = [a.legs[i] for i in fa] + [b.legs[i] for i in fb]
    groups = {}
    for kb, vb in b.blocks.items():
        groups.setdefault(tuple(kb[i] for i in ib), []).append((kb, vb))
    out = {}
    for ka in sorted(a.blocks):
        va = a.blocks[ka]
        ckey = tuple(ka[i] for i in ia)
        for kb, vb in groups.get(ckey, ()):
            key = tuple(ka[i] for i in fa) + tuple(kb[i] for i in fb)
            r = np.tensordot(va, vb, axes=(ia, ib))
            if key in out:
                out[key] = out[key] + r
            else:
                out[key] = r
    return BT(legs, out)


def relabel_free(t: BT) -> BT:
    """Drop blocks that are exactly absent sectors (no-op helper kept for symmetry)."""
    return t


# ── direct sums and sector selection ─────────────────────────────────────────────────────────


def oplus(tensors, leg: int) -> BT:
    """Direct sum along ``leg`` (``tlarray/oplus.jl:451-504``): per charge, the tensors' sector
    ranges are concatenated in list order; every other leg is shared."""
    dims = {}
    for t in tensors:
        for q, d in t.legs[leg].sectors.items():
            dims[q] = dims.get(q, 0) + d
    legs = []
    for i in range(tensors[0].rank):
        if i == leg:
            legs.append(Leg(tensors[0].legs[leg].dir, dims))
        else:
            acc = tensors[0].legs[i]
            for t in tensors[1:]:
                acc = merge_legs(acc, t.legs[i])
            legs.append(acc)
    out = {}
    offset = {q: 0 for q in dims}
    for t in tensors:
        for key, v in t.blocks.items():
            q = key[leg]
            if key not in out:
                shape = [legs[i].sectors[key[i]] for i in range(len(legs))]
                out[key] = np.zeros(shape, dtype=np.complex128)
            sl = [slice(None)] * len(legs)
            sl[leg] = slice(offset[q], offset[q] + v.shape[leg])
            out[key][tuple(sl)] = v
        for q, d in t.legs[leg].sectors.items():
            offset[q] += d
    return BT(legs, out)


def trim_per_sector(t: BT, leg: int, counts) -> BT | None:
    """Keep the leading ``counts[q]`` entries of each sector ``q`` of ``leg``; drop the rest
    (``truncation.jl:283-288``). ``None`` when nothing is kept."""
    if not any(c > 0 for c in counts.values()):
        return None
    keep = {q: min(counts.get(q, 0), d) for q, d in t.legs[leg].sectors.items()}
    keep = {q: c for q, c in keep.items() if c > 0}
    legs = list(t.legs)
    legs[leg] = Leg(t.legs[leg].dir, keep)
    out = {}
    for key, v in t.blocks.items():
        c = keep.get(key[leg], 0)
        if c == 0:
            continue
        sl = [slice(None)] * t.rank
        sl[leg] = slice(0, c)
        out[key] = np.ascontiguousarray(v[tuple(sl)])
    return BT(legs, out)


def trim_total(t: BT, leg: int, column_count: int) -> BT | None:
    """At most ``column_count`` entries of ``leg``, walking sectors in ascending charge order
    (``cbe.jl:219-236``)."""
    if column_count <= 0:
        return None
    if t.dim(leg) <= column_count:
        return t
    left = column_count
    keep = {}
    for q, d in t.legs[leg].sectors.items():
        keep[q] = min(d, left)
        left -= keep[q]
    if not any(v > 0 for v in keep.values()):
        return None
    return trim_per_sector(t, leg, keep)


# ── SVD with Telum's selection ───────────────────────────────────────────────────────────────


@dataclass
class SVDResult:
    U: BT
    S: dict  # charge -> kept singular values (descending within the sector)
    Vd: BT
    kept: list = field(default_factory=list)  # (sigma, degeneracy, charge, index)
    trunc: list = field(default_factory=list)

    def US(self) -> BT:
        """``U * S``."""
        return BT(
            self.U.legs,
            {k: v * self.S[k[-1]] for k, v in self.U.blocks.items()},
        )

    def SVd(self) -> BT:
        """``S * Vd``."""
        out = {}
        for k, v in self.Vd.blocks.items():
            s = self.S[k[0]]
            out[k] = v * s.reshape((-1,) + (1,) * (v.ndim - 1))
        return BT(self.Vd.legs, out)


def sector_matrix(t: BT, left):
    """Group ``t``'s blocks by the charge flowing through the split.

    Returns ``{c: (row_keys, col_keys, M)}`` where ``c = -sum_{i in left} dir_i q_i``, rows are
    the left charge tuples in ascending order, columns the right ones, and ``M`` the dense sector
    matrix (rows in C order within each block)."""
    left = tuple(left)
    right = tuple(i for i in range(t.rank) if i not in left)
    groups = {}
    for key in t.blocks:
        c = -sum(t.legs[i].dir * key[i] for i in left)
        lk = tuple(key[i] for i in left)
        rk = tuple(key[i] for i in right)
        g = groups.setdefault(c, (set(), set()))
        g[0].add(lk)
        g[1].add(rk)
    out = {}
    for c in sorted(groups):
        rows = sorted(groups[c][0])
        cols = sorted(groups[c][1])
        rdim = [int(np.prod([t.legs[i].sectors[q] for i, q in zip(left, rk)])) for rk in rows]
        cdim = [int(np.prod([t.legs[i].sectors[q] for i, q in zip(right, ck)])) for ck in cols]
        M = np.zeros((sum(rdim), sum(cdim)), dtype=np.complex128)
        roff = np.concatenate([[0], np.cumsum(rdim)])
        coff = np.concatenate([[0], np.cumsum(cdim)])
        for ri, rk in enumerate(rows):
            for ci, ck in enumerate(cols):
                key = [0] * t.rank
                for i, q in zip(left, rk):
                    key[i] = q
                for i, q in zip(right, ck):
                    key[i] = q
                key = tuple(key)
                blk = t.blocks.get(key)
                if blk is None:
                    continue
                m = blk.transpose(left + right).reshape(rdim[ri], cdim[ci])
                M[roff[ri]:roff[ri + 1], coff[ci]:coff[ci + 1]] = m
        out[c] = (rows, cols, rdim, cdim, M)
    return out


def _fix_phases(U, Vh):
    """Fix the free phase of each singular pair: ``f = sum_i U[i,k] / (i + phi)`` is made real
    and positive. The functional has no rational zeros, so structured vectors do not sit on its
    null space; two SVDs that agree to roundoff then agree on their vectors too."""
    m = U.shape[0]
    c = 1.0 / (np.arange(m, dtype=np.float64) + _PHI)
    f = c @ U
    a = np.abs(f)
    ph = np.where(a > 0, np.conj(f) / np.where(a > 0, a, 1.0), 1.0)
    return U * ph[None, :], Vh * np.conj(ph)[:, None]


def svd(t: BT, left, cutoff: float = 0.0, nkeep: int | None = None) -> SVDResult:
    """Symmetry-adapted SVD over the split ``left | rest`` (``svd.jl:1-40``, selection
    ``svd.jl:1825-1921``): ``U`` = (left legs..., bond +1), ``Vd`` = (bond -1, right legs...),
    bond charge ``c = -sum_left dir*q``."""
    left = tuple(left)
    right = tuple(i for i in range(t.rank) if i not in left)
    sm = sector_matrix(t, left)
    per = {}
    entries = []
    smax = 0.0
    for c, (rows, cols, rdim, cdim, M) in sm.items():
        u, s, vh = np.linalg.svd(M, full_matrices=False)
        u, vh = _fix_phases(u, vh)
        per[c] = (rows, cols, rdim, cdim, u, s, vh)
        for j, sv in enumerate(s):
            smax = max(smax, float(sv))
            entries.append((float(sv), c, j))
    thresh = cutoff * smax
    sel = [e for e in entries if e[0] > thresh]
    sel.sort(key=lambda e: -e[0])  # Python's sort is stable, like MergeSort
    if nkeep is not None:
        sel = sel[: max(nkeep, 0)]
    chosen = {}
    for sv, c, j in sel:
        chosen.setdefault(c, []).append(j)
    for c in chosen:
        chosen[c].sort()
    selected = {(c, j) for _, c, j in sel}
    full = sorted(entries, key=lambda e: -e[0])
    kept, trunc = [], []
    for sv, c, j in full:
        (kept if (c, j) in selected else trunc).append((sv, 1, c, j))
    # build U, S, Vd
    bond = {c: len(js) for c, js in chosen.items()}
    ulegs = [t.legs[i] for i in left] + [Leg(+1, bond)]
    vlegs = [Leg(-1, bond)] + [t.legs[i] for i in right]
    ublocks, vblocks, S = {}, {}, {}
    for c, js in chosen.items():
        rows, cols, rdim, cdim, u, s, vh = per[c]
        js = np.asarray(js)
        S[c] = s[js].copy()
        roff = 0
        for rk, rd in zip(rows, rdim):
            blk = u[roff:roff + rd, js]
            roff += rd
            shape = [t.legs[i].sectors[q] for i, q in zip(left, rk)] + [len(js)]
            ublocks[tuple(rk) + (c,)] = np.ascontiguousarray(blk.reshape(shape))
        coff = 0
        for ck, cd in zip(cols, cdim):
            blk = vh[js, coff:coff + cd]
            coff += cd
            shape = [len(js)] + [t.legs[i].sectors[q] for i, q in zip(right, ck)]
            vblocks[(c,) + tuple(ck)] = np.ascontiguousarray(blk.reshape(shape))
    return SVDResult(BT(ulegs, ublocks), S, BT(vlegs, vblocks), kept, trunc)


def sq_weight(lst) -> float:
    """``sum sigma^2 * deg`` of an SVD list (``truncation.jl:163``)."""
    return sum(float(s) ** 2 * float(d) for (s, d, _, _) in lst)


def trunc_weight(res: SVDResult) -> float:
    """``sqrt(sum_cut sigma^2 / sum_all sigma^2)`` (``truncation.jl:166-170``)."""
    kept, cut = sq_weight(res.kept), sq_weight(res.trunc)
    tot = kept + cut
    return 0.0 if tot == 0.0 else math.sqrt(cut / tot)


# ── canonical Gaussian draws ─────────────────────────────────────────────────────────────────


def complex_normals(rng: np.random.Generator, n: int) -> np.ndarray:
    """``n`` complex normals with ``E|z|^2 = 1`` (Julia's ``randn(ComplexF64)``): real and
    imaginary parts are consecutive draws of ``rng.standard_normal`` scaled by ``sqrt(1/2)``."""
    x = rng.standard_normal(2 * n)
    return (x[0::2] + 1j * x[1::2]) * math.sqrt(0.5)


def fused_sectors(la: Leg, lb: Leg, out_dir: int):
    """Charges of the fused space ``la (x) lb`` seen by a new leg of arrow ``out_dir``:
    ``{c: [(qa, qb), ...]}`` with the pairs ascending, ``c`` chosen so that
    ``la.dir*qa + lb.dir*qb + out_dir*c == 0``."""
    out = {}
    for qa in la.sectors:
        for qb in lb.sectors:
            c = -(la.dir * qa + lb.dir * qb) * out_dir
            out.setdefault(c, []).append((qa, qb))
    return {c: sorted(v) for c, v in sorted(out.items())}


def gaussian_fused(rng, la: Leg, lb: Leg, cols: dict, new_first: bool) -> BT | None:
    """A Gaussian tensor on the fused space ``la (x) lb`` with ``cols[c]`` columns in sector
    ``c`` (``cbe.jl:156-178`` followed by ``_trim_per_sector``).

    Draw order (shared with the engine's host side): sectors ``c`` ascending; per sector one
    C-ordered ``(n_c, cols[c])`` matrix, its rows the ``(qa, qb)`` pairs ascending, each pair
    ``dim(qa)*dim(qb)`` rows in C order. ``new_first=False`` gives legs ``(la, lb, g:+1)``
    (a left frame's layout), ``True`` gives ``(g:-1, la, lb)`` (a right frame's)."""
    return _fused(la, lb, cols, new_first, lambda n, k: complex_normals(rng, n * k).reshape(n, k))


def identity_fused(la: Leg, lb: Leg, new_first: bool) -> BT | None:
    """The complete fused basis of ``la (x) lb`` (``fusion_basis``, used by ``_dd_probe(...;
    exact = true)``, ``dd_cbe.jl:140-148``): in every fused sector ``c`` the ``n_c x n_c`` identity,
    rows and columns both in the ``(qa, qb)``-pair order of :func:`gaussian_fused`, same layouts."""
    fs = fused_sectors(la, lb, -1 if new_first else +1)
    cols = {c: sum(la.sectors[qa] * lb.sectors[qb] for qa, qb in pairs) for c, pairs in fs.items()}
    return _fused(la, lb, cols, new_first, lambda n, k: np.eye(n, k, dtype=np.complex128))


def _fused(la: Leg, lb: Leg, cols: dict, new_first: bool, matrix) -> BT | None:
    gdir = -1 if new_first else +1
    fs = fused_sectors(la, lb, gdir)
    gsec = {c: cols.get(c, 0) for c in fs if cols.get(c, 0) > 0}
    if not gsec:
        return None
    glegs = Leg(gdir, gsec)
    legs = [glegs, la, lb] if new_first else [la, lb, glegs]
    blocks = {}
    for c in fs:
        k = gsec.get(c, 0)
        if k == 0:
            continue
        pairs = fs[c]
        rd = [la.sectors[qa] * lb.sectors[qb] for qa, qb in pairs]
        n = sum(rd)
        M = matrix(n, k)
        off = 0
        for (qa, qb), r in zip(pairs, rd):
            blk = M[off:off + r].reshape(la.sectors[qa], lb.sectors[qb], k)
            off += r
            if new_first:
                blocks[(c, qa, qb)] = np.ascontiguousarray(blk.transpose(2, 0, 1))
            else:
                blocks[(qa, qb, c)] = np.ascontiguousarray(blk)
    return BT(legs, blocks)


def to_dense(t: BT) -> np.ndarray:
    """The tensor as a dense array, legs expanded sector by sector in ascending charge order."""
    offs = []
    for l in t.legs:
        o, acc = {}, 0
        for q, d in l.sectors.items():
            o[q] = acc
            acc += d
        offs.append(o)
    out = np.zeros([l.dim() for l in t.legs], dtype=np.complex128)
    for key, v in t.blocks.items():
        sl = tuple(slice(offs[i][q], offs[i][q] + v.shape[i]) for i, q in enumerate(key))
        out[sl] += v
    return out
