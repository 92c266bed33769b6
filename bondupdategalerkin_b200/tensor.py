"""Device-resident block-sparse tensors: the host-side handle type of the B200 engine.

A ``DT`` is an opaque engine tensor (block table on the host, payload in HBM) plus a lazily
fetched copy of its metadata. The operations mirror the block-sparse container the reference's
BUG step is written against (Telum's ``TLArray``: ``contract``, ``svd``, ``norm``, ``oplus``,
``getsub``...; ``deps/Telum/src/Telum.jl:97-117``), with the same leg/arrow conventions:

* a leg is an arrow (+1 out, -1 in) and an ascending ``charge -> dim`` map;
* a block keyed by one charge per leg exists only if ``sum_i dir_i q_i == 0``;
* MPS sites are ``(link_l:-1, site:-1, link_r:+1)``, MPO tensors ``(w_l:-1, s_in:+1, s_out:-1, w_r:+1)``.

Every numeric operation runs in the engine (``libbug_b200.so``); this module only moves handles,
metadata and the host-drawn Gaussian probes.
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field

import numpy as np

from . import _engine as E

_vp = ctypes.c_void_p
_ip = ctypes.POINTER(ctypes.c_int)
_dp = ctypes.POINTER(ctypes.c_double)


def _ints(a):
    arr = np.ascontiguousarray(np.asarray(a, dtype=np.int32))
    return arr, arr.ctypes.data_as(_ip)


def _dbls(a):
    arr = np.ascontiguousarray(np.asarray(a, dtype=np.float64))
    return arr, arr.ctypes.data_as(_dp)


class Leg:
    """An arrow and an ascending ``charge -> dim`` map."""

    __slots__ = ("dir", "sectors")

    def __init__(self, dir: int, sectors):
        self.dir = int(dir)
        self.sectors = {int(q): int(d) for q, d in sorted(dict(sectors).items()) if int(d) > 0}

    def dim(self) -> int:
        return sum(self.sectors.values())

    def flip(self) -> "Leg":
        return Leg(-self.dir, self.sectors)

    def __repr__(self):
        return f"Leg({self.dir:+d}, {self.sectors})"


class DT:
    """Handle to an engine tensor. Immutable; freed when the handle is dropped."""

    __slots__ = ("h", "ctx", "_legs", "_keys", "_nelem")

    def __init__(self, ctx: E.Context, h: _vp):
        self.h = h
        self.ctx = ctx
        self._legs = None
        self._keys = None
        self._nelem = None

    def __del__(self):
        h = getattr(self, "h", None)
        if h is not None and h.value:
            try:
                self.ctx.lib.bug_tensor_free(self.ctx.h, h)
            except Exception:
                pass
            self.h = None

    def _fetch(self):
        lib = self.ctx.lib
        rank, nb, ns = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        ne = ctypes.c_int64()
        E.check(lib.bug_tensor_shape(self.h, ctypes.byref(rank), ctypes.byref(nb), ctypes.byref(ne),
                                     ctypes.byref(ns)))
        r, nb, ns = rank.value, nb.value, ns.value
        dirs = np.zeros(max(r, 1), np.int32)
        nsec = np.zeros(max(r, 1), np.int32)
        ch = np.zeros(max(ns, 1), np.int32)
        dm = np.zeros(max(ns, 1), np.int32)
        keys = np.zeros(max(nb * r, 1), np.int32)
        E.check(lib.bug_tensor_meta(self.h, dirs.ctypes.data_as(_ip), nsec.ctypes.data_as(_ip),
                                    ch.ctypes.data_as(_ip), dm.ctypes.data_as(_ip),
                                    keys.ctypes.data_as(_ip)))
        legs, p = [], 0
        for l in range(r):
            n = int(nsec[l])
            legs.append(Leg(int(dirs[l]), {int(ch[p + i]): int(dm[p + i]) for i in range(n)}))
            p += n
        self._legs = legs
        self._keys = [tuple(int(x) for x in keys[b * r:(b + 1) * r]) for b in range(nb)]
        self._nelem = int(ne.value)

    @property
    def legs(self):
        if self._legs is None:
            self._fetch()
        return self._legs

    @property
    def keys(self):
        if self._keys is None:
            self._fetch()
        return self._keys

    @property
    def nelem(self) -> int:
        if self._nelem is None:
            self._fetch()
        return self._nelem

    @property
    def rank(self) -> int:
        return len(self.legs)

    def dim(self, leg: int) -> int:
        return self.legs[leg].dim()

    def elements(self) -> int:
        return self.nelem

    def __repr__(self):
        return f"DT(legs={self.legs}, nblocks={len(self.keys)})"


def _new(ctx, h) -> DT:
    return DT(ctx, h)


# ── host <-> device ──────────────────────────────────────────────────────────────────────────


def from_blocks(legs, blocks: dict, ctx: E.Context | None = None) -> DT:
    """Create an engine tensor from host blocks (``key -> ndarray``) and upload the payload."""
    ctx = ctx or E.context()
    rank = len(legs)
    keys = sorted(blocks)
    # one int32 array carries the arrows, sector counts, charges, dims and keys (views into it)
    nsec = [len(l.sectors) for l in legs]
    ns = sum(nsec)
    meta = np.empty(2 * rank + 2 * ns + rank * len(keys) + 1, dtype=np.int32)
    meta[:rank] = [l.dir for l in legs]
    meta[rank:2 * rank] = nsec
    p = 2 * rank
    for l in legs:
        k = len(l.sectors)
        meta[p:p + k] = list(l.sectors)
        meta[p + ns:p + ns + k] = list(l.sectors.values())
        p += k
    p = 2 * rank + 2 * ns
    if keys:
        meta[p:p + rank * len(keys)] = np.array(keys, dtype=np.int32).reshape(-1)
    base = meta.ctypes.data
    i4 = 4

    def at(off):
        return ctypes.cast(base + i4 * off, _ip)

    h = _vp()
    E.check(ctx.lib.bug_tensor_create(ctx.h, rank, at(0), at(rank), at(2 * rank), at(2 * rank + ns),
                                      len(keys), at(p), ctypes.byref(h)))
    t = DT(ctx, h)
    if keys:
        data = np.concatenate([blocks[k].reshape(-1) for k in keys]).astype(np.complex128, copy=False)
        E.check(ctx.lib.bug_tensor_upload(ctx.h, h, data.ctypes.data_as(_dp), data.size))
    return t


def to_blocks(t: DT):
    """Download: ``(legs, {key: ndarray})``."""
    legs, keys = t.legs, t.keys
    data = np.zeros(max(t.nelem, 1), dtype=np.complex128)
    E.check(t.ctx.lib.bug_tensor_download(t.ctx.h, t.h, data.ctypes.data_as(_dp), t.nelem))
    out, off = {}, 0
    for k in keys:
        shape = tuple(legs[i].sectors[q] for i, q in enumerate(k))
        n = int(np.prod(shape))
        out[k] = data[off:off + n].reshape(shape).copy()
        off += n
    return legs, out


# ── algebra ──────────────────────────────────────────────────────────────────────────────────


def contract(a: DT, ia, b: DT, ib, conja: bool = False, conjb: bool = False) -> DT:
    ia, ib = tuple(ia), tuple(ib)
    if len(ia) != len(ib):
        raise ValueError("contract: leg lists differ in length")
    xa, pa = _ints(list(ia) or [0])
    xb, pb = _ints(list(ib) or [0])
    h = _vp()
    E.check(a.ctx.lib.bug_contract(a.ctx.h, a.h, len(ia), pa, b.h, pb, int(conja), int(conjb),
                                   ctypes.byref(h)))
    return DT(a.ctx, h)


@dataclass
class SVDResult:
    U: DT
    S: dict
    Vd: DT
    kept: list = field(default_factory=list)
    trunc: list = field(default_factory=list)

    def US(self) -> DT:
        return scale_leg(self.U, self.U.rank - 1, self.S)

    def SVd(self) -> DT:
        return scale_leg(self.Vd, 0, self.S)


def svd(t: DT, left, cutoff: float = 0.0, nkeep: int | None = None) -> SVDResult:
    """Block-sparse SVD with Telum's selection; see ``bug_svd`` in ``include/bug_b200.h``."""
    left = tuple(left)
    xl, pl = _ints(list(left) or [0])
    cap = max(1, t.nelem)
    sv = np.zeros(cap, np.float64)
    sq = np.zeros(cap, np.int32)
    nall, nk = ctypes.c_int(), ctypes.c_int()
    U, V = _vp(), _vp()
    E.check(t.ctx.lib.bug_svd(t.ctx.h, t.h, len(left), pl, float(cutoff),
                              -1 if nkeep is None else int(nkeep), ctypes.byref(U), ctypes.byref(V),
                              sv.ctypes.data_as(_dp), sq.ctypes.data_as(_ip), cap,
                              ctypes.byref(nall), ctypes.byref(nk)))
    nall, nk = nall.value, nk.value
    kept = [(float(sv[i]), 1, int(sq[i]), i) for i in range(nk)]
    trunc = [(float(sv[i]), 1, int(sq[i]), i) for i in range(nk, nall)]
    S = {}
    for s, _, q, _ in kept:
        S.setdefault(q, []).append(s)
    S = {q: np.asarray(v) for q, v in sorted(S.items())}
    return SVDResult(DT(t.ctx, U), S, DT(t.ctx, V), kept, trunc)


def thin_qr(t: DT, leg: int, ref_dir: int, thr: float):
    """Pivoted thin QR basis of the leg-``leg`` columns per charge sector; see ``bug_thin_qr`` in
    ``include/bug_b200.h``. None when no pivot exceeds ``thr``."""
    h = _vp()
    E.check(t.ctx.lib.bug_thin_qr(t.ctx.h, t.h, int(leg), int(ref_dir), float(thr), ctypes.byref(h)))
    return DT(t.ctx, h) if h.value else None


def scale_leg(t: DT, leg: int, w_by_charge: dict) -> DT:
    L = t.legs[leg]
    w = np.concatenate([np.asarray(w_by_charge[q], dtype=np.float64) for q in L.sectors]) if L.sectors else np.zeros(1)
    xw, pw = _dbls(w)
    h = _vp()
    E.check(t.ctx.lib.bug_scale_leg(t.ctx.h, t.h, leg, pw, ctypes.byref(h)))
    return DT(t.ctx, h)


def norm(t: DT) -> float:
    out = ctypes.c_double()
    E.check(t.ctx.lib.bug_norm2(t.ctx.h, t.h, ctypes.byref(out)))
    return math.sqrt(max(out.value, 0.0))


def inner(a: DT, b: DT) -> complex:
    out = (ctypes.c_double * 2)()
    E.check(a.ctx.lib.bug_inner(a.ctx.h, a.h, b.h, out))
    return complex(out[0], out[1])


def inner_many(vs, w: DT):
    """``[<v_i|w>]`` in one launch."""
    n = len(vs)
    if n == 0:
        return []
    arr = (_vp * n)(*[v.h for v in vs])
    out = np.zeros(2 * n, np.float64)
    E.check(w.ctx.lib.bug_inner_many(w.ctx.h, n, arr, w.h, out.ctypes.data_as(_dp)))
    return [complex(out[2 * i], out[2 * i + 1]) for i in range(n)]


def lincomb(terms) -> DT:
    """``sum c_i t_i`` over the union of the blocks."""
    terms = list(terms)
    n = len(terms)
    coef = np.zeros(2 * n, np.float64)
    for i, (c, _) in enumerate(terms):
        c = complex(c)
        coef[2 * i], coef[2 * i + 1] = c.real, c.imag
    arr = (_vp * n)(*[t.h for _, t in terms])
    h = _vp()
    ctx = terms[0][1].ctx
    E.check(ctx.lib.bug_lincomb(ctx.h, n, coef.ctypes.data_as(_dp), arr, ctypes.byref(h)))
    return DT(ctx, h)


def scale(t: DT, s) -> DT:
    return lincomb([(s, t)])


def add(a: DT, b: DT, alpha=1.0, beta=1.0) -> DT:
    return lincomb([(alpha, a), (beta, b)])


def sub(a: DT, b: DT) -> DT:
    return lincomb([(1.0, a), (-1.0, b)])


def conj(t: DT) -> DT:
    h = _vp()
    E.check(t.ctx.lib.bug_conj(t.ctx.h, t.h, ctypes.byref(h)))
    return DT(t.ctx, h)


def permute(t: DT, perm) -> DT:
    xp, pp = _ints(list(perm))
    h = _vp()
    E.check(t.ctx.lib.bug_permute(t.ctx.h, t.h, pp, ctypes.byref(h)))
    return DT(t.ctx, h)


def flip_leg(t: DT, leg: int) -> DT:
    h = _vp()
    E.check(t.ctx.lib.bug_flip_leg(t.ctx.h, t.h, leg, ctypes.byref(h)))
    return DT(t.ctx, h)


def oplus(tensors, leg: int) -> DT:
    n = len(tensors)
    arr = (_vp * n)(*[t.h for t in tensors])
    h = _vp()
    ctx = tensors[0].ctx
    E.check(ctx.lib.bug_oplus(ctx.h, n, arr, leg, ctypes.byref(h)))
    return DT(ctx, h)


def trim_per_sector(t: DT, leg: int, counts: dict) -> DT | None:
    """Leading ``counts[q]`` entries of each sector ``q`` of ``leg``; ``None`` if nothing kept."""
    if not any(c > 0 for c in counts.values()):
        return None
    cs = [int(counts.get(q, 0)) for q in t.legs[leg].sectors]
    xc, pc = _ints(cs or [0])
    h = _vp()
    E.check(t.ctx.lib.bug_trim(t.ctx.h, t.h, leg, pc, ctypes.byref(h)))
    if not h.value:
        return None
    return DT(t.ctx, h)


def trim_total(t: DT, leg: int, column_count: int) -> DT | None:
    """At most ``column_count`` entries of ``leg``, sectors in ascending charge order."""
    if column_count <= 0:
        return None
    if t.dim(leg) <= column_count:
        return t
    left, keep = column_count, {}
    for q, d in t.legs[leg].sectors.items():
        keep[q] = min(d, left)
        left -= keep[q]
    return trim_per_sector(t, leg, keep)


def sq_weight(lst) -> float:
    return sum(float(s) ** 2 * float(d) for (s, d, _, _) in lst)


def trunc_weight(res: SVDResult) -> float:
    kept, cut = sq_weight(res.kept), sq_weight(res.trunc)
    tot = kept + cut
    return 0.0 if tot == 0.0 else math.sqrt(cut / tot)


# ── host-drawn Gaussian probes ───────────────────────────────────────────────────────────────


def complex_normals(rng: np.random.Generator, n: int) -> np.ndarray:
    """``n`` complex normals with ``E|z|^2 = 1``: consecutive ``standard_normal`` draws as real
    and imaginary parts, scaled by ``sqrt(1/2)`` (``randn(rng, ComplexF64, ...)``,
    ``src/BUG/Randomised/cbe.jl:156-178``)."""
    x = rng.standard_normal(2 * n)
    return (x[0::2] + 1j * x[1::2]) * math.sqrt(0.5)


def fused_sectors(la: Leg, lb: Leg, out_dir: int):
    out = {}
    for qa in la.sectors:
        for qb in lb.sectors:
            c = -(la.dir * qa + lb.dir * qb) * out_dir
            out.setdefault(c, []).append((qa, qb))
    return {c: sorted(v) for c, v in sorted(out.items())}


def gaussian_fused(rng, la: Leg, lb: Leg, cols: dict, new_first: bool, ctx=None) -> DT | None:
    """Draw a sector-graded Gaussian probe on the host and upload it.

    Draw order: sectors ``c`` ascending; per sector one C-ordered ``(n_c, cols[c])`` matrix whose
    rows are the ``(qa, qb)`` pairs ascending, ``dim(qa)*dim(qb)`` rows each in C order. Layout
    ``(la, lb, g:+1)`` or, with ``new_first``, ``(g:-1, la, lb)``."""
    gdir = -1 if new_first else +1
    fs = fused_sectors(la, lb, gdir)
    gsec = {c: cols.get(c, 0) for c in fs if cols.get(c, 0) > 0}
    if not gsec:
        return None
    g = Leg(gdir, gsec)
    legs = [g, la, lb] if new_first else [la, lb, g]
    blocks = {}
    for c in fs:
        k = gsec.get(c, 0)
        if k == 0:
            continue
        pairs = fs[c]
        rd = [la.sectors[qa] * lb.sectors[qb] for qa, qb in pairs]
        n = sum(rd)
        M = complex_normals(rng, n * k).reshape(n, k)
        off = 0
        for (qa, qb), r in zip(pairs, rd):
            blk = M[off:off + r].reshape(la.sectors[qa], lb.sectors[qb], k)
            off += r
            if new_first:
                blocks[(c, qa, qb)] = np.ascontiguousarray(blk.transpose(2, 0, 1))
            else:
                blocks[(qa, qb, c)] = np.ascontiguousarray(blk)
    return from_blocks(legs, blocks, ctx)


# ── many tensors through one flat host layout (bug_tensors_from_host / bug_tensors_to_host) ──


@dataclass
class HostTensors:
    """Tensors in host memory in the engine's flat layout: ``meta`` (int32) holds, per tensor at
    ``meta_off[i]``, its rank, arrows, sector counts, sector charges and dims, block count and
    block keys; ``payload`` (complex128) holds its blocks in key order from ``payload_off[i]``."""

    meta: np.ndarray
    meta_off: np.ndarray
    payload: np.ndarray
    payload_off: np.ndarray

    def __len__(self):
        return len(self.meta_off)

    @property
    def nbytes(self) -> int:
        return int(self.payload.nbytes)


def _i64p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))


def to_host_many(ts, ctx: E.Context | None = None) -> HostTensors:
    """Download tensors into the flat host layout: two engine calls, one synchronisation."""
    ctx = ctx or ts[0].ctx
    n = len(ts)
    arr = (_vp * max(n, 1))(*[t.h.value for t in ts])
    mlen = np.zeros(max(n, 1), np.int64)
    nel = np.zeros(max(n, 1), np.int64)
    E.check(ctx.lib.bug_tensors_layout(n, arr, _i64p(mlen), _i64p(nel)))
    moff = np.zeros(max(n, 1), np.int64)
    poff = np.zeros(max(n, 1), np.int64)
    if n > 1:
        moff[1:n] = np.cumsum(mlen[:n - 1])
        poff[1:n] = np.cumsum(nel[:n - 1])
    meta = np.zeros(max(int(mlen[:n].sum()), 1), np.int32)
    payload = np.zeros(max(int(nel[:n].sum()), 1), np.complex128)
    E.check(ctx.lib.bug_tensors_to_host(ctx.h, n, arr, meta.ctypes.data_as(_ip), _i64p(moff),
                                        payload.ctypes.data_as(_dp), _i64p(poff)))
    return HostTensors(meta, moff[:n], payload, poff[:n])


def from_host_many(ht: HostTensors, ctx: E.Context | None = None) -> list:
    """Create and upload tensors from the flat host layout: one engine call, no wait."""
    ctx = ctx or E.context()
    n = len(ht)
    out = (_vp * max(n, 1))()
    moff = np.ascontiguousarray(ht.meta_off, dtype=np.int64)
    poff = np.ascontiguousarray(ht.payload_off, dtype=np.int64)
    E.check(ctx.lib.bug_tensors_from_host(ctx.h, n, ht.meta.ctypes.data_as(_ip), _i64p(moff),
                                          ht.payload.ctypes.data_as(_dp), _i64p(poff), out))
    return [DT(ctx, _vp(out[i])) for i in range(n)]


def host_from_blocks(tensors) -> HostTensors:
    """The flat host layout of ``(legs, {key: ndarray})`` tensors (as ``to_blocks`` returns)."""
    metas, pays = [], []
    for legs, blocks in tensors:
        keys = sorted(blocks)
        m = [len(legs)] + [l.dir for l in legs] + [len(l.sectors) for l in legs]
        m += [q for l in legs for q in l.sectors] + [d for l in legs for d in l.sectors.values()]
        m += [len(keys)] + [q for k in keys for q in k]
        metas.append(np.array(m, np.int32))
        pays.append(np.concatenate([np.asarray(blocks[k], np.complex128).reshape(-1) for k in keys])
                    if keys else np.zeros(0, np.complex128))
    moff = np.concatenate([[0], np.cumsum([len(m) for m in metas])[:-1]]).astype(np.int64)
    poff = np.concatenate([[0], np.cumsum([len(p) for p in pays])[:-1]]).astype(np.int64)
    meta = np.concatenate(metas) if metas else np.zeros(1, np.int32)
    payload = np.concatenate(pays) if pays else np.zeros(1, np.complex128)
    if payload.size == 0:
        payload = np.zeros(1, np.complex128)
    return HostTensors(meta, moff, payload, poff)


def host_to_blocks(ht: HostTensors) -> list:
    """``(legs, {key: ndarray})`` per tensor of a flat host layout."""
    out = []
    for i in range(len(ht)):
        m = ht.meta[int(ht.meta_off[i]):]
        r = int(m[0])
        dirs, nsec = m[1:1 + r], m[1 + r:1 + 2 * r]
        ns = int(nsec.sum())
        ch, dm = m[1 + 2 * r:1 + 2 * r + ns], m[1 + 2 * r + ns:1 + 2 * r + 2 * ns]
        nb = int(m[1 + 2 * r + 2 * ns])
        keys = m[2 + 2 * r + 2 * ns:2 + 2 * r + 2 * ns + nb * r].reshape(nb, r) if r else []
        legs, p = [], 0
        for l in range(r):
            k = int(nsec[l])
            legs.append(Leg(int(dirs[l]), {int(ch[p + j]): int(dm[p + j]) for j in range(k)}))
            p += k
        blocks, off = {}, int(ht.payload_off[i])
        for row in keys:
            key = tuple(int(x) for x in row)
            shape = tuple(legs[j].sectors[q] for j, q in enumerate(key))
            size = int(np.prod(shape))
            blocks[key] = ht.payload[off:off + size].reshape(shape).copy()
            off += size
        out.append((legs, blocks))
    return out
