"""Engine operations against the oracle's block-sparse arithmetic, one by one (GPU).

Each case builds random U(1) block tensors on the host, runs the oracle operation
(``oracle/blocks.py``) and the engine operation through the C-ABI, and compares: contractions
(every operand layout the planner distinguishes), the Telum-selection SVD with its phase
convention, reductions, linear combinations, permutations, direct sums and trims.
"""

import numpy as np
import pytest

from oracle import blocks as OB
from tests.gpu_util import rand_bt, same, to_dev, to_host

pytestmark = pytest.mark.gpu

S3 = {-2: 3, 0: 4, 2: 2}
S2 = {-1: 2, 1: 3}
SS = {-1: 1, 1: 1}


@pytest.fixture(scope="module")
def D():
    from bondupdategalerkin_b200 import build, tensor

    build.build()
    return tensor


def mps_like(rng, L=S3, R=None):
    R = R or {q + s: d for q, d in L.items() for s in (-1, 1)}
    R = {q: (d % 5) + 2 for q, d in R.items()}
    return rand_bt(rng, (-1, -1, +1), (L, SS, R))


@pytest.mark.parametrize("case", range(8))
def test_contract(D, case):
    rng = np.random.default_rng(100 + case)
    A = mps_like(rng)
    # env-like (bra:-1, w:+1, ket:+1) contracted on its ket with A's left link
    E = rand_bt(rng, (-1, +1, +1), ({q: 3 for q in range(-4, 5)}, {-2: 1, 0: 3, 2: 1}, A.legs[0].sectors))
    patterns = [
        (E, (2,), A, (0,), False, False),           # tail x head
        (A, (0, 1), A, (0, 1), True, False),        # head x head, conj
        (A, (2,), A, (2,), False, True),            # tail x tail, conj
        (A, (1, 2), A, (1, 2), False, True),        # tail x tail (2 legs)
        (A, (0, 2), A, (0, 2), True, False),        # split legs -> permute both
        (E, (0, 2), E, (0, 2), True, False),
        (A, (1,), E, (1,), False, False) if False else (A, (0,), E, (2,), False, False),  # head x tail
        (E, (1,), E, (1,), True, False),            # middle legs -> permute
    ]
    a, ia, b, ib, ca, cb = patterns[case]
    want = OB.contract(a, ia, b, ib, conja=ca, conjb=cb)
    got = to_host(D.contract(to_dev(a), ia, to_dev(b), ib, conja=ca, conjb=cb))
    assert sorted(got.blocks) == sorted(want.blocks)
    assert same(got, want) < 1e-13


def _big_cases(rng):
    """Contractions at the block sizes maxdim 256-512 allows: sector dims 33-256, contracted
    extents 17, 100 and 512, and 3- and 4-dim strided index groups on either operand."""
    SS2 = {-1: 1, 1: 1}
    A = rand_bt(rng, (-1, -1, +1), ({0: 64, 2: 33}, SS2, {-1: 64, 1: 128, 3: 33}), 1.0)
    E = rand_bt(rng, (-1, +1, +1), ({q: 128 for q in (-2, 0, 2, 4)}, {-2: 1, 0: 3, 2: 1},
                                    {0: 64, 2: 33}), 1.0)
    M = rand_bt(rng, (-1, +1), ({0: 256, 2: 128, 4: 64}, {0: 17, 2: 100, 4: 512}), 1.0)
    N = rand_bt(rng, (-1, +1), ({0: 17, 2: 100, 4: 512}, {0: 64, 2: 33, 4: 256}), 1.0)
    sec = {-2: 3, 0: 5, 2: 2}
    P = rand_bt(rng, (+1, -1, +1, -1, +1), (sec,) * 5, 1.0)
    Q = rand_bt(rng, (-1, +1, -1, +1, -1), (sec,) * 5, 1.0)
    S = rand_bt(rng, (+1, -1, +1), (sec, {0: 33, 2: 64}, {-2: 4, 0: 5, 2: 6}), 1.0)
    R4 = rand_bt(rng, (-1, +1, -1, +1), ({0: 33, 2: 40}, {0: 2, 2: 3}, {0: 4, 2: 5}, {0: 66, 2: 70, 4: 9}),
                 1.0)
    return [
        (A, (0, 1), A, (0, 1), True, False),      # K = 33/64, outputs up to 128 x 128
        (E, (2,), A, (0,), False, False),          # env x site, K = 33/64, 128-row outputs
        (M, (1,), N, (0,), False, False),          # K = 17, 100, 512 on 256/128/64 x 64/33/256
        (N, (0,), M, (1,), True, True),            # the same pairs transposed and conjugated
        (P, (0, 2, 3, 4), Q, (4, 0, 1, 2), False, False),  # 4-dim strided contracted groups
        (P, (1,), S, (0,), False, False),          # a 4-dim free group (rows) x 2 free legs
        (R4, (0, 3), R4, (0, 3), True, False),     # split contracted legs, 2-dim free group
        (R4, (3,), R4, (3,), False, True),         # 3-dim free groups, K up to 70
    ]


@pytest.mark.parametrize("case", range(8))
def test_contract_large_blocks(D, case):
    rng = np.random.default_rng(500 + case)
    a, ia, b, ib, ca, cb = _big_cases(rng)[case]
    want = OB.contract(a, ia, b, ib, conja=ca, conjb=cb)
    got = to_host(D.contract(to_dev(a), ia, to_dev(b), ib, conja=ca, conjb=cb))
    assert sorted(got.blocks) == sorted(want.blocks)
    assert same(got, want) < 1e-13


@pytest.mark.parametrize("left,cutoff,nkeep", [((0, 1), 0.0, None), ((0,), 0.0, None),
                                                ((0, 1), 1e-1, None), ((0, 1), 0.0, 5),
                                                ((1, 2), 0.0, None), ((0, 2), 1e-3, 7)])
def test_svd(D, left, cutoff, nkeep):
    rng = np.random.default_rng(7)
    A = mps_like(rng)
    want = OB.svd(A, left, cutoff=cutoff, nkeep=nkeep)
    got = D.svd(to_dev(A), left, cutoff=cutoff, nkeep=nkeep)
    assert len(got.kept) == len(want.kept) and len(got.trunc) == len(want.trunc)
    for (s1, _, q1, _), (s2, _, q2, _) in zip(got.kept + got.trunc, want.kept + want.trunc):
        assert q1 == q2 and abs(s1 - s2) <= 1e-13 * max(1.0, want.kept[0][0])
    assert same(to_host(got.U), want.U) < 1e-11
    assert same(to_host(got.Vd), want.Vd) < 1e-11
    rec = OB.contract(to_host(got.US()), (len(left),), to_host(got.Vd), (0,))
    ref = OB.contract(want.US(), (len(left),), want.Vd, (0,))
    assert same(rec, ref) < 1e-12


def test_svd_wide_and_big(D):
    rng = np.random.default_rng(11)
    A = rand_bt(rng, (-1, -1, +1), ({0: 40}, {0: 2}, {0: 130}))   # 80 x 130: transposed path
    want = OB.svd(A, (0, 1))
    got = D.svd(to_dev(A), (0, 1))
    assert np.allclose([s for s, *_ in got.kept], [s for s, *_ in want.kept], rtol=1e-12)
    assert same(to_host(got.U), want.U) < 1e-10
    B = rand_bt(rng, (-1, -1, +1), ({0: 200}, {0: 2}, {0: 150}))  # global-memory path
    want = OB.svd(B, (0, 1))
    got = D.svd(to_dev(B), (0, 1))
    assert np.allclose([s for s, *_ in got.kept], [s for s, *_ in want.kept], rtol=1e-12)
    assert same(to_host(got.U), want.U) < 1e-10


def test_reductions_and_lincomb(D):
    rng = np.random.default_rng(3)
    A = mps_like(rng)
    B = OB.BT(A.legs, {k: v * (1 + 0.5j) + 0.1 for k, v in A.blocks.items() if rng.random() < 0.7})
    dA, dB = to_dev(A), to_dev(B)
    assert abs(D.norm(dA) - OB.norm(A)) < 1e-12 * OB.norm(A)
    assert abs(D.inner(dA, dB) - OB.inner(A, B)) < 1e-12 * OB.norm(A) * OB.norm(B)
    many = D.inner_many([dA, dB, dA], dB)
    assert abs(many[1] - OB.inner(B, B)) < 1e-12 * OB.norm(B) ** 2
    lc = to_host(D.lincomb([(0.3 - 1j, dA), (2.0, dB), (-1.0, dA)]))
    want = OB.add(OB.add(OB.scale(A, 0.3 - 1j), B, 1.0, 2.0), A, 1.0, -1.0)
    assert same(lc, want) < 1e-13


def test_permute_conj_flip_oplus_trim_scale(D):
    rng = np.random.default_rng(5)
    A = mps_like(rng)
    dA = to_dev(A)
    assert same(to_host(D.permute(dA, (2, 0, 1))), OB.permute(A, (2, 0, 1))) < 1e-15
    assert same(to_host(D.conj(dA)), OB.conj(A)) < 1e-15
    B = mps_like(np.random.default_rng(6), L=S3)
    B = OB.BT([A.legs[0], A.legs[1], B.legs[2]], {k: v for k, v in B.blocks.items()
                                                   if k[0] in A.legs[0].sectors})
    got = to_host(D.oplus([dA, to_dev(B)], 2))
    assert same(got, OB.oplus([A, B], 2)) < 1e-15
    counts = {q: 1 + i % 2 for i, q in enumerate(A.legs[2].sectors)}
    assert same(to_host(D.trim_per_sector(dA, 2, counts)), OB.trim_per_sector(A, 2, counts)) < 1e-15
    res = OB.svd(A, (0, 1))
    w = {q: np.arange(1, d + 1, dtype=float) for q, d in A.legs[2].sectors.items()}
    got = to_host(D.scale_leg(dA, 2, w))
    want = OB.BT(A.legs, {k: v * w[k[2]][None, None, :] for k, v in A.blocks.items()})
    assert same(got, want) < 1e-15
    fl = to_host(D.flip_leg(dA, 2))
    assert fl.legs[2].dir == -A.legs[2].dir
    assert all(np.array_equal(fl.blocks[(k[0], k[1], -k[2])], v) for k, v in A.blocks.items())


def test_gaussian_matches_oracle_draws(D):
    la, lb = D.Leg(-1, {-1: 2, 1: 3}), D.Leg(-1, {-1: 1, 1: 1})
    cols = {-2: 1, 0: 3, 2: 2}
    got = to_host(D.gaussian_fused(np.random.default_rng(9), la, lb, cols, new_first=False))
    want = OB.gaussian_fused(np.random.default_rng(9), OB.Leg(-1, la.sectors), OB.Leg(-1, lb.sectors),
                             cols, new_first=False)
    assert same(got, want) == 0.0


def _isometry_err(U, cols):
    """max |U^H U - I| over the sector matrices of an isometry whose columns are leg `cols`."""
    err = 0.0
    for c, (_, _, _, _, M) in OB.sector_matrix(U, tuple(i for i in range(len(U.legs)) if i != cols)).items():
        err = max(err, float(np.max(np.abs(M.conj().T @ M - np.eye(M.shape[1])))))
    return err


def test_svd_rank_deficient(D):
    """Numerically zero singular values (rank-deficient sectors, a column of rounding noise, an
    exactly zero column): the Jacobi SVD converges, keeps U and V isometries, and matches the
    non-negligible singular triples of LAPACK."""
    # the 3 x 3 sector met in a random-product-state step: a singular value of 5e-168
    legs = [OB.Leg(-1, {-3: 3}), OB.Leg(-1, {-1: 1, 1: 1}), OB.Leg(+1, {-4: 1, -2: 2})]
    blk1 = np.array([0.01, 0.0, 0.0], dtype=np.complex128).reshape(3, 1, 1)
    blk2 = np.array([[7.12816426e-2 - 4.22641607e-36j, 5.55681849e-3 + 1.20924481e-36j],
                     [-1.85546035e-2 + 6.83848485e-36j, 2.13477560e-2 - 1.95659921e-36j],
                     [7.20192925e-186 + 1.21465880e-151j, 3.04118525e-185 - 1.39750977e-151j]])
    A = OB.BT(legs, {(-3, -1, -4): blk1, (-3, 1, -2): blk2.reshape(3, 1, 2)})
    rng = np.random.default_rng(13)
    left = rng.standard_normal((40, 6)) + 1j * rng.standard_normal((40, 6))
    right = rng.standard_normal((6, 2, 25)) + 1j * rng.standard_normal((6, 2, 25))
    lowrank = np.einsum("ak,kbc->abc", left, right)  # 40 x 50, rank 6
    lowrank[:, :, 3] = 0.0                           # and an exactly zero column
    B = OB.BT([OB.Leg(-1, {0: 40}), OB.Leg(-1, {0: 2}), OB.Leg(+1, {0: 25})], {(0, 0, 0): lowrank})
    for T, split in ((A, (0,)), (B, (0,)), (B, (0, 1))):
        want = OB.svd(T, split)
        got = D.svd(to_dev(T), split)
        gs = np.array([s for s, *_ in got.kept])
        ws = np.array([s for s, *_ in want.kept])
        big = ws > 1e-12 * ws[0]
        assert np.allclose(gs[: big.sum()], ws[big], rtol=1e-12, atol=0)
        assert np.all(gs[big.sum():] <= 1e-12 * ws[0])  # the numerically zero ones stay tiny
        Uh, Vh = to_host(got.U), to_host(got.Vd)
        assert _isometry_err(Uh, len(split)) < 1e-12
        rec = OB.contract(to_host(got.US()), (len(split),), Vh, (0,))
        assert same(rec, T) < 1e-13


def _qr_cases(rng):
    """(tensor, leg, ref_dir, thr) cases for the pivoted thin QR."""
    A = mps_like(rng)
    # a sketch-like tensor whose column sectors are wider than their row space (m < n), with
    # graded column norms so the pivot order is not the storage order
    W = rand_bt(rng, (-1, -1, +1), ({0: 2, 2: 1}, SS, {-1: 9, 1: 7, 3: 5}), p_present=1.0)
    for k, v in W.blocks.items():
        W.blocks[k] = v * np.geomspace(1.0, 1e-3, v.shape[2])[None, None, :]
    # rank-deficient sector: column 4 of sector +1 is twice column 0
    legs = [OB.Leg(-1, {0: 6, 2: 4}), OB.Leg(-1, {-1: 1, 1: 1}), OB.Leg(+1, {-1: 3, 1: 5})]
    blocks = {}
    for key in [(0, -1, -1), (0, 1, 1), (2, -1, 1)]:
        shp = tuple(l.sectors[q] for l, q in zip(legs, key))
        blocks[key] = rng.standard_normal(shp) + 1j * rng.standard_normal(shp)
    for key in [(0, 1, 1), (2, -1, 1)]:
        blocks[key][..., 4] = blocks[key][..., 0] * 2.0
    R = OB.BT(legs, blocks)
    # columns of norm ~ 1 with some pivots below 1/sqrt(2): the second-pass keep rule
    N = mps_like(rng)
    for k, v in N.blocks.items():
        N.blocks[k] = v / max(np.linalg.norm(v), 1e-300) * 0.9
    return [(A, 2, +1, 1e-10), (A, 2, -1, 1e-10), (A, 0, -1, 1e-10), (A, 0, +1, 1e-3),
            (W, 2, +1, 1e-10), (W, 2, +1, 1e-2), (R, 2, +1, 1e-10), (N, 2, +1, 1 / np.sqrt(2))]


@pytest.mark.parametrize("case", range(8))
def test_thin_qr_matches_oracle(D, case):
    """The device column-pivoted Householder QR against LAPACK geqp3 (scipy) with the phase that
    makes R_kk real positive: same kept ranks per sector, same basis vectors."""
    from oracle import cbe as OC

    rng = np.random.default_rng(700 + case)
    T, leg, ref, thr = _qr_cases(rng)[case]
    want = OC.thin_qr(T, leg, ref, thr)
    got = D.thin_qr(to_dev(T), leg, ref, thr)
    if want is None:
        assert got is None
        return
    got = to_host(got)
    assert got.legs[leg].dir == want.legs[leg].dir
    assert got.legs[leg].sectors == want.legs[leg].sectors
    assert sorted(got.blocks) == sorted(want.blocks)
    assert same(got, want) < 1e-11
