"""Helpers shared by the GPU tests: random oracle tensors and host/device conversion."""

import numpy as np

from oracle import blocks as OB


def rand_bt(rng, dirs, sectors, p_present=0.85):
    """A random oracle tensor: legs with the given arrows/sectors, random present blocks."""
    import itertools

    legs = [OB.Leg(d, s) for d, s in zip(dirs, sectors)]
    blocks = {}
    for key in itertools.product(*[list(l.sectors) for l in legs]):
        if sum(l.dir * q for l, q in zip(legs, key)) != 0:
            continue
        if rng.random() > p_present:
            continue
        shape = tuple(l.sectors[q] for l, q in zip(legs, key))
        blocks[key] = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    return OB.BT(legs, blocks)


def to_dev(t, ctx=None):
    from bondupdategalerkin_b200 import tensor as DTm

    legs = [DTm.Leg(l.dir, l.sectors) for l in t.legs]
    return DTm.from_blocks(legs, t.blocks, ctx)


def to_host(d):
    from bondupdategalerkin_b200 import tensor as DTm

    legs, blocks = DTm.to_blocks(d)
    return OB.BT([OB.Leg(l.dir, l.sectors) for l in legs], blocks)


def same(a, b, tol=1e-12):
    """Max abs difference of two oracle tensors over the union of their blocks, relative to the
    larger norm; also checks that legs agree."""
    assert len(a.legs) == len(b.legs)
    for la, lb in zip(a.legs, b.legs):
        assert la.dir == lb.dir and la.sectors == lb.sectors, (la, lb)
    keys = set(a.blocks) | set(b.blocks)
    scale = max(OB.norm(a), OB.norm(b), 1e-300)
    err = 0.0
    for k in keys:
        x = a.blocks.get(k)
        y = b.blocks.get(k)
        if x is None:
            x = np.zeros_like(y)
        if y is None:
            y = np.zeros_like(x)
        err = max(err, float(np.max(np.abs(x - y))) if x.size else 0.0)
    return err / scale


def mps_to_host(psi):
    """Download a device MPS into an oracle MPS (same centre)."""
    from oracle.models import MPS as OMPS

    return OMPS([to_host(t) for t in psi.tensors], psi.center)


def overlap(a, b):
    """<a|b> of two oracle MPS by left-to-right transfer contraction."""
    E = None
    for i in range(1, len(a) + 1):
        if E is None:
            E = OB.contract(a[i], (0, 1), b[i], (0, 1), conja=True)
        else:
            t = OB.contract(E, (0,), a[i], (0,), conjb=True)      # (b_r, s, a_r')
            E = OB.contract(t, (0, 1), b[i], (0, 1))             # (a_r', b_r)
    tot = 0j
    for k, v in E.blocks.items():
        tot += complex(np.sum(v))
    return tot


def fidelity(a, b):
    ab = overlap(a, b)
    return abs(ab) ** 2 / (overlap(a, a).real * overlap(b, b).real)


def perturbed_mpo(mpo, seed, eps=1e-14):
    """The oracle MPO with every core perturbed by eps (relative): another valid compression of
    the same operator, whose runs show which of the oracle's decisions hang on round-off."""
    from oracle.models import MPO

    r = np.random.default_rng(seed)
    return MPO([OB.BT(t.legs, {k: v * (1 + eps * r.standard_normal(v.shape))
                               for k, v in t.blocks.items()}) for t in mpo.tensors])
