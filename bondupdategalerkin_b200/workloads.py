"""Seeded job streams of the batched and served workloads, and their host-side inputs.

* ``batch_specs`` -- 64 independent U(1) XXZ chains advanced together: L drawn from
  {32, 48, 64, 96}, delta uniform in [-1, 1], J = 1, a seeded random product state with total
  S^z = 0, maxdim drawn from {64, 128, 256}, 50 steps of tau = -0.02i at order 2.
* ``served_specs`` -- a stream of jobs with Poisson arrivals (20 jobs/s): 70 % XXZ chains (L uniform
  in [16, 128], delta uniform in [-1, 1], Neel or domain-wall start, maxdim uniform in [32, 512]
  with ``work_ceiling_rule = maxdim`` for Neel starts, 20-200 steps of tau = -0.05i) and 30 %
  Heston fields (8-11 bits per axis, r in [0, 0.05], kappa in [1, 3], theta in [0.04, 0.12], sigma
  in [0.2, 0.6], rho in [-0.9, -0.3], maxdim 32-128, 10-50 steps of tau = 0.02, Arnoldi). With
  ``scale < 1`` the ranges of L, maxdim, bits and steps shrink toward their lower ends by that
  factor (``scale = 1`` is the stream as specified).

Every job carries its own seed (fixed per job id), so the stream and each job's result are
reproducible. ``job_inputs`` turns a spec into host blocks for ``server.Server.submit``.
"""

from __future__ import annotations

import numpy as np


def batch_specs(n: int = 64, seed: int = 2024):
    rng = np.random.default_rng(seed)
    out = []
    for j in range(n):
        L = int(rng.choice([32, 48, 64, 96]))
        delta = float(rng.uniform(-1.0, 1.0))
        spins = ["up"] * (L // 2) + ["down"] * (L - L // 2)
        rng.shuffle(spins)
        out.append(dict(kind="xxz", L=L, delta=delta, spins=spins, tau=-0.02j, nsteps=50,
                        seed=seed * 1000 + j,
                        kw=dict(order=2, maxdim=int(rng.choice([64, 128, 256])))))
    return out


def _scaled_int(rng, lo, hi, scale):
    return int(rng.integers(lo, lo + max(int(round((hi - lo) * scale)), 0) + 1))


def served_specs(n: int = 1000, rate: float = 20.0, seed: int = 7, scale: float = 1.0):
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for j in range(n):
        t += float(rng.exponential(1.0 / rate))
        jseed = seed * 100000 + j
        if rng.random() < 0.7:
            L = _scaled_int(rng, 16, 128, scale)
            neel = bool(rng.random() < 0.5)
            spins = (["up" if i % 2 == 0 else "down" for i in range(L)] if neel
                     else ["up" if i < L // 2 else "down" for i in range(L)])
            kw = dict(maxdim=_scaled_int(rng, 32, 512, scale))
            if neel:
                kw["work_ceiling_rule"] = "maxdim"
            out.append(dict(kind="xxz", arrival=t, L=L, delta=float(rng.uniform(-1, 1)),
                            spins=spins, tau=-0.05j, nsteps=_scaled_int(rng, 20, 200, scale),
                            seed=jseed, kw=kw))
        else:
            bits = _scaled_int(rng, 8, 11, scale)
            params = (float(rng.uniform(0.0, 0.05)), 0.0, float(rng.uniform(1, 3)),
                      float(rng.uniform(0.04, 0.12)), float(rng.uniform(0.2, 0.6)),
                      float(rng.uniform(-0.9, -0.3)))
            out.append(dict(kind="heston", arrival=t, bits=bits, params=params, tau=0.02,
                            nsteps=_scaled_int(rng, 10, 50, scale), seed=jseed,
                            kw=dict(maxdim=_scaled_int(rng, 32, 128, scale), hermitian=False)))
    return out


def job_inputs(spec):
    """``(state blocks, centre, MPO blocks)`` on the host for ``Server.submit``."""
    from . import models as DM
    from .server import host_blocks

    if spec["kind"] == "xxz":
        psi = DM.product_state(spec["spins"])
        mpo = DM.xxz_mpo(spec["L"], J=1.0, delta=spec["delta"])
        return host_blocks(psi.tensors), psi.center, host_blocks(mpo.tensors)
    from . import qtt as P

    b = spec["bits"]
    g = P.qtt_grid(b, b, x=(-1.0, 1.0), y=(0.0, 0.5), periodic_x=False, periodic_y=False)
    psi = P.qtt_mps(P.qtt_separable(g, lambda x: np.exp(0.5 * x), lambda v: np.exp(-v)))
    mpo = P.heston_mpo(g, P.HestonParams(*spec["params"]))
    return host_blocks(psi.tensors), psi.center, host_blocks(mpo.tensors)
