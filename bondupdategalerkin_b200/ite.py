"""Normalised imaginary-time CBE-BUG on HBM-resident states (``src/BUG/ITE/ite_step.jl``,
``src/BUG/ITE/schedules.jl``).

One step is ``cbe_bug_step`` at ``tau = -dbeta`` on the generators ``H - eshift`` (by default the
state's energy), with the root report and the outside-Galerkin defect charged to ``tol_basis``,
then renormalisation through the centre tensor. A rejected step is redone from the saved state as
sub-steps (their number from the defect's scaling, ``(resid / tol_basis)^(1/(p+1))``, else two)
while ``retries`` last; resource-capped failures are flagged at once. The step runs in the library
(``native.cbe_bug_step``); energies are ``<psi|H|psi> / <psi|psi>`` from a device environment
sweep. ``root_method`` is ``exp``, ``trapezoid``, ``radau2``, ``radau3`` or ``radau2_gmres``. Not
built: ``parallel`` half-sweeps.
"""

from __future__ import annotations

import math
import time

import numpy as np

from . import native as N
from . import tensor as T

ITE_MAXSPLIT = 64  # _ITE_MAXSPLIT (ite_step.jl:24)


def mpo_energy(psi, mpo) -> complex:
    """``<psi|H|psi>``: the left environment pushed through every site on the device."""
    ctx = psi.tensors[0].ctx
    env = N.env_boundary(ctx, "left")
    for a, w in zip(psi.tensors, mpo.tensors):
        env = N.env_step(env, a, w, "left")
    _, blocks = T.to_blocks(env)
    (v,) = blocks.values()
    return complex(v.reshape(-1)[0])


def ite_energy(psi, mpo) -> float:
    """``_ite_energy`` (``ite_step.jl:4-5``): ``<psi|H|psi> / <psi|psi>``."""
    n2 = T.norm(psi[psi.center]) ** 2
    return mpo_energy(psi, mpo).real / max(n2, np.finfo(float).eps)


def ite_normalise(psi) -> float:
    """``_ite_normalise!`` (``ite_step.jl:7-17``): renormalise through the centre; the old norm."""
    n = T.norm(psi[psi.center])
    if not (math.isfinite(n) and n > 0):
        raise ArithmeticError(f"imaginary-time step produced a state of norm {n} -- not representable")
    psi[psi.center] = T.scale(psi[psi.center], 1.0 / n)
    return n


def _nsplit(attempt, tol_basis, order) -> int:
    """``_ite_nsplit`` (``ite_step.jl:40-44``)."""
    r = attempt["resid"]
    if not ("outside" in attempt["unmet"] and math.isfinite(r) and r > tol_basis):
        return 2
    return min(max(math.ceil(1.2 * (r / tol_basis) ** (1.0 / (order + 1))), 2), ITE_MAXSPLIT)


def _capped(attempt) -> bool:
    """``_ite_capped`` (``ite_step.jl:53``)."""
    lg = attempt["info"]["ledger"]
    return bool(lg.maxdim_reached or lg.workcap_reached)


def _attempt(psi, mpo, dbeta, *, order, tol_basis, tol_trunc, tol_root, maxdim, eshift,
             outside_residual, rng, closure_checks=False, **kwargs):
    """``_ite_attempt!`` (``ite_step.jl:62-126``)."""
    t0 = time.perf_counter()
    e_before = ite_energy(psi, mpo)
    es = e_before if eshift == "energy" else float(eshift)
    rep = {}
    info = N.cbe_bug_step(psi, mpo, complex(-dbeta), order=order, eshift=es, tol_basis=tol_basis,
                          tol_trunc=tol_trunc, tol_expv=tol_root, maxdim=maxdim, root_report=rep,
                          outside_residual=outside_residual, closure_checks=closure_checks,
                          rng=rng, **kwargs)
    growth = ite_normalise(psi)
    e_after = ite_energy(psi, mpo)
    unmet = list(info["ledger"].unmet)
    if outside_residual and not (rep["resid"] <= tol_basis):
        unmet.append("outside")
    return dict(
        dbeta=dbeta, ok=not unmet, unmet=unmet, eshift=es, e_before=e_before,
        e_pre_root=rep["e_pre"], e_root=rep["e_root"], e_after=e_after,
        de_root=rep["e_root"] - rep["e_pre"], de_compression=e_after - rep["e_root"],
        outside=rep["outside"], resid=rep["resid"], resid_initial=rep["resid_initial"],
        outside_passes=rep["outside_passes"], outside_added=rep["outside_added"],
        root_err=info["ledger"].expv_err, root_iters=info["ledger"].expv_iters,
        discarded=info["ledger"].discarded, growth=growth, chi=max(psi.bond_dims(), default=0),
        r_aug=info["ledger"].r_aug,
        closure_checks=closure_checks, wall=time.perf_counter() - t0, info=info)


def _result(status, pieces, attempts, t0):
    """``_ite_result`` (``ite_step.jl:238-262``)."""
    unmet = []
    for piece in pieces:
        for u in piece["unmet"]:
            if u not in unmet:
                unmet.append(u)
    return dict(
        status=status, unmet=unmet, dbeta=sum(p["dbeta"] for p in pieces),
        e_before=pieces[0]["e_before"], e_pre_root=pieces[0]["e_pre_root"],
        e_root=pieces[-1]["e_root"], e_after=pieces[-1]["e_after"],
        de_root=sum(p["de_root"] for p in pieces),
        de_compression=sum(p["de_compression"] for p in pieces),
        resid=max(p["resid"] for p in pieces), outside=max(p["outside"] for p in pieces),
        root_err=max(p["root_err"] for p in pieces), discarded=max(p["discarded"] for p in pieces),
        chi=pieces[-1]["chi"], nsub=sum(p.get("nsub", 1) for p in pieces), attempts=attempts,
        wall=time.perf_counter() - t0)


def ite_step(psi, mpo, dbeta, *, order=2, root_method="exp", tol_basis=1e-5, tol_trunc=1e-6,
             tol_root=1e-6, maxdim=128, eshift="energy", outside_residual=True, retries=2,
             on_fail="flag", parallel=False, rng=None, **kwargs) -> dict:
    """``ite_step!(psi, mpo, dbeta; ...)`` (``ite_step.jl:129-231``): one normalised imaginary-time
    step in place. Returns ``status`` (met / retried / failed), ``unmet``, the energies, ``resid``,
    ``nsub`` and ``attempts``. ``kwargs`` go to ``cbe_bug_step``."""
    if not dbeta > 0:
        raise ValueError(f"dbeta must be positive, got {dbeta}")
    if root_method not in ("exp", "trapezoid", "radau2", "radau3", "radau2_gmres"):
        raise ValueError(f"root_method must be exp, trapezoid, radau2, radau3 or radau2_gmres, got {root_method!r}")
    if on_fail not in ("flag", "error"):
        raise ValueError("on_fail must be flag or error")
    if retries < 0:
        raise ValueError(f"retries must be >= 0, got {retries}")
    if parallel:
        raise NotImplementedError("parallel half-sweeps are not built")
    if rng is None:
        rng = np.random.default_rng(0x5EED)
    t0 = time.perf_counter()
    ite_normalise(psi)
    saved = psi.copy()  # the step replaces tensors and never mutates them: a stable snapshot
    akw = dict(order=order, tol_basis=tol_basis, tol_trunc=tol_trunc, tol_root=tol_root,
               maxdim=maxdim, eshift=eshift, outside_residual=outside_residual, rng=rng,
               root_method=root_method)

    def restore():
        for site in range(1, len(psi) + 1):
            psi[site] = saved[site]
        psi.center = saved.center

    attempts = []
    attempt = _attempt(psi, mpo, float(dbeta), **akw, closure_checks=False, **kwargs)
    attempts.append(attempt)
    # an unclosed closure is re-attempted with the measured, multi-pass closure
    if not attempt["ok"] and order > 1 and "closure" in attempt["unmet"]:
        restore()
        attempt = _attempt(psi, mpo, float(dbeta), **akw, closure_checks=True, **kwargs)
        attempts.append(attempt)
    if attempt["ok"]:
        return _result("met" if len(attempts) == 1 else "retried", [attempt], attempts, t0)
    if retries > 0 and not _capped(attempt):
        restore()
        count = _nsplit(attempt, tol_basis, order)
        halves = []
        for _ in range(count):
            sub = ite_step(psi, mpo, dbeta / count, retries=retries - 1,
                           on_fail="flag", **akw, **kwargs)
            attempts += sub["attempts"]
            halves.append(sub)
        ok = all(h["status"] != "failed" for h in halves)
        res = _result("retried" if ok else "failed", halves, attempts, t0)
        if not ok and on_fail == "error":
            raise ArithmeticError(f"imaginary-time step dbeta={dbeta} failed after retries: "
                                  f"unmet {res['unmet']}")
        return res
    if on_fail == "error":
        raise ArithmeticError(f"imaginary-time step dbeta={dbeta} failed: unmet {attempt['unmet']}")
    return _result("failed", [attempt], attempts, t0)


def ite_evolve(psi, mpo, steps, observe=None, **kwargs) -> list:
    """``ite_evolve!`` (``ite_step.jl:273-301``): one ``ite_step`` per entry of ``steps``; one record
    per step with the ``beta`` reached, and ``obs = observe(psi)`` when given. A failed step is
    recorded and the evolution continues (``on_fail = "error"`` stops it)."""
    log = []
    beta = 0.0
    for db in steps:
        rec = ite_step(psi, mpo, db, **kwargs)
        beta += db
        rec = dict(beta=beta, **rec)
        if observe is not None:
            rec["obs"] = observe(psi)
        log.append(rec)
    return log


# ── step-size schedules (schedules.jl) ──────────────────────────────────────────────────────


def log_panel_steps(beta_max, panel_count, per_panel=4):
    """``log_panel_steps``: ``panel_count`` dyadic panels ``0, beta_max / 2^(P-1), ..., beta_max``,
    each split into ``per_panel`` uniform steps."""
    if not beta_max > 0:
        raise ValueError(f"beta_max must be positive, got {beta_max}")
    if panel_count < 1:
        raise ValueError(f"log_panel_steps needs panel_count >= 1, got {panel_count}")
    if per_panel < 1:
        raise ValueError(f"per_panel must be >= 1, got {per_panel}")
    edges = [0.0] + [float(beta_max) / 2.0 ** (panel_count - p) for p in range(1, panel_count + 1)]
    out = []
    for p in range(panel_count):
        out += [(edges[p + 1] - edges[p]) / per_panel] * per_panel
    return out


def uniform_beta_steps(beta_max, step_count):
    """``step_count`` equal steps reaching ``beta_max``."""
    if not beta_max > 0:
        raise ValueError(f"beta_max must be positive, got {beta_max}")
    if step_count < 1:
        raise ValueError(f"step_count must be >= 1, got {step_count}")
    return [float(beta_max) / step_count] * step_count


def beta_grid(steps):
    """The grid points ``0, b_1, ..., beta_max`` a step list reaches."""
    return [0.0] + list(np.cumsum(np.asarray(steps, dtype=float)))


def uniform_schedule(step_size, step_count):
    return [float(step_size)] * step_count


def geometric_schedule(first_step, ratio, hmax, step_count):
    """``dtau_k = min(hmax, first_step * ratio^k)``, ``k = 0..step_count-1``."""
    return [min(float(hmax), first_step * ratio ** k) for k in range(step_count)]
