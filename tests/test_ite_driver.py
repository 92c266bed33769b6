"""The imaginary-time driver's host logic (``ite_step!`` / ``ite_evolve!``, ``ite_step.jl:62-301``)
on CPU: the product's driver (``bondupdategalerkin_b200/ite.py``) and the oracle's against one
scripted step, so the decisions are exercised without a device. The step is a stand-in whose
outside defect grows as dbeta^3 and whose closure, cap and ledger verdicts are scripted; both
drivers must take the same attempts, split the same way and fold the same record.
"""

import math

import numpy as np
import pytest

TOL = 1e-5


class _Ledger:
    def __init__(self, unmet=(), capped=False):
        self.unmet = list(unmet)
        self.maxdim_reached = capped
        self.workcap_reached = False
        self.expv_err, self.expv_iters, self.discarded, self.r_aug = 1e-12, 3, 1e-9, 4


class _Chain:
    """A chain of scalars standing in for site tensors (ite_step only copies and restores them)."""

    def __init__(self, n=4):
        self.sites = [1.0] * n
        self.center = 1

    def __len__(self):
        return len(self.sites)

    def __getitem__(self, i):
        return self.sites[i - 1]

    def __setitem__(self, i, v):
        self.sites[i - 1] = v

    def copy(self):
        c = _Chain(len(self))
        c.sites, c.center = list(self.sites), self.center
        return c

    def bond_dims(self):
        return [2] * (len(self) - 1)


def _script(closure_until=math.inf, cap_above=math.inf):
    """A step whose outside defect is (dbeta / 0.01)^3 tol: tol at dbeta = 0.01, 8 tol at 0.02;
    the closure is unmet for dbeta > closure_until unless closure_checks is set; the maxdim cap
    is reached for dbeta > cap_above."""
    calls = []

    def step(psi, mpo, tau, *, root_report, closure_checks=False, **kw):
        db = -complex(tau).real
        calls.append((round(db, 12), bool(closure_checks)))
        resid = (db / 0.01) ** 3 * TOL
        root_report.update(e_pre=-1.0, e_root=-1.0 - db, resid=resid, resid_initial=2 * resid,
                           outside=resid, outside_passes=1, outside_added=2)
        unmet = []
        if db > closure_until and not closure_checks:
            unmet.append("closure")
        capped = db > cap_above
        if capped:
            unmet.append("krylov")
        psi[1] = psi[1] + db  # a visible change, so restores are observable
        return {"ledger": _Ledger(unmet, capped)}

    return step, calls


def _energy(psi, mpo):
    return -float(psi[1])


def _normalise(psi):
    return 1.0


def _run(which, monkeypatch, step, dbeta, **kw):
    psi = _Chain()
    if which == "oracle":
        from oracle import ite as I

        rec = I.ite_step(psi, None, dbeta, step=step, energy=_energy, normalise=_normalise,
                         tol_basis=TOL, **kw)
    else:
        from bondupdategalerkin_b200 import ite as P
        from bondupdategalerkin_b200 import native as N

        monkeypatch.setattr(N, "cbe_bug_step", step)
        monkeypatch.setattr(P, "ite_energy", _energy)
        monkeypatch.setattr(P, "ite_normalise", _normalise)
        rec = P.ite_step(psi, None, dbeta, tol_basis=TOL, **kw)
    return rec, psi


def _summary(rec, psi):
    return (rec["status"], tuple(rec["unmet"]), round(rec["dbeta"], 12), rec["nsub"],
            len(rec["attempts"]), round(psi[1], 12))


@pytest.mark.parametrize("which", ["oracle", "product"])
def test_met_step_takes_one_attempt(which, monkeypatch):
    step, calls = _script()
    rec, psi = _run(which, monkeypatch, step, 0.01)
    assert rec["status"] == "met" and rec["nsub"] == 1 and calls == [(0.01, False)]


@pytest.mark.parametrize("which", ["oracle", "product"])
def test_outside_defect_splits_by_its_scaling(which, monkeypatch):
    """resid = 8 tol at dbeta 0.02 (order 2): ceil(1.2 * 8^(1/3)) = 3 sub-steps, each met, and the
    state restored before the split (the rejected attempt's change is undone)."""
    step, calls = _script()
    rec, psi = _run(which, monkeypatch, step, 0.02, order=2)
    assert rec["status"] == "retried" and rec["nsub"] == 3
    assert calls == [(0.02, False)] + [(round(0.02 / 3, 12), False)] * 3
    assert psi[1] == pytest.approx(1.0 + 0.02)  # three sub-steps of dbeta / 3 on the restored state


@pytest.mark.parametrize("which", ["oracle", "product"])
def test_unclosed_closure_is_reattempted_with_checks(which, monkeypatch):
    step, calls = _script(closure_until=0.0)
    rec, psi = _run(which, monkeypatch, step, 0.01, order=2)
    assert rec["status"] == "retried" and calls == [(0.01, False), (0.01, True)]
    assert psi[1] == pytest.approx(1.01)


@pytest.mark.parametrize("which", ["oracle", "product"])
def test_capped_failure_is_flagged_not_split(which, monkeypatch):
    step, calls = _script(cap_above=0.0)
    rec, _ = _run(which, monkeypatch, step, 0.01, order=1)
    assert rec["status"] == "failed" and len(calls) == 1 and "krylov" in rec["unmet"]
    step, _ = _script(cap_above=0.0)
    with pytest.raises(ArithmeticError):
        _run(which, monkeypatch, step, 0.01, order=1, on_fail="error")


@pytest.mark.parametrize("which", ["oracle", "product"])
def test_retries_run_out(which, monkeypatch):
    """A defect that no split within two retries can meet (tol scaled down 1e6): the step ends
    failed after nested splits, each capped at 64 sub-steps."""
    step, calls = _script()

    def harsh(psi, mpo, tau, *, root_report, **kw):
        out = step(psi, mpo, tau, root_report=root_report, **kw)
        root_report["resid"] *= 1e6
        return out

    rec, _ = _run(which, monkeypatch, harsh, 0.02, order=2, retries=1)
    assert rec["status"] == "failed" and "outside" in rec["unmet"]
    first = calls[0][0]
    count = min(max(math.ceil(1.2 * (8e6) ** (1 / 3)), 2), 64)
    assert first == 0.02 and len(calls) == 1 + count


def test_drivers_agree(monkeypatch):
    """Both drivers produce the same record on every scripted case."""
    cases = [dict(dbeta=0.01), dict(dbeta=0.02, order=2), dict(dbeta=0.05, order=3),
             dict(dbeta=0.01, order=2, closure_until=0.0)]
    for case in cases:
        case = dict(case)
        cu = case.pop("closure_until", math.inf)
        db = case.pop("dbeta")
        out = []
        for which in ("oracle", "product"):
            step, _ = _script(closure_until=cu)
            out.append(_summary(*_run(which, monkeypatch, step, db, **case)))
        assert out[0] == out[1], (case, out)


def test_evolve_records_beta(monkeypatch):
    from bondupdategalerkin_b200 import ite as P
    from oracle import ite as I

    steps = I.uniform_beta_steps(0.03, 3)
    logs = []
    for which in ("oracle", "product"):
        step, _ = _script()
        psi = _Chain()
        if which == "oracle":
            log = I.ite_evolve(psi, None, steps, observe=lambda p: p[1], step=step, energy=_energy,
                               normalise=_normalise, tol_basis=TOL)
        else:
            from bondupdategalerkin_b200 import native as N

            monkeypatch.setattr(N, "cbe_bug_step", step)
            monkeypatch.setattr(P, "ite_energy", _energy)
            monkeypatch.setattr(P, "ite_normalise", _normalise)
            log = P.ite_evolve(psi, None, steps, observe=lambda p: p[1], tol_basis=TOL)
        logs.append([(round(r["beta"], 12), r["status"], round(r["obs"], 12)) for r in log])
    assert logs[0] == logs[1]
    assert [b for b, _, _ in logs[0]] == [0.01, 0.02, 0.03]
    assert np.allclose([o for _, _, o in logs[0]], [1.01, 1.02, 1.03])
