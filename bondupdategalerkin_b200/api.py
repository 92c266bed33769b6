"""Public entry points of the B200 BUG engine.

* ``cbe_bug_step(psi, mpo, tau; ...)`` -- the drop-in for ``cbe_bug_step!``
  (``src/BUG/TimeEvolution/bug_step.jl:17-513``) on HBM-resident states, run as one call into the
  library (``native.py``); ``Batch`` steps many chains together (``bug_step_batch``);
* ``step_host(...)`` -- the same step for a caller whose state lives in host memory: the site
  tensors and the MPO are uploaded, the step runs on the device, and the new site tensors come back
  (the shape of a ``ccall`` from a Julia host that keeps its own containers);
* ``magnetisation(psi)`` -- ``<S^z_j>`` for every site (``src/QMB/Observables/bond_observables.jl:15``);
* ``tdvp2_step(psi, mpo, tau; ...)`` -- the two-site TDVP baseline (``src/Baselines/TDVP/tdvp2.jl``),
  ``tdvp2_step_host`` its host-buffer form;
* ``ite_step`` / ``ite_evolve`` and the step schedules -- normalised imaginary time
  (``src/BUG/ITE/ite_step.jl``, ``schedules.jl``);
* ``qtt_bug_step`` -- ``qtt_bug_step!`` for a linear flow (the rational-root BUG step,
  ``src/QTTS/Tooling/nonlinear_step.jl``);
* the quantics builders under the reference's names: ``qtt_grid``, ``qtt_separable``, ``qtt_mps``,
  ``qtt_shift``, ``qtt_derivative``, ``qtt_to_mpo``, ``HestonParams``, ``heston_op``,
  ``heston_mpo`` (``src/QTTS/Tooling``, ``src/QTTS/Models/Heston``).
"""

from __future__ import annotations

from .models import MPO, MPS, domain_wall_state, neel_state, product_state, sz_profile, xxz_mpo
from .ite import (beta_grid, geometric_schedule, ite_energy, ite_evolve, ite_step, log_panel_steps,
                  uniform_beta_steps, uniform_schedule)
from .native import Batch, cbe_bug_step, tdvp2_step
from .options import DDQRExpansion
from .qtt import (HestonParams, heston_mpo, heston_op, qtt_bug_step, qtt_derivative, qtt_grid, qtt_mps,
                  qtt_separable, qtt_shift, qtt_step_tolerance, qtt_to_mpo)
from .tensor import from_blocks, to_blocks

__all__ = ["cbe_bug_step", "Batch", "step_host", "step_host_flat", "magnetisation", "DDQRExpansion", "MPS", "MPO",
           "domain_wall_state", "neel_state", "product_state", "xxz_mpo", "tdvp2_step",
           "tdvp2_step_host", "ite_step", "ite_step_host", "ite_evolve", "ite_energy", "log_panel_steps",
           "uniform_beta_steps", "beta_grid", "uniform_schedule", "geometric_schedule",
           "qtt_grid", "qtt_separable", "qtt_mps", "qtt_shift", "qtt_derivative", "qtt_to_mpo",
           "HestonParams", "heston_op", "heston_mpo", "qtt_bug_step", "qtt_step_tolerance"]


def magnetisation(psi):
    return sz_profile(psi)


def step_host(host_state, center, host_mpo, tau, **kwargs):
    """One BUG step on host-resident data.

    ``host_state`` / ``host_mpo``: per site ``(legs, {key: ndarray})`` as ``tensor.to_blocks``
    returns. Returns ``(new_host_state, new_center, io)`` with ``io`` holding the bytes moved each
    way and the step info."""
    h2d = 0
    sites = []
    for legs, blocks in host_state:
        t = from_blocks(legs, blocks)
        h2d += 16 * t.nelem
        sites.append(t)
    ws = []
    for legs, blocks in host_mpo:
        t = from_blocks(legs, blocks)
        h2d += 16 * t.nelem
        ws.append(t)
    psi = MPS(sites, center)
    info = cbe_bug_step(psi, MPO(ws), tau, **kwargs)
    out = [to_blocks(t) for t in psi.tensors]
    d2h = sum(16 * t.nelem for t in psi.tensors)
    return out, psi.center, dict(h2d_bytes=h2d, d2h_bytes=d2h, info=info)


def step_host_flat(state, center, mpo, tau, **kwargs):
    """One BUG step on host-resident data in the engine's flat layout (``tensor.HostTensors``):
    the state and the MPO go up in one engine call each, the step runs on the device, and the new
    state comes back in one call with one synchronisation. Returns ``(new_state, new_center,
    io)`` with ``io`` holding the bytes moved each way and the step info."""
    from .tensor import from_host_many, to_host_many

    sites = from_host_many(state)
    ws = from_host_many(mpo)
    psi = MPS(sites, center)
    info = cbe_bug_step(psi, MPO(ws), tau, **kwargs)
    out = to_host_many(psi.tensors)
    return out, psi.center, dict(h2d_bytes=state.nbytes + mpo.nbytes, d2h_bytes=out.nbytes,
                                 info=info)


def tdvp2_step_host(host_state, center, host_mpo, tau, **kwargs):
    """One two-site TDVP step (``tdvp2_step!``) on host-resident data, as :func:`step_host` does
    for the BUG step: upload, step on the device, download. Returns ``(new_host_state,
    new_center, io)``."""
    from .native import tdvp2_step

    h2d = 0
    sites = []
    for legs, blocks in host_state:
        t = from_blocks(legs, blocks)
        h2d += 16 * t.nelem
        sites.append(t)
    ws = []
    for legs, blocks in host_mpo:
        t = from_blocks(legs, blocks)
        h2d += 16 * t.nelem
        ws.append(t)
    psi = MPS(sites, center)
    info = tdvp2_step(psi, MPO(ws), tau, **kwargs)
    out = [to_blocks(t) for t in psi.tensors]
    d2h = sum(16 * t.nelem for t in psi.tensors)
    return out, psi.center, dict(h2d_bytes=h2d, d2h_bytes=d2h, info=info)


def ite_step_host(host_state, center, host_mpo, dbeta, **kwargs):
    """One normalised imaginary-time step (``ite_step!``) on host-resident data: upload, step on
    the device, download. Returns ``(new_host_state, new_center, io)``."""
    h2d = 0
    sites = []
    for legs, blocks in host_state:
        t = from_blocks(legs, blocks)
        h2d += 16 * t.nelem
        sites.append(t)
    ws = []
    for legs, blocks in host_mpo:
        t = from_blocks(legs, blocks)
        h2d += 16 * t.nelem
        ws.append(t)
    psi = MPS(sites, center)
    rec = ite_step(psi, MPO(ws), dbeta, **kwargs)
    out = [to_blocks(t) for t in psi.tensors]
    d2h = sum(16 * t.nelem for t in psi.tensors)
    return out, psi.center, dict(h2d_bytes=h2d, d2h_bytes=d2h, info=rec)
