#!/usr/bin/env python
"""Benchmark of the rank-adaptive BUG step (``cbe_bug_step``) on B200.

Metric: BUG steps/s. Workload (the L = 64 U(1) XXZ quench): J = 1, delta = 0.5, domain-wall
start, tau = -0.05i, order 2, tol_basis 1e-4, maxdim 256, bond_ceiling_factor 1.2, DD-QR
:rank_tail with an 8-column sketch, Gaussians from a generator seeded 1234. A "step" is one
``cbe_bug_step`` of the chain. ``--warmup W`` steps from the product state are untimed, then the
next ``--steps K`` steps of the same trajectory are timed, each between CUDA events on the engine
stream with a 256 MiB write (2x L2) flushing the cache before it.

Printed JSON line: ``value`` (steps/s, HBM-resident state), ``e2e`` (the same K steps replayed
through host buffers: the state and MPO uploaded and the new state downloaded every step),
``roofline`` (the dominant kernel family from a profiled replay of the same K steps),
``cpu_baseline`` (the CPU oracle over a bounded sample of the same steps), ``clocks``.
``--impl reference`` times the CPU oracle (the restatement of the reference's CPU path) on the
same steps. Under torchrun each rank runs an independent replica (the step does not shard).

``--workload tdvp2`` measures the reference's matched-accuracy comparator, two-site TDVP
(``tdvp2_step!``, maxdim 256, per-cut allowance ``weight_tol`` 1e-7, Lanczos with 30 iterations),
over the same chain and 100-step trajectory (metric TDVP2 steps/s). ``--workload ite`` measures
normalised imaginary time (``ite_step!`` with its energy shift, outside residual and retries) on the
L = 32 Heisenberg chain from Neel, dbeta 0.125 to beta 4 (metric ITE steps/s).
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = dict(L=64, J=1.0, delta=0.5, tau=-0.05j, order=2, tol_basis=1e-4, maxdim=256,
                bond_ceiling_factor=1.2, seed=1234)
WORKLOAD_NAME = "xxz_quench_L64_delta0.5_domainwall_maxdim256_order2_tol1e-4"
# The Heston PDE on a quantics grid: 10 + 10 bits (x in [-1, 1], v in [0, 0.5], end points on the
# grid), r 0.03, q 0.01, kappa 2, theta 0.09, sigma 0.4, rho -0.7, start exp(0.5 x) exp(-v),
# tau = 0.02 (real), Arnoldi (non-Hermitian), maxdim 64, order 1, 50 steps.
HESTON = dict(nbits=10, params=(0.03, 0.01, 2.0, 0.09, 0.4, -0.7), tau=0.02, maxdim=64, seed=1234)
HESTON_NAME = "heston_qtt_10x10bits_maxdim64_tau0.02_arnoldi"
# The reference's matched-accuracy comparator on the headline chain: two-site TDVP with the BUG's
# per-cut allowance (weight_tol = the step's default tol_trunc 1e-7), maxdim 256, Lanczos.
TDVP2 = dict(maxdim=256, weight_tol=1e-7)
TDVP2_NAME = "tdvp2_xxz_quench_L64_delta0.5_domainwall_maxdim256_wtol1e-7"
# Normalised imaginary time (ite_step!) on the Heisenberg chain from Neel, the setting of the
# reference's heisenberg_ite fixture at L = 32: dbeta 0.125, order 2, maxdim 128, the ite_step!
# defaults (tol_basis 1e-5, tol_trunc 1e-6, tol_root 1e-6, energy shift, outside residual).
ITE = dict(L=32, delta=1.0, dbeta=0.125, kw=dict(order=2, maxdim=128))
ITE_NAME = "ite_heisenberg_L32_neel_dbeta0.125_order2_maxdim128"
KIND = ["xxz"]
PARALLEL = [False]  # parallel = true: half-sweeps and frontier halves on two streams
L2_FLUSH_BYTES = 256 << 20
_HESTON_DOMAIN = dict(x=(-1.0, 1.0), y=(0.0, 0.5), periodic_x=False, periodic_y=False)


def tau():
    return HESTON["tau"] if KIND[0] == "heston" else WORKLOAD["tau"]


def seed():
    return HESTON["seed"] if KIND[0] == "heston" else WORKLOAD["seed"]


def dev_step(mod, psi, mpo, rng):
    """One step of the workload through the product module ``mod`` (the native step)."""
    if KIND[0] == "tdvp2":
        from bondupdategalerkin_b200 import native as N

        return N.tdvp2_step(psi, mpo, tau(), **TDVP2)
    if KIND[0] == "ite":
        from bondupdategalerkin_b200 import ite as DI

        return DI.ite_step(psi, mpo, ITE["dbeta"], rng=rng, **ITE["kw"])
    return mod.cbe_bug_step(psi, mpo, tau(), rng=rng, **step_kwargs())


def oracle_step(psi, mpo, rng):
    """The same step in the CPU oracle."""
    if KIND[0] == "tdvp2":
        from oracle import tdvp as OT

        return OT.tdvp2_step(psi, mpo, tau(), **TDVP2)
    if KIND[0] == "ite":
        from oracle import ite as OI

        return OI.ite_step(psi, mpo, ITE["dbeta"], rng=rng, **ITE["kw"])
    from oracle import step as OS

    return OS.cbe_bug_step(psi, mpo, tau(), rng=rng, **step_kwargs())


def metric_name():
    return {"tdvp2": "tdvp2_steps_per_s", "ite": "ite_steps_per_s"}.get(KIND[0], "bug_steps_per_s")


def step_kwargs():
    extra = dict(parallel=True) if PARALLEL[0] else {}
    if KIND[0] == "heston":
        return dict(maxdim=HESTON["maxdim"], hermitian=False, **extra)
    w = WORKLOAD
    return dict(order=w["order"], tol_basis=w["tol_basis"], maxdim=w["maxdim"],
                bond_ceiling_factor=w["bond_ceiling_factor"], **extra)


def device_inputs():
    """(state, MPO) of the workload, built by the product's host builders and uploaded."""
    if KIND[0] == "heston":
        from bondupdategalerkin_b200 import qtt as P

        g = P.qtt_grid(HESTON["nbits"], HESTON["nbits"], **_HESTON_DOMAIN)
        psi = P.qtt_mps(P.qtt_separable(g, lambda x: np.exp(0.5 * x), lambda v: np.exp(-v)))
        return psi, P.heston_mpo(g, P.HestonParams(*HESTON["params"]))
    from bondupdategalerkin_b200 import models as DM

    if KIND[0] == "ite":
        return DM.neel_state(ITE["L"]), DM.xxz_mpo(ITE["L"], J=1.0, delta=ITE["delta"])
    w = WORKLOAD
    return DM.domain_wall_state(w["L"]), DM.xxz_mpo(w["L"], J=w["J"], delta=w["delta"])


def oracle_inputs():
    """(state, MPO) of the workload in the CPU oracle."""
    if KIND[0] == "heston":
        from oracle import qtt as Q

        g = Q.qtt_grid(HESTON["nbits"], HESTON["nbits"], **_HESTON_DOMAIN)
        psi = Q.qtt_mps(Q.qtt_separable(g, lambda x: np.exp(0.5 * x), lambda v: np.exp(-v)))
        return psi, Q.heston_mpo(g, Q.HestonParams(*HESTON["params"]))
    from oracle import models as OM

    if KIND[0] == "ite":
        return OM.neel_state(ITE["L"]), OM.xxz_mpo(ITE["L"], J=1.0, delta=ITE["delta"])
    w = WORKLOAD
    return OM.domain_wall_state(w["L"]), OM.xxz_mpo(w["L"], J=w["J"], delta=w["delta"])


def config_dict(args, ws, max_bond=None):
    cfg = _config_dict(args, ws, max_bond)
    if getattr(args, "mixed", 0) > 0:
        cfg["precision"] = f"3xTF32 tensor cores for contraction blocks >= {args.mixed} x {args.mixed}"
    if PARALLEL[0]:
        cfg["half_sweeps"] = "parallel = true: the two halves on two streams and two host threads"
    return cfg


def _config_dict(args, ws, max_bond=None):
    if KIND[0] == "heston":
        h = HESTON
        cfg = {"workload": HESTON_NAME, "L": 2 * h["nbits"], "grid": "1024 x 1024", "tau": "0.02",
               "order": 1, "maxdim": h["maxdim"], "hermitian": False,
               "timed_steps": f"{args.warmup + 1}..{args.warmup + args.steps}",
               "l2": "flushed before every step (256 MiB write)",
               "parallelism": f"replicas x{ws}" if ws > 1 else "single GPU"}
        if max_bond is not None:
            cfg["max_bond_dim_after"] = max_bond
        return cfg
    w = WORKLOAD
    if KIND[0] == "ite":
        cfg = {"workload": ITE_NAME, "L": ITE["L"], "delta": ITE["delta"], "dbeta": ITE["dbeta"],
               "order": 2, "maxdim": 128, "tol_basis": 1e-5, "eshift": "energy",
               "outside_residual": True,
               "timed_steps": f"{args.warmup + 1}..{args.warmup + args.steps}",
               "l2": "flushed before every step (256 MiB write)",
               "parallelism": f"replicas x{ws}" if ws > 1 else "single GPU"}
        if max_bond is not None:
            cfg["max_bond_dim_after"] = max_bond
        return cfg
    if KIND[0] == "tdvp2":
        cfg = {"workload": TDVP2_NAME, "L": w["L"], "delta": w["delta"], "tau": "-0.05i",
               "maxdim": TDVP2["maxdim"], "weight_tol": TDVP2["weight_tol"], "krylov": "lanczos, maxiter 30",
               "timed_steps": f"{args.warmup + 1}..{args.warmup + args.steps}",
               "l2": "flushed before every step (256 MiB write)",
               "parallelism": f"replicas x{ws}" if ws > 1 else "single GPU"}
        if max_bond is not None:
            cfg["max_bond_dim_after"] = max_bond
        return cfg
    cfg = {"workload": WORKLOAD_NAME, "L": w["L"], "delta": w["delta"], "tau": "-0.05i",
           "order": w["order"], "tol_basis": w["tol_basis"], "maxdim": w["maxdim"],
           "timed_steps": f"{args.warmup + 1}..{args.warmup + args.steps}",
           "l2": "flushed before every step (256 MiB write)",
           "parallelism": f"replicas x{ws}" if ws > 1 else "single GPU"}
    if max_bond is not None:
        cfg["max_bond_dim_after"] = max_bond
    return cfg


def dist_env():
    from bondupdategalerkin_b200.replicas import world

    return world()


class ClockSampler:
    """``nvidia-smi`` clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows)}


def measure_zgemm_tflops(torch, device):
    """cuBLAS ZGEMM (torch.matmul, complex128, n = 4096) as the FP64 compute reference, burst."""
    n = 4096
    a = torch.randn(n, n, dtype=torch.complex128, device=device)
    b = torch.randn(n, n, dtype=torch.complex128, device=device)
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize(device)
    best = 1e30
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize(device)
        best = min(best, e0.elapsed_time(e1) / 1e3)
    return 8.0 * n ** 3 / best / 1e12


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def measured_traffic():
    """DRAM bytes per launch of each kernel family from a committed ncu capture
    (profiles/dram_traffic.json: family -> {dram_bytes_per_launch, source}), or {}."""
    p = os.path.join(ROOT, "profiles", "dram_traffic.json")
    if os.path.exists(p):
        return json.load(open(p))
    return {}


def blas_threads():
    try:
        from threadpoolctl import threadpool_info

        return max([i.get("num_threads", 1) for i in threadpool_info()] or [1])
    except Exception:
        return os.cpu_count() or 1


def oracle_steps(warmup, k):
    """Run the CPU oracle over the same trajectory: ``warmup`` untimed steps, then ``k`` timed.
    Returns (seconds for the k steps, bond dims after)."""
    psi, mpo = oracle_inputs()
    rng = np.random.default_rng(seed())
    for _ in range(warmup):
        oracle_step(psi, mpo, rng)
    t0 = time.perf_counter()
    for _ in range(k):
        oracle_step(psi, mpo, rng)
    return time.perf_counter() - t0, psi.bond_dims()


def oracle_sampled_steps(snaps, mpo_host=None):
    """Time one CPU-oracle step from each saved device state (downloaded first, untimed), with
    the generator state the device step started from. Returns (seconds, step numbers)."""
    from oracle import blocks as OB
    from oracle import models as OM
    from bondupdategalerkin_b200 import tensor as DT

    mpo = mpo_host or oracle_inputs()[1]
    secs, which = 0.0, []
    for step_no, psi_d, rng_state in snaps:
        tensors = []
        for t in psi_d.tensors:
            legs, blocks = DT.to_blocks(t)
            tensors.append(OB.BT([OB.Leg(l.dir, l.sectors) for l in legs], blocks))
        psi = OM.MPS(tensors, psi_d.center)
        rng = np.random.default_rng()
        rng.bit_generator.state = rng_state
        t0 = time.perf_counter()
        oracle_step(psi, mpo, rng)
        secs += time.perf_counter() - t0
        which.append(step_no)
    return secs, which


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    k = args.steps
    secs, bd = oracle_steps(args.warmup, k)
    value = k / secs
    cores = blas_threads()
    line = {
        "impl": "reference", "metric": metric_name(), "value": value, "unit": "steps/s",
        "n_gpus": ws, "steps": k, "warmup": args.warmup, "ms_per_step": 1e3 * secs / k,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
        "data": "synthetic (deterministic product-state start, seeded Gaussian probes)",
        "config": config_dict(args, ws, max(bd)),
        "cpu_baseline": {"value": value, "unit": "steps/s", "cores": cores, "kind": "port",
                         "sample": f"steps {args.warmup + 1}..{args.warmup + k} of the quench, "
                                   f"max bond dim after {max(bd)}"},
        "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def mps_bytes(psi):
    return sum(16 * t.nelem for t in psi.tensors)


def run_engine(args):
    import torch

    from bondupdategalerkin_b200.replicas import Replicas

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    reps = Replicas("nccl", device=dev)  # N independent replicas: timing collectives only
    from bondupdategalerkin_b200 import _engine as E
    from bondupdategalerkin_b200 import build as Bld

    if Bld.needs_build():
        Bld.build()
    E.set_default_device(local)
    from bondupdategalerkin_b200 import tensor as DT

    from bondupdategalerkin_b200 import native as DS

    ctx = E.context(local)
    ctx.set_mixed(args.mixed)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    psi, mpo = device_inputs()
    rng = np.random.default_rng(seed())
    for _ in range(args.warmup):
        dev_step(DS, psi, mpo, rng)
    start_psi = psi.copy()
    start_rng = rng.bit_generator.state

    # ── timed region ──
    ctx.synchronize()
    torch.cuda.synchronize(dev)
    reps.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    launches0 = ctx.launches()
    ctx.reset_stats()
    # states (and generator states) before a few evenly spread steps, for the CPU baseline sample;
    # keeping them costs nothing in the timed region (the step replaces tensors, never mutates them)
    sample_at = sorted({int(round(i * (args.steps - 1) / max(args.cpu_steps - 1, 1)))
                        for i in range(min(args.cpu_steps, args.steps))})
    snaps = []
    evs = []
    for i in range(args.steps):
        if i in sample_at:
            snaps.append((args.warmup + i + 1, psi.copy(), rng.bit_generator.state))
        with torch.cuda.stream(stream):
            flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        dev_step(DS, psi, mpo, rng)
        e1.record(stream)
        evs.append((e0, e1))
    ctx.synchronize()
    torch.cuda.synchronize(dev)
    launches = ctx.launches() - launches0
    hstats = ctx.host_stats()
    host_line = {"syncs_per_step": hstats["syncs"] / args.steps,
                 "sync_wait_ms_per_step": 1e3 * hstats["wait_s"] / args.steps,
                 "launch_call_ms_per_step": 1e3 * hstats["launch_s"] / args.steps,
                 "alloc_call_ms_per_step": 1e3 * hstats["alloc_s"] / args.steps}
    reps.barrier()
    clk = clocks.stop()
    step_ms = [a.elapsed_time(b) for a, b in evs]
    value, total_ms = reps.rate(args.steps, float(sum(step_ms)))  # max over ranks
    final_dims = psi.bond_dims()
    if args.no_replay:
        if rank == 0:
            print(json.dumps({"metric": metric_name(), "value": value, "unit": "steps/s",
                              "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
                              "ms_per_step": total_ms / args.steps, "gpu_launches": int(launches),
                              "host_waits": host_line,
                              "note": "--no-replay: timing run only (no e2e, roofline or baseline)"}),
                  flush=True)
        reps.close()
        return

    # ── profiled replay of the same steps (kernel durations on the engine stream) ──
    psi_r = start_psi.copy()
    rng_r = np.random.default_rng()
    rng_r.bit_generator.state = start_rng
    ctx.reset_stats()
    ctx.set_profiling(True)
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        dev_step(DS, psi_r, mpo, rng_r)
    ctx.synchronize()
    stats = ctx.kernel_stats()
    ctx.set_profiling(False)
    assert psi_r.bond_dims() == final_dims, "profiled replay diverged from the timed steps"

    # ── end to end through host buffers: upload state+MPO, step, download the new state ──
    from bondupdategalerkin_b200.api import ite_step_host, step_host_flat, tdvp2_step_host

    host_state = [DT.to_blocks(t) for t in start_psi.tensors]
    host_mpo = [DT.to_blocks(t) for t in mpo.tensors]
    if KIND[0] in ("xxz", "heston"):  # the flat host layout: one engine call each way
        host_state, host_mpo = DT.host_from_blocks(host_state), DT.host_from_blocks(host_mpo)
    rng_e = np.random.default_rng()
    rng_e.bit_generator.state = start_rng
    center = start_psi.center
    e2e_ms, h2d, d2h = 0.0, 0, 0
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        if KIND[0] == "tdvp2":
            host_state, center, io = tdvp2_step_host(host_state, center, host_mpo, tau(), **TDVP2)
        elif KIND[0] == "ite":
            host_state, center, io = ite_step_host(host_state, center, host_mpo, ITE["dbeta"],
                                                   rng=rng_e, **ITE["kw"])
        else:
            host_state, center, io = step_host_flat(host_state, center, host_mpo, tau(), rng=rng_e,
                                                    **step_kwargs())
        e1.record(stream)
        ctx.synchronize()
        e2e_ms += e0.elapsed_time(e1)
        h2d += io["h2d_bytes"]
        d2h += io["d2h_bytes"]
    e2e_value, e2e_ms = reps.rate(args.steps, e2e_ms)  # max over ranks

    # ── roofline of the dominant kernel family ──
    hbm_peak, hbm_src = measured_peaks()
    fam = max(stats, key=lambda f: stats[f]["ms"])
    st = stats[fam]
    per_launch_ms = st["ms"] / max(st["launches"], 1)
    zgemm = None
    if fam == "gemm":
        zgemm = measure_zgemm_tflops(torch, dev)
        achieved = st["flops"] / max(st["launches"], 1) / (per_launch_ms / 1e3) / 1e12
        roof = {"bound": "tensor", "achieved": achieved, "peak": zgemm, "unit": "TFLOP/s",
                "frac": achieved / zgemm, "traffic": None,
                "peak_source": "cuBLAS ZGEMM (torch.matmul complex128 4096^3) measured in this run"}
    else:
        achieved = st["bytes"] / max(st["launches"], 1) / (per_launch_ms / 1e3) / 1e9
        roof = {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                "frac": achieved / hbm_peak, "traffic": None,
                "peak_source": f"MEASURED_PEAKS.json hbm_gbs ({hbm_src})"}
    traffic = measured_traffic().get(fam)
    if traffic:
        roof["traffic"] = traffic["dram_bytes_per_launch"]
        roof["traffic_source"] = traffic["source"]
    tot_ms = sum(s["ms"] for s in stats.values())
    roof["kernel"] = E.KERNEL_NAMES[fam]
    roof["launches"] = st["launches"]
    roof["avg_launch_us"] = 1e3 * per_launch_ms
    roof["share_of_device_time"] = st["ms"] / tot_ms if tot_ms > 0 else None
    roof["families"] = {f: {"launches": s["launches"], "ms": round(s["ms"], 3)} for f, s in stats.items()}

    # the bandwidth-bound families (copies, inner products, combinations, leg scaling): the one
    # with the most device time, its algorithmic bytes per launch over its average launch time
    bw = {f: x for f, x in stats.items() if f in ("copy", "dot", "lincomb", "scale") and x["launches"]}
    if bw:
        bf = max(bw, key=lambda f: bw[f]["ms"])
        b_ms = bw[bf]["ms"] / bw[bf]["launches"]
        b_ach = bw[bf]["bytes"] / bw[bf]["launches"] / (b_ms / 1e3) / 1e9
        roof["hbm_family"] = {"family": bf, "bound": "hbm", "achieved": b_ach, "peak": hbm_peak,
                              "unit": "GB/s", "frac": b_ach / hbm_peak, "avg_launch_us": 1e3 * b_ms,
                              "peak_source": f"MEASURED_PEAKS.json hbm_gbs ({hbm_src})"}

    line = {
        "metric": metric_name(), "value": value, "unit": "steps/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
        "data": "synthetic (deterministic product-state start, seeded Gaussian probes)",
        "config": config_dict(args, ws, max(final_dims)),
        "gpu_launches": int(launches),
        "e2e": {"value": e2e_value, "unit": "steps/s", "h2d_bytes_per_step": h2d // args.steps,
                "d2h_bytes_per_step": d2h // args.steps},
        "roofline": roof,
        "clocks": clk,
        "host_waits": host_line,
    }
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        secs, which = oracle_sampled_steps(snaps, mpo_host=None)
        line["cpu_baseline"] = {"value": len(which) / secs, "unit": "steps/s",
                                "cores": blas_threads(), "kind": "port",
                                "sample": "CPU oracle, one step from each of the device "
                                          f"trajectory's states before steps {which} (of "
                                          f"{args.warmup + 1}..{args.warmup + args.steps})"}
    if zgemm is not None:
        line["fp64_zgemm_tflops_measured"] = zgemm
    if rank == 0:
        print(json.dumps(line), flush=True)
    reps.close()


# ── batched and served workloads (the native job server) ─────────────────────────────────────

def _stream_oracle_inputs(spec):
    """A job spec's inputs in the CPU oracle (the baseline leg)."""
    if spec["kind"] == "xxz":
        from oracle import models as OM

        return OM.product_state(spec["spins"]), OM.xxz_mpo(spec["L"], J=1.0, delta=spec["delta"])
    from oracle import qtt as Q

    b = spec["bits"]
    g = Q.qtt_grid(b, b, **_HESTON_DOMAIN)
    psi = Q.qtt_mps(Q.qtt_separable(g, lambda x: np.exp(0.5 * x), lambda v: np.exp(-v)))
    return psi, Q.heston_mpo(g, Q.HestonParams(*spec["params"]))


def _oracle_from_blocks(blocks, center):
    from oracle import blocks as OB
    from oracle import models as OM

    return OM.MPS([OB.BT([OB.Leg(l.dir, l.sectors) for l in legs], b) for legs, b in blocks], center)


def stream_cpu_sample(specs, jobs, k=4):
    """The oracle on a bounded sample: for k jobs, one step from the job's start and one from its
    final state (so the sample spans the jobs' range of bond dimensions). Returns (steps, s)."""
    from oracle import step as OS

    secs, n = 0.0, 0
    idx = np.linspace(0, len(specs) - 1, min(k, len(specs))).round().astype(int)
    for i in idx:
        spec, job = specs[i], jobs[i]
        psi, mpo = _stream_oracle_inputs(spec)
        starts = [psi]
        if job is not None and job.result is not None:
            starts.append(_oracle_from_blocks(job.result, job.result_center))
        for st in starts:
            rng = np.random.default_rng(spec["seed"])
            t0 = time.perf_counter()
            OS.cbe_bug_step(st, mpo, spec["tau"], rng=rng, **spec["kw"])
            secs += time.perf_counter() - t0
            n += 1
    return n, secs


def _cpu_stream_task(task):
    """One oracle step of a job-stream sample, in a worker process (single-threaded BLAS)."""
    from oracle import step as OS

    st, mpo, tau, seed, kw = task
    rng = np.random.default_rng(seed)
    t0 = time.perf_counter()
    OS.cbe_bug_step(st, mpo, tau, rng=rng, **kw)
    return time.perf_counter() - t0


def stream_cpu_sample_concurrent(specs, jobs, workers, k=16):
    """The oracle's aggregate rate on the same sample as :func:`stream_cpu_sample` (one step from
    the start and one from the final state of k jobs), with `workers` processes running those
    steps at once, each on one BLAS thread: the CPU counterpart of the GPU arm's worker threads.
    Returns (steps, wall seconds)."""
    import multiprocessing as mp

    idx = np.linspace(0, len(specs) - 1, min(k, len(specs))).round().astype(int)
    tasks = []
    for i in idx:
        spec, job = specs[i], jobs[i]
        psi, mpo = _stream_oracle_inputs(spec)
        starts = [psi]
        if job is not None and job.result is not None:
            starts.append(_oracle_from_blocks(job.result, job.result_center))
        tasks += [(st, mpo, spec["tau"], spec["seed"], spec["kw"]) for st in starts]
    keys = ("OPENBLAS_NUM_THREADS", "OMP_NUM_THREADS", "MKL_NUM_THREADS")
    saved = {key: os.environ.get(key) for key in keys}
    for key in keys:
        os.environ[key] = "1"
    try:
        with mp.get_context("spawn").Pool(workers) as pool:
            pool.map(_cpu_stream_task, tasks[:1])  # workers up and imports done, untimed
            t0 = time.perf_counter()
            pool.map(_cpu_stream_task, tasks, chunksize=1)
            wall = time.perf_counter() - t0
    finally:
        for key, v in saved.items():
            if v is None:
                os.environ.pop(key, None)
            else:
                os.environ[key] = v
    return len(tasks), wall


def _block_bytes(blocks):
    return sum(16 * v.size for _, b in blocks for v in b.values())


def run_stream(args):
    """``--workload batch`` (64 chains submitted at once) or ``served`` (Poisson arrivals)."""
    import torch

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    from bondupdategalerkin_b200 import _engine as E
    from bondupdategalerkin_b200 import build as Bld
    from bondupdategalerkin_b200 import server as S
    from bondupdategalerkin_b200 import workloads as WL

    if Bld.needs_build():
        Bld.build()
    E.set_default_device(local)
    workers = args.workers or min(16, os.cpu_count() or 1)
    free, total = torch.cuda.mem_get_info(local)
    budget = int(0.8 * free)
    if KIND[0] == "batch":
        specs = WL.batch_specs(args.jobs or 64)
        name = f"batch_{len(specs)}_xxz_chains_L32-96_maxdim64-256_50steps_order2"
    else:
        specs = WL.served_specs(args.jobs or 48, rate=20.0, scale=args.scale)
        name = (f"served_poisson20_{len(specs)}jobs_70xxz_30heston_scale{args.scale:g}")
    inputs = [WL.job_inputs(sp) for sp in specs]  # host blocks, untimed
    h2d = sum(_block_bytes(a) + _block_bytes(c) for a, _, c in inputs)
    clocks = ClockSampler(local)
    clocks.start()
    with S.Server(workers=workers, budget_bytes=budget, device=local) as srv:
        t0 = time.perf_counter()
        jobs = []
        for sp, (st, cen, mp) in zip(specs, inputs):
            if KIND[0] == "served":
                delay = t0 + sp["arrival"] - time.perf_counter()
                if delay > 0:
                    time.sleep(delay)
            jobs.append(srv.submit(st, cen, mp, sp["tau"], sp["nsteps"], sp["seed"], **sp["kw"]))
        srv.wait()
        wall = time.perf_counter() - t0
        launches = srv.launches()
        stats = [j.stats for j in jobs]
        lat = S.latency_summary(jobs)
    clk = clocks.stop()
    failed = [s for s in stats if s["state"] != "done"]
    steps = sum(s["steps_done"] for s in stats)
    d2h = sum(_block_bytes(j.result) for j in jobs if j.result)
    value = steps / wall
    line = {
        "metric": "chain_steps_per_s" if KIND[0] == "batch" else "served_steps_per_s",
        "value": value, "unit": "steps/s", "n_gpus": 1, "steps": steps, "warmup": 0,
        "ms_per_step": 1e3 * wall / max(steps, 1), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "c128",
        "data": "synthetic (seeded job stream: product/QTT starts, seeded Gaussian probes)",
        "config": {"workload": name, "jobs": len(specs), "workers": workers,
                   "hbm_budget_bytes": budget, "wall_s": wall,
                   "timing": "host wall clock from the first submit to the last job's end, every "
                             "worker stream drained (inputs uploaded and results downloaded by the "
                             "jobs inside the timed region)"},
        "gpu_launches": int(launches),
        "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": h2d // max(steps, 1),
                "d2h_bytes_per_step": d2h // max(steps, 1)},
        "latency": lat, "jobs_failed": len(failed),
        "failures": [(s["steps_done"], s["status"], s["error"]) for s in failed[:3]], "clocks": clk,
    }
    if KIND[0] == "served":
        line["config"]["arrivals"] = "Poisson, 20 jobs/s"
        line["config"]["scale"] = (f"{args.scale:g}: L, maxdim, bits and steps ranges shrunk toward "
                                   "their lower ends by this factor (1 = the stream as specified)")
        line["throughput_jobs_per_s"] = len(specs) / wall
    if not args.no_cpu_baseline:
        n, secs = stream_cpu_sample_concurrent(specs, jobs, workers)
        n1, secs1 = stream_cpu_sample(specs, jobs)
        line["cpu_baseline"] = {"value": n / secs, "unit": "steps/s", "cores": workers,
                                "kind": "port",
                                "sample": f"CPU oracle, one step from the start and one from the end "
                                          f"state of {n // 2} jobs spread over the stream, {workers} "
                                          f"processes at once on one BLAS thread each (as many "
                                          f"as the GPU arm's workers)",
                                "one_at_a_time": {"value": n1 / secs1, "cores": blas_threads(),
                                                  "sample": f"{n1 // 2} of those jobs, one step "
                                                            f"at a time on all BLAS threads"}}
    print(json.dumps(line), flush=True)


def run_stream_reference(args):
    from bondupdategalerkin_b200 import workloads as WL

    specs = WL.batch_specs(args.jobs or 64) if KIND[0] == "batch" else \
        WL.served_specs(args.jobs or 48, rate=20.0, scale=args.scale)
    workers = args.workers or min(16, os.cpu_count() or 1)
    n, secs = stream_cpu_sample_concurrent(specs, [None] * len(specs), workers)
    value = n / secs
    print(json.dumps({"impl": "reference", "metric": "chain_steps_per_s" if KIND[0] == "batch"
                      else "served_steps_per_s", "value": value, "unit": "steps/s", "n_gpus": 1,
                      "steps": n, "warmup": 0, "higher_is_better": True, "dtype": "c128",
                      "cpu_baseline": {"value": value, "unit": "steps/s", "cores": workers,
                                       "kind": "port",
                                       "sample": f"CPU oracle, the first step of {n} jobs spread "
                                                 f"over the stream, {workers} processes at once "
                                                 f"on one BLAS thread each"},
                      "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0,
                              "d2h_bytes_per_step": 0}}), flush=True)


def _rand_device_tensor(DT, rng, dirs, sectors):
    """A device tensor with every charge-conserving block present and Gaussian entries."""
    import itertools

    legs = [DT.Leg(d, s) for d, s in zip(dirs, sectors)]
    blocks = {}
    for key in itertools.product(*[sorted(s) for s in sectors]):
        if sum(d * q for d, q in zip(dirs, key)) != 0:
            continue
        shape = tuple(s[q] for s, q in zip(sectors, key))
        blocks[key] = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    return DT.from_blocks(legs, blocks)


def envpush_inputs(DT, rng, kind, D=256):
    """E (bra, w, ket), A (l, s, r), W (w_l, s_in, s_out, w_r) of a chi = D environment push: one
    dense block per tensor (no symmetry), or U(1) with 33 link sectors of a Gaussian profile summing
    to D and the XXZ MPO's sectors (w = 5: charges -2, 0 x 3, +2)."""
    if kind == "dense":
        link, wl, sl = {0: D}, {0: 5}, {0: 2}
        rlink = link
    else:
        qs = list(range(-32, 33, 2))
        wts = np.exp(-np.array(qs, float) ** 2 / (2 * 12.0 ** 2))
        dims = np.maximum(1, np.floor(wts / wts.sum() * D)).astype(int)
        dims[len(qs) // 2] += D - dims.sum()
        link, wl, sl = {q: int(d) for q, d in zip(qs, dims)}, {-2: 1, 0: 3, 2: 1}, {-1: 1, 1: 1}
        rlink = {q + 1: d for q, d in link.items()}
    E = _rand_device_tensor(DT, rng, (-1, +1, +1), (link, wl, link))
    A = _rand_device_tensor(DT, rng, (-1, -1, +1), (link, sl, rlink))
    W = _rand_device_tensor(DT, rng, (-1, +1, -1, +1), (wl, sl, sl, wl))
    return E, A, W


def run_envpush(args):
    """The environment push E' = A^dag (E A W) (bug_env_step) at chi = 256 on the FP64 stage kernel
    and on the tensor-core 3xTF32 path (blocks of at least 64 x 64), timed with CUDA events on the
    engine stream after an L2 flush; TFLOP/s counts the algorithmic 8 m n k per block pair."""
    import torch

    from bondupdategalerkin_b200 import _engine as E
    from bondupdategalerkin_b200 import build as Bld
    from bondupdategalerkin_b200 import native as N
    from bondupdategalerkin_b200 import tensor as DT

    if Bld.needs_build():
        Bld.build()
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    ctx = E.context(0)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    peaks = {}
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        peaks = json.load(open(p))
    bf16 = peaks.get("bf16_tflops", 1590.0)
    tf32_peak = bf16 / 2.0  # dense TF32 issues at half the BF16 rate
    zgemm = measure_zgemm_tflops(torch, dev)
    out = {"metric": "env_push_tflops", "unit": "TFLOP/s", "n_gpus": 1, "steps": args.steps,
           "warmup": args.warmup, "higher_is_better": True, "dtype": "c128 (fp64) / 3xtf32 (mixed)",
           "data": "synthetic (Gaussian blocks)", "l2": "flushed before every push (256 MiB write)",
           "cases": {},
           "peaks": {"fp64_zgemm_tflops_measured": zgemm,
                     "tf32_dense_tflops": tf32_peak,
                     "tf32_source": ("MEASURED_PEAKS.json bf16_tflops / 2" if "bf16_tflops" in peaks
                                     else "fallback 1590 bf16 / 2")}}
    for kind in ("dense", "u1"):
        rng = np.random.default_rng(5)
        Et, At, Wt = envpush_inputs(DT, rng, kind)
        res = {}
        results = {}
        for mode, min_dim in (("fp64", 0), ("mixed", 64)):
            ctx.set_mixed(min_dim)
            for _ in range(args.warmup):
                N.env_step(Et, At, Wt, "left")
            ctx.synchronize()
            ctx.reset_stats()
            times = []
            for _ in range(args.steps):
                with torch.cuda.stream(stream):
                    flush.zero_()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                r = N.env_step(Et, At, Wt, "left")
                e1.record(stream)
                times.append((e0, e1))
            ctx.synchronize()
            torch.cuda.synchronize(dev)
            ms = statistics.median(a.elapsed_time(b) for a, b in times)
            st = ctx.kernel_stats()
            flops = (st["gemm"]["flops"] + st["mixed"]["flops"]) / args.steps
            results[mode] = DT.to_blocks(r)[1]
            res[mode] = {"ms_per_push": ms, "tflops": flops / (ms / 1e3) / 1e12,
                         "gflop_per_push": flops / 1e9,
                         "mixed_share_of_flops": st["mixed"]["flops"] / max(st["gemm"]["flops"] + st["mixed"]["flops"], 1.0),
                         "launches_per_push": (st["gemm"]["launches"] + st["mixed"]["launches"]) / args.steps}
        ctx.set_mixed(0)
        num = max(float(np.max(np.abs(results["mixed"][k] - v))) for k, v in results["fp64"].items())
        den = max(float(np.max(np.abs(v))) for v in results["fp64"].values())
        res["mixed_rel_err_vs_fp64"] = num / den
        res["fp64_frac_of_zgemm"] = res["fp64"]["tflops"] / zgemm
        # the tensor pipe does three TF32 products per algorithmic one
        res["mixed_tensor_frac_of_tf32_peak"] = 3.0 * res["mixed"]["tflops"] / tf32_peak
        res["speedup_mixed_vs_fp64"] = res["fp64"]["ms_per_push"] / res["mixed"]["ms_per_push"]
        out["cases"][kind] = res
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=97)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--cpu-steps", type=int, default=5)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-replay", action="store_true",
                    help="time the steps only (for profiler runs)")
    ap.add_argument("--L", type=int, default=None,
                    help="chain length override (smaller cases for profiler captures only)")
    ap.add_argument("--workload", default="xxz",
                    choices=["xxz", "heston", "tdvp2", "ite", "batch", "served", "envpush"],
                    help="xxz: the L = 64 XXZ quench (the headline); heston: the 10 + 10-bit "
                         "Heston QTT field (47 timed steps after 3 warm-up make its 50); tdvp2: the "
                         "two-site TDVP baseline over the headline's 100-step trajectory; ite: normalised "
                         "imaginary time on the L = 32 Heisenberg chain (29 timed steps of dbeta "
                         "0.125 after 3 warm-up reach beta 4); batch: 64 chains at once on the job server; served: a Poisson "
                         "job stream")
    ap.add_argument("--parallel", action="store_true",
                    help="parallel = true: the half-sweeps and frontier halves on two streams")
    ap.add_argument("--mixed", type=int, default=0,
                    help="contraction blocks with both extents >= this run on the tensor cores "
                         "(3xTF32); 0 (default): everything in FP64")
    ap.add_argument("--workers", type=int, default=0, help="job server workers (0: min(16, cores))")
    ap.add_argument("--jobs", type=int, default=0, help="batch/served: number of jobs")
    ap.add_argument("--scale", type=float, default=0.25,
                    help="served: shrink the stream's size ranges toward their lower ends")
    args = ap.parse_args()
    KIND[0] = args.workload
    PARALLEL[0] = args.parallel
    if args.workload == "heston" and "--steps" not in sys.argv:
        args.steps = 47
    if args.workload == "ite" and "--steps" not in sys.argv:
        args.steps = 29
    if args.warmup < 3:
        print("warning: fewer than 3 warm-up steps", file=sys.stderr)
    if args.L is not None:
        WORKLOAD["L"] = args.L
        global WORKLOAD_NAME
        WORKLOAD_NAME = WORKLOAD_NAME.replace("L64", f"L{args.L}")
    if args.workload == "envpush":
        run_envpush(args)
        return
    if args.workload in ("batch", "served"):
        if args.impl == "reference":
            if dist_env()[1] == 0:
                run_stream_reference(args)
        elif dist_env()[1] == 0:
            run_stream(args)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_engine(args)


if __name__ == "__main__":
    main()
