"""The N-replica path (one process per GPU, timing collectives only) on CPU with ``gloo``.

One chain's step does not shard, so ``bench.py --gpus N`` runs N independent replicas; the only
collectives are a barrier and the max over ranks of each rank's device time. These tests run that
plumbing (``bondupdategalerkin_b200/replicas.py``) as two ``gloo`` ranks in child processes, and a
rank that leaves early, whose peer must end its next collective with an error, not wait.
"""

from __future__ import annotations

import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _env(rank: int, ws: int, port: int) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(ws),
                      RANK=str(rank), LOCAL_RANK=str(rank))


def _timing_rank(rank, ws, port, out):
    _env(rank, ws, port)
    sys.path.insert(0, ROOT)
    from bondupdategalerkin_b200.replicas import Replicas

    with Replicas("gloo", timeout_s=60) as reps:
        reps.barrier()
        value, ms = reps.rate(97, 100.0 + 50.0 * rank)  # rank 1 is the slowest
        lowest = -reps.max(-float(rank))
        reps.barrier()
        out.put((rank, reps.size, value, ms, lowest))


def _leaving_rank(rank, ws, port, out):
    _env(rank, ws, port)
    sys.path.insert(0, ROOT)
    from bondupdategalerkin_b200.replicas import Replicas

    reps = Replicas("gloo", timeout_s=10)
    reps.barrier()
    if rank == 1:
        out.put((rank, "left"))
        out.close()
        out.join_thread()  # the message is out before the process ends
        os._exit(0)  # leaves between steps, with no collective in flight
    try:
        reps.max(1.0)
        out.put((rank, "no error"))
    except Exception as exc:  # the backend's error type differs between torch versions
        out.put((rank, f"error: {type(exc).__name__}"))


def _spawn(target, ws):
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=target, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    try:
        res = sorted(q.get(timeout=120) for _ in range(ws))
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    return res, [p.exitcode for p in procs]


def test_two_gloo_replicas_agree_on_the_slowest_rank():
    res, codes = _spawn(_timing_rank, 2)
    assert codes == [0, 0]
    for rank, size, value, ms, lowest in res:
        assert size == 2
        assert ms == 150.0  # the max over ranks, on every rank
        assert value == pytest.approx(2 * 97 / 0.150)  # all ranks' steps over the slowest time
        assert lowest == 0.0


def test_a_rank_that_leaves_ends_its_peers_collective_with_an_error():
    res, _ = _spawn(_leaving_rank, 2)
    assert res[1] == (1, "left")
    assert res[0][0] == 0 and res[0][1].startswith("error"), res


def test_single_process_needs_no_process_group(monkeypatch):
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    from bondupdategalerkin_b200.replicas import Replicas

    with Replicas("nccl") as reps:  # no group is made for one rank, so no device is touched
        assert (reps.size, reps.rank) == (1, 0)
        reps.barrier()
        assert reps.rate(10, 500.0) == (20.0, 500.0)


def _bench(args, **env):
    e = dict(os.environ, **env)
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], env=e,
                          capture_output=True, text=True, timeout=600, cwd=ROOT)


def test_reference_arm_prints_one_line_on_rank_zero_only():
    """``bench.py --impl reference`` (the CPU oracle on the headline quench) keeps the JSON
    contract; under a launcher only rank 0 runs and prints, the other ranks exit 0 at once."""
    r = _bench(["--impl", "reference", "--steps", "1", "--warmup", "3"])
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    line = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
                "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference" and line["unit"] == "steps/s" and line["value"] > 0
    assert line["config"]["workload"].startswith("xxz_quench_L64")
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "port"

    r1 = _bench(["--impl", "reference", "--steps", "1", "--warmup", "3"],
                WORLD_SIZE="2", RANK="1", LOCAL_RANK="1")
    assert r1.returncode == 0 and r1.stdout.strip() == ""


@pytest.mark.parametrize("workload,metric", [("tdvp2", "tdvp2_steps_per_s"), ("ite", "ite_steps_per_s")])
def test_reference_arm_other_workloads(workload, metric):
    """The reference arm keeps the same contract on the TDVP2 and imaginary-time workloads."""
    r = _bench(["--impl", "reference", "--workload", workload, "--steps", "1", "--warmup", "3"])
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads([ln for ln in r.stdout.splitlines() if ln.strip()][-1])
    assert line["impl"] == "reference" and line["metric"] == metric and line["value"] > 0
    assert line["config"]["workload"].startswith(workload) and line["higher_is_better"] is True
