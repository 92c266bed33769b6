"""Independent replicas of a chain's step, one process per GPU.

One chain's BUG step is a sequential chain of bond updates: it does not shard over GPUs, so N GPUs
run N independent replicas and no collective touches the data path. The only collectives are the
timing ones a benchmark needs: a barrier on both sides of the timed region and the maximum of each
rank's device time. Every rank takes the same collective steps in the same order.

The plumbing is backend-agnostic: ``nccl`` on GPUs (the timing tensor lives on the rank's device),
``gloo`` on CPU (multi-process tests). The process group gets a short timeout, so a rank whose
peer died ends its next collective with an error instead of waiting.
"""

from __future__ import annotations

import datetime
import os

DEFAULT_TIMEOUT_S = 180


def world() -> tuple[int, int, int]:
    """``(world_size, rank, local_rank)`` from the launcher's environment (1, 0, 0 without one)."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


class Replicas:
    """The timing collectives of N replicas. With a world size of 1 every call is local."""

    def __init__(self, backend: str = "nccl", device=None, timeout_s: float = DEFAULT_TIMEOUT_S):
        import torch

        self.size, self.rank, self.local = world()
        self.device = device if device is not None else torch.device("cpu")
        self._torch = torch
        self._dist = None
        if self.size > 1:
            import torch.distributed as dist

            kw = dict(timeout=datetime.timedelta(seconds=timeout_s))
            if backend == "nccl":
                kw["device_id"] = self.device
            dist.init_process_group(backend, **kw)
            self._dist = dist

    def barrier(self) -> None:
        if self._dist is not None:
            self._dist.barrier()

    def max(self, x: float) -> float:
        """The largest ``x`` over the ranks (every rank gets it)."""
        if self._dist is None:
            return float(x)
        t = self._torch.tensor([float(x)], dtype=self._torch.float64, device=self.device)
        self._dist.all_reduce(t, op=self._dist.ReduceOp.MAX)
        return float(t.item())

    def rate(self, units_per_rank: float, ms_local: float) -> tuple[float, float]:
        """Whole-job throughput: all ranks' units over the slowest rank's time. Returns
        ``(units per second, the max-over-ranks milliseconds)``."""
        ms = self.max(ms_local)
        return self.size * units_per_rank / (ms / 1e3), ms

    def close(self) -> None:
        if self._dist is not None:
            self._dist.destroy_process_group()
            self._dist = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
        return False
