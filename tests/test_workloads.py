"""The batched and served job streams (``bondupdategalerkin_b200/workloads.py``) on CPU: seeded,
reproducible, and inside the ranges the workloads are specified with (64 XXZ chains with
L in {32, 48, 64, 96}, maxdim in {64, 128, 256}, total S^z = 0, 50 steps; a Poisson stream at
20 jobs/s, 70 % XXZ / 30 % Heston, with the scaled ranges shrinking toward their lower ends).
"""

import numpy as np
import pytest

from bondupdategalerkin_b200 import workloads as W


def test_batch_stream():
    a, b = W.batch_specs(64), W.batch_specs(64)
    assert a == b  # reproducible
    assert len(a) == 64 and len({s["seed"] for s in a}) == 64
    for s in a:
        assert s["L"] in (32, 48, 64, 96) and s["kw"]["maxdim"] in (64, 128, 256)
        assert -1.0 <= s["delta"] <= 1.0 and s["nsteps"] == 50 and s["tau"] == -0.02j
        assert s["spins"].count("up") == s["L"] // 2  # total S^z = 0
        assert s["kw"]["order"] == 2


@pytest.mark.parametrize("scale", [1.0, 0.25])
def test_served_stream(scale):
    a = W.served_specs(1000, rate=20.0, scale=scale)
    assert a == W.served_specs(1000, rate=20.0, scale=scale)
    arrivals = np.array([s["arrival"] for s in a])
    assert np.all(np.diff(arrivals) > 0)
    gaps = np.diff(np.concatenate([[0.0], arrivals]))
    assert abs(gaps.mean() - 1 / 20) < 0.1 / 20  # Poisson at 20 jobs/s
    xxz = [s for s in a if s["kind"] == "xxz"]
    hes = [s for s in a if s["kind"] == "heston"]
    assert abs(len(xxz) / len(a) - 0.7) < 0.05
    top = lambda lo, hi: lo + round((hi - lo) * scale)  # noqa: E731
    for s in xxz:
        assert 16 <= s["L"] <= top(16, 128) and 32 <= s["kw"]["maxdim"] <= top(32, 512)
        assert 20 <= s["nsteps"] <= top(20, 200) and s["tau"] == -0.05j
        neel = s["spins"][:2] == ["up", "down"]
        assert (s["kw"].get("work_ceiling_rule") == "maxdim") == neel
    for s in hes:
        r, q, kappa, theta, sigma, rho = s["params"]
        assert 8 <= s["bits"] <= top(8, 11) and 32 <= s["kw"]["maxdim"] <= top(32, 128)
        assert 10 <= s["nsteps"] <= top(10, 50) and s["kw"]["hermitian"] is False
        assert 0 <= r <= 0.05 and q == 0 and 1 <= kappa <= 3 and 0.04 <= theta <= 0.12
        assert 0.2 <= sigma <= 0.6 and -0.9 <= rho <= -0.3
    if scale < 1:
        assert max(s["L"] for s in xxz) <= 44 and max(s["bits"] for s in hes) <= 9
