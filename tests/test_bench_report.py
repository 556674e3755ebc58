"""The bench line's per-kernel roofline fractions (host arithmetic only) and the
reference arm of the Poisson workloads (the oracle on the host)."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import bench  # noqa: E402
from paratc_b200 import cases  # noqa: E402


def test_kernel_fractions():
    p = cases.channel_c1().params
    alg = bench.algorithmic_bytes(p)
    # 3 launches of the RHS in 0.2 ms (66.7 us each) and one check in 0.02 ms
    prof = {"rhs": (0.2, 3), "check": (0.02, 1), "unknown_class": (1.0, 1), "fft_x_fwd": (0.0, 0)}
    fr = bench.kernel_fractions(prof, alg, 6536.0)
    assert set(fr) == {"rhs", "check"}
    assert fr["rhs"] == pytest.approx(alg["rhs"] / (0.2 / 3 / 1e3) / 1e9 / 6536.0, abs=1e-3)
    assert fr["check"] == pytest.approx(alg["check"] / 20e-6 / 1e9 / 6536.0, abs=1e-3)
    assert list(fr) == ["rhs", "check"]  # ordered by total time


def test_algorithmic_bytes_c1():
    p = cases.channel_c1().params
    alg = bench.algorithmic_bytes(p)
    n = 128 * 96 * 128
    assert alg["rhs"] == 13 * 8 * n and alg["helmholtz"] == 9 * 8 * n and alg["project"] == 9 * 8 * n
    s = 2 * 65 * 96 * 128
    assert alg["fft_z_fwd"] == 16 * s and alg["prsrc"] == 8 * (3 * n + s)


def test_reference_arm_of_the_poisson_workloads():
    """--impl reference on the Poisson workloads times the oracle's solve on
    the host and prints one line with the workload's metric (a small grid)."""
    import json
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for wl, scaling in (("poisson_c2", "weak"), ("poisson_c2_zslabs", "strong")):
        out = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--impl", "reference", "--workload", wl,
                              "--grid", "32", "16", "24", "--steps", "2", "--warmup", "1"],
                             capture_output=True, text=True, timeout=300)
        assert out.returncode == 0, out.stderr[-2000:]
        line = json.loads([x for x in out.stdout.splitlines() if x.startswith("{")][-1])
        assert line["impl"] == "reference" and line["metric"] == "grid-point Poisson solves/s"
        assert line["value"] > 0 and line["scaling"] == scaling
        assert line["config"]["grid"] == [32, 16, 24]
        assert line["cpu_baseline"]["kind"] == "port"
