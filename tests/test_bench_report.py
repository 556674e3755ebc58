"""The bench line's per-kernel roofline fractions (host arithmetic only)."""
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
