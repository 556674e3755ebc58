"""The oracle's transforms and Poisson solve against FFTW 3.3.9 itself.

The reference transforms with FFTW (R2HC / HC2R, src/m_Poisson.f90:180-244,
executes at :371-373,433-435) pinned at version 3.3.9
(src/ThirdParty/install_thirdParty.sh:12).  oracle/fftw/Makefile builds that
library from the tarball the reference carries into oracle/_ref/ (test
infrastructure; the product never loads it).  These tests check

- the oracle's restated R2HC and HC2R against FFTW's, for every length the
  compiled transforms cover (radices 2, 3, 5), to 1e-14 of the largest
  coefficient;
- the oracle's clcPPE_x1 against an independent restatement of it
  (src/m_Poisson.f90:352-452) whose x and z transforms are FFTW's R2HC /
  HC2R and whose wall-normal systems are solved per halfcomplex slot with
  scipy's banded solver: 1e-12 of max|phi|, the Poisson tolerance of the
  GPU parity tests.

Skipped when the library has not been built (no reference sources here).
"""
import ctypes
import os

import numpy as np
import pytest
from scipy.linalg import solve_banded

from oracle import oracle_lib as ol
from paratc_b200 import cases

from .helpers import yp_of

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "oracle", "_ref", "libfftw3_ref.so")
FFTW_R2HC, FFTW_HC2R, FFTW_ESTIMATE = 0, 1, 1 << 6

pytestmark = pytest.mark.skipif(not os.path.exists(LIB), reason="FFTW checker not built (oracle/fftw/Makefile)")


def _fftw():
    L = ctypes.CDLL(LIB)
    L.fftw_plan_r2r_1d.restype = ctypes.c_void_p
    L.fftw_plan_r2r_1d.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_uint]
    L.fftw_execute_r2r.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    L.fftw_destroy_plan.argtypes = [ctypes.c_void_p]
    return L


class R2R:
    """One FFTW r2r plan of length n, executed on any contiguous rows."""

    def __init__(self, L, n, kind):
        self.L, self.n = L, n
        a, b = np.zeros(n), np.zeros(n)
        self.plan = L.fftw_plan_r2r_1d(n, a.ctypes.data, b.ctypes.data, kind, FFTW_ESTIMATE)

    def rows(self, x):
        """The transform of every row of x (last axis of length n)."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        flat = x.reshape(-1, self.n)
        out = np.empty_like(flat)
        for r in range(flat.shape[0]):
            src, dst = np.ascontiguousarray(flat[r]), out[r]
            self.L.fftw_execute_r2r(self.plan, src.ctypes.data, dst.ctypes.data)
        return out.reshape(x.shape)

    def close(self):
        self.L.fftw_destroy_plan(self.plan)


LENGTHS = [4, 6, 8, 10, 12, 16, 24, 30, 32, 40, 48, 60, 64, 96, 120, 128, 192, 256, 384, 512, 768, 1024, 1152,
           1536, 2304]


@pytest.mark.parametrize("n", LENGTHS)
def test_oracle_halfcomplex_matches_fftw(n):
    L = _fftw()
    rng = np.random.Generator(np.random.PCG64(n))
    x = rng.standard_normal(n)
    fwd, bwd = R2R(L, n, FFTW_R2HC), R2R(L, n, FFTW_HC2R)
    hc_f = fwd.rows(x)
    hc_o = ol.r2hc(x)
    assert np.abs(hc_o - hc_f).max() <= 1e-14 * np.abs(hc_f).max()
    # the unnormalised inverse of a halfcomplex array
    y_f = bwd.rows(hc_f)
    y_o = ol.hc2r(hc_f)
    assert np.abs(y_o - y_f).max() <= 1e-14 * np.abs(y_f).max()
    assert np.abs(y_f / n - x).max() <= 1e-14 * np.abs(x).max()
    fwd.close()
    bwd.close()


def _ppe_with_fftw(L, o, p, src):
    """clcPPE_x1 (src/m_Poisson.f90:352-452) with FFTW's transforms: R2HC
    along x, then along z; per halfcomplex slot (kx, kz) the wall-normal
    system am2ph phi(j-1) + (ac2ph + lambda_x + lambda_z) phi(j) + ap2ph
    phi(j+1) = f(j), with the kx = kz = 0 row 1 replaced by phi = 0
    (:399-404); HC2R along z, then x; times normfft = 1/(nxc nzc)."""
    nx, ny, nz = p.nxc, p.nyc, p.nzc
    am, ac, ap = o.metric("am2ph"), o.metric("ac2ph"), o.metric("ap2ph")
    wx, wz = o.metric("WaveNumX"), o.metric("WaveNumZ")
    fx, fz = R2R(L, nx, FFTW_R2HC), R2R(L, nz, FFTW_R2HC)
    bx, bz = R2R(L, nx, FFTW_HC2R), R2R(L, nz, FFTW_HC2R)
    s = fx.rows(src)                                   # [z][y][x-slot]
    s = fz.rows(np.moveaxis(s, 0, 2)).copy()           # [y][x-slot][z-slot]
    phi_h = np.empty_like(s)
    for i in range(nx):
        for k in range(nz):
            b = ac + wx[i] + wz[k]
            rhs = s[:, i, k].copy()
            ab = np.zeros((3, ny))
            ab[0, 1:] = ap[:-1]
            ab[1, :] = b
            ab[2, :-1] = am[1:]
            if i == 0 and k == 0:
                ab[1, 0], ab[0, 1], rhs[0] = 1.0, 0.0, 0.0
            phi_h[:, i, k] = solve_banded((1, 1), ab, rhs)
    t = bz.rows(phi_h)                                 # [y][x-slot][z]
    phi = bx.rows(np.moveaxis(t, 2, 0))                # [z][y][x]
    for r in (fx, fz, bx, bz):
        r.close()
    return phi / (nx * nz)


@pytest.mark.parametrize("dims", [(32, 24, 16), (24, 20, 30), (48, 36, 60)])
def test_oracle_poisson_matches_fftw_restatement(dims):
    L = _fftw()
    case = cases.small_channel(*dims)
    p = case.params
    yp = yp_of(case)
    o = ol.Oracle(p, yp)
    src = cases.gaussian_source(cases.Case("src", p, case.mesh, "gauss_src", 42, 1.0))
    ref = _ppe_with_fftw(L, o, p, src)
    got = o.poisson(src)
    o.close()
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()
