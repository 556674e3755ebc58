"""Parity at the benchmark sizes themselves.

C2 (512 x 256 x 512) reaches the kernels only large grids use (the streaming
y-solve, 512-point z transforms, 256-point x transforms); the oracle solves
it in a few seconds on the host.  C1 (128 x 96 x 128) is the bench workload:
two full RK3 steps against the oracle, the solenoidality of the result, and
the 1-D spectra of the stepped fields.
Tolerances as in test_gpu_parity (Poisson 1e-12 relative to max|phi|; fields
after one step 1e-10, after two 1e-8).
"""
import numpy as np
import pytest

from oracle import oracle_lib as ol
from paratc_b200 import cases
from paratc_b200.lib import ChannelSystem

from .helpers import fields_of, rel_err, yp_of

pytestmark = pytest.mark.gpu


def test_poisson_c2_full_size():
    case = cases.poisson_c2()
    yp = yp_of(case)
    src = cases.gaussian_source(cases.Case("src", case.params, case.mesh, "gauss_src", 42, 1.0))
    phi_o = ol.Oracle(case.params, yp).poisson(src)
    g = ChannelSystem(case.params, yp)
    phi_g = g.poisson(src)
    e = rel_err(phi_g, phi_o)
    assert e <= 1e-12, "C2 poisson rel err %.3e" % e
    # linearity: solve(2 src) = 2 solve(src) exactly up to rounding
    phi_2 = g.poisson(2.0 * src)
    assert rel_err(phi_2, 2.0 * phi_g) <= 1e-14
    g.close()


def test_channel_c1_two_steps():
    case = cases.channel_c1()
    yp = yp_of(case)
    f = fields_of(case, yp)
    o = ol.Oracle(case.params, yp)
    g = ChannelSystem(case.params, yp)
    o.set_fields(f["ux"], f["uy"], f["uz"], f["p"], f["c"])
    g.set_fields(f["ux"], f["uy"], f["uz"], f["p"], f["c"])
    o.project()
    g.project()
    for s, tol in ((1, 1e-10), (2, 1e-8)):
        rc, do = o.step()
        assert rc == 0
        dg = g.iterate(1)
        fo, fg = o.get_fields(), g.get_fields()
        for n in ("ux", "uy", "uz", "p", "hx", "hy", "hz"):
            e = rel_err(fg[n], fo[n])
            assert e <= tol, "C1 step %d %s rel err %.3e" % (s, n, e)
        assert dg.divmax <= 1e-10
        assert abs(dg.dt - do.dt) <= 1e-12 * do.dt
    # 1-D spectra at the bench size (128-point x and z transforms, 96 rows),
    # on the oracle's fields loaded into the context: transform rounding only
    fo = o.get_fields()
    g.set_fields(fo["ux"], fo["uy"], fo["uz"], fo["p"])
    jl = 24
    ref = o.spectra(jl)
    g.spectra_accumulate(jl)
    ex, ez, ns = g.spectra_get()
    assert ns == 1
    for got, r in zip((ex, ez), ref):
        for m in range(r.shape[0]):
            e = np.abs(got[m] - r[m]).max() / np.abs(r[m]).max()
            assert e <= 1e-12, "C1 spectrum %d rel err %.3e" % (m + 1, e)
    g.close()
