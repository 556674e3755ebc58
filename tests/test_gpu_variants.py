"""Parity of the alternative kernel variants that size selects automatically.

The spectral y-solve has a staged variant (whole column strips copied to
shared memory first) and a streaming variant (rows streamed from HBM), chosen
by grid size; the Poisson transforms have compile-time-length kernels and a
generic Stockham path for lengths outside their list.  The small grids of
the other tests reach only one variant of each, so here every variant is
forced through the environment (read when a context is created) and
compared with the oracle.  Tolerances as in test_gpu_parity.
"""
import pytest

from oracle import oracle_lib as ol
from paratc_b200 import cases
from paratc_b200.abi import SCHED_NCHOICES
from paratc_b200.lib import ChannelSystem

from .helpers import fields_of, rel_err, variant, yp_of

pytestmark = pytest.mark.gpu

TOL_STEP1 = 1e-10
TOL_STEPS = 1e-8
TOL_POISSON = 1e-12


def _steps_vs_oracle(case, nsteps):
    yp = yp_of(case)
    f = fields_of(case, yp)
    o = ol.Oracle(case.params, yp)
    g = ChannelSystem(case.params, yp)
    o.set_fields(f["ux"], f["uy"], f["uz"], f["p"], f["c"])
    g.set_fields(f["ux"], f["uy"], f["uz"], f["p"], f["c"])
    for s in range(nsteps):
        rc, _ = o.step()
        assert rc == 0
        g.iterate(1, raise_on_guard=False)
        fo, fg = o.get_fields(), g.get_fields()
        tol = TOL_STEP1 if s == 0 else TOL_STEPS
        for n in ("ux", "uy", "uz", "p", "c"):
            if fo.get(n) is None:
                continue
            e = rel_err(fg[n], fo[n])
            assert e <= tol, "%s step %d: %s rel err %.3e" % (case.name, s + 1, n, e)


@pytest.mark.parametrize("solver", ["staged", "streaming"])
@pytest.mark.parametrize("name", ["channel", "halfchannel_scalar"])
def test_solver_variants_steps(monkeypatch, solver, name):
    monkeypatch.setenv("PARATC_YSOLVER", solver)
    _steps_vs_oracle(variant(name), 3)


@pytest.mark.parametrize("solver", [None, "staged", "streaming"])
def test_tall_columns(monkeypatch, solver):
    """A tall grid (ny = 120): long dependent chains in every y-solve."""
    if solver:
        monkeypatch.setenv("PARATC_YSOLVER", solver)
    _steps_vs_oracle(cases.small_channel(16, 120, 8), 2)


@pytest.mark.parametrize("dims", [(24, 20, 30), (32, 24, 16)])
def test_generic_fft_path(monkeypatch, dims):
    monkeypatch.setenv("PARATC_GENERIC_FFT", "1")
    _steps_vs_oracle(cases.small_channel(*dims), 2)
    case = cases.small_channel(*dims)
    yp = yp_of(case)
    src = cases.gaussian_source(cases.Case("src", case.params, case.mesh, "gauss_src", 42, 1.0))
    phi_o = ol.Oracle(case.params, yp).poisson(src)
    phi_g = ChannelSystem(case.params, yp).poisson(src)
    assert rel_err(phi_g, phi_o) <= TOL_POISSON


@pytest.mark.parametrize("dims", [(48, 16, 24), (96, 12, 40), (80, 10, 64), (2048, 10, 16), (2304, 10, 16),
                                  (3072, 10, 16)])
def test_fixed_length_sizes(dims):
    """Other compile-time lengths (nx/2 = 24, 48, 40 and the long rows 1024,
    1152, 1536 of the bulk-copy x transforms; nz = 24, 40, 64, 16)."""
    case = cases.small_channel(*dims)
    yp = yp_of(case)
    src = cases.gaussian_source(cases.Case("src", case.params, case.mesh, "gauss_src", 7, 1.0))
    phi_o = ol.Oracle(case.params, yp).poisson(src)
    phi_g = ChannelSystem(case.params, yp).poisson(src)
    assert rel_err(phi_g, phi_o) <= TOL_POISSON


@pytest.mark.parametrize("plane", [True, False])
@pytest.mark.parametrize("dims", [(64, 24, 64), (96, 20, 96), (128, 96, 128)])
def test_plane_and_split_transforms(monkeypatch, plane, dims):
    """The one-CTA-per-plane transforms (k_plane.cu) and the separate x / z
    kernels on the same grids (plane pairs (32,64), (48,96), (64,128))."""
    if not plane:
        monkeypatch.setenv("PARATC_NO_PLANE", "1")
    case = cases.small_channel(*dims)
    yp = yp_of(case)
    src = cases.gaussian_source(cases.Case("src", case.params, case.mesh, "gauss_src", 11, 1.0))
    phi_o = ol.Oracle(case.params, yp).poisson(src)
    phi_g = ChannelSystem(case.params, yp).poisson(src)
    assert rel_err(phi_g, phi_o) <= TOL_POISSON
    if dims[1] <= 24:
        _steps_vs_oracle(case, 2)


@pytest.mark.parametrize("dims", [(64, 48, 64), (24, 20, 30), (128, 96, 128), (32, 24, 256)])
def test_schedules_and_autotune(dims):
    """Every Poisson schedule this grid supports (fused plane transforms,
    separate fixed-length transforms, generic transforms, separate transforms
    with TMA-fed z passes, the same with the warp-specialised divergence
    source of the x transform; staged or streaming y-solve) gives the oracle's
    fields after two steps; the auto-tuner times all of them and keeps the
    fastest."""
    case = cases.small_channel(*dims)
    yp = yp_of(case)
    f = fields_of(case, yp)
    o = ol.Oracle(case.params, yp)
    o.set_fields(f["ux"], f["uy"], f["uz"], f["p"])
    for _ in range(2):
        o.step()
    fo = o.get_fields()
    g = ChannelSystem(case.params, yp)
    choice, times = g.autotune(nrep=3)
    assert times[choice] > 0 and times[choice] == min(t for t in times if t > 0)
    assert g.schedule == choice
    assert len(times) == SCHED_NCHOICES
    supported = [c for c in range(SCHED_NCHOICES) if times[c] > 0]
    assert 4 in supported and 5 in supported  # the generic transforms take any 2^a 3^b 5^c size
    tma_z = dims[2] in (128, 256, 512, 768, 1024)
    assert 8 in supported and 9 in supported  # the divergence-fed x transform, register-fed z
    assert (6 in supported) == tma_z and (10 in supported) == tma_z and (11 in supported) == tma_z
    for c in range(SCHED_NCHOICES):
        if c not in supported:
            with pytest.raises(Exception):
                g.schedule = c
            continue
        g.schedule = c
        g.set_fields(f["ux"], f["uy"], f["uz"], f["p"])
        g.iterate(2)
        fg = g.get_fields()
        for n in ("ux", "uy", "uz", "p"):
            e = rel_err(fg[n], fo[n])
            assert e <= 1e-8, "schedule %d %s rel err %.3e" % (c, n, e)
    g.close()
