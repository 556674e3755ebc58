"""Parity of the CUDA hot path (through the C ABI) with the CPU oracle.

Tolerances (FP64 on both sides; the kernels contract multiply-adds into FMA,
multiply by precomputed pivot reciprocals where the reference divides, and
sum the FFTs in another order, so results agree to rounding, not bit for
bit):
  - each routine of one substep (clcRhsXYZ, the Helmholtz solves, clcPrSrc,
    clcPPE, the projection): relative max error <= 1e-11
  - Poisson solve: <= 1e-12 (relative to max|phi|)
  - fields after one step: <= 1e-10; after 10 steps: <= 1e-8
"""
import os
import tempfile

import numpy as np
import pytest

from oracle import oracle_lib as ol
from paratc_b200 import cases
from paratc_b200.lib import ChannelSystem

from .helpers import VARIANTS, discrete_poiseuille, fields_of, rel_err, variant, yp_of

pytestmark = pytest.mark.gpu

TOL_STAGE = 1e-11
TOL_POISSON = 1e-12
TOL_STEP1 = 1e-10
TOL_STEP10 = 1e-8


def _pair(case):
    yp = yp_of(case)
    f = fields_of(case, yp)
    o = ol.Oracle(case.params, yp)
    g = ChannelSystem(case.params, yp)
    o.set_fields(f["ux"], f["uy"], f["uz"], f["p"], f["c"])
    g.set_fields(f["ux"], f["uy"], f["uz"], f["p"], f["c"])
    return o, g, yp


def _cmp_fields(o, g, names, tol, what):
    fo = o.get_fields()
    fg = g.get_fields()
    for n in names:
        if fo.get(n) is None:
            continue
        e = rel_err(fg[n], fo[n])
        assert e <= tol, "%s: %s rel err %.3e > %.1e" % (what, n, e, tol)


@pytest.mark.parametrize("name", VARIANTS)
@pytest.mark.parametrize("stage", [1, 2, 3, 4, 5])
def test_substep_stage(name, stage):
    case = variant(name)
    o, g, _ = _pair(case)
    # one full substep first so the histories are non-zero, then ns = 2 staged
    ns_first = 1
    dt = case.params.dt_max
    o.substep(ns_first, dt)
    g.substep(ns_first, dt)
    ns = 2 if case.params.ischeme != 1 else 1
    dmo = o.substep(ns, dt, stop_stage=stage)
    dmg = g.substep_stage(ns, dt, stage)
    p = case.params
    if stage == 1:
        for n in ["rhsx", "rhsy", "rhsz"] + (["rhsc"] if p.scalar_on else []):
            e = rel_err(g.get_work(n), o.get_work(n))
            assert e <= TOL_STAGE, "%s %s rel err %.3e" % (name, n, e)
        _cmp_fields(o, g, ["hx", "hy", "hz", "hc"], TOL_STAGE, name + " hist")
    elif stage == 2:
        _cmp_fields(o, g, ["ux", "uy", "uz", "c"], TOL_STAGE, name + " helmholtz")
    elif stage == 3:
        e = rel_err(g.get_work("prsrc"), o.get_work("prsrc"))
        assert e <= TOL_STAGE, "%s prsrc rel err %.3e" % (name, e)
        assert abs(dmg - dmo) <= 1e-10 * max(abs(dmo), 1e-300)
    elif stage == 4:
        e = rel_err(g.get_work("phi"), o.get_work("phi"))
        assert e <= TOL_STAGE, "%s phi rel err %.3e" % (name, e)
    else:
        _cmp_fields(o, g, ["ux", "uy", "uz", "p", "c"], TOL_STAGE, name + " substep")


@pytest.mark.parametrize("name", VARIANTS)
def test_steps(name):
    case = variant(name)
    o, g, _ = _pair(case)
    for s in range(10):
        rco, do = o.step()
        dg = g.iterate(1, raise_on_guard=False)
        assert rco == 0
        tol = TOL_STEP1 if s == 0 else TOL_STEP10
        _cmp_fields(o, g, ["ux", "uy", "uz", "p", "c", "hx", "hy", "hz", "hc"], tol, "%s step %d" % (name, s + 1))
        assert abs(dg.dt - do.dt) <= 1e-12 * do.dt
        assert abs(dg.sim_time - do.sim_time) <= 1e-12 * max(do.sim_time, 1e-300)
        for q in range(3):
            assert abs(dg.vmax[q] - do.vmax[q]) <= 1e-9 * max(do.vmax[q], 1e-300)
        assert abs(dg.ux_mean - do.ux_mean) <= 1e-10 * max(abs(do.ux_mean), 1e-3)
        assert dg.divmax <= 1e-8
        assert abs(dg.pr_grad_aver - do.pr_grad_aver) <= 1e-8 * max(abs(do.pr_grad_aver), 1e-6)


@pytest.mark.parametrize("dims", [(16, 12, 16), (32, 24, 16), (24, 20, 30), (64, 48, 40), (128, 96, 128)])
def test_poisson_parity(dims):
    case = cases.small_channel(*dims)
    yp = yp_of(case)
    src = cases.gaussian_source(cases.Case("src", case.params, case.mesh, "gauss_src", 42, 1.0))
    o = ol.Oracle(case.params, yp)
    g = ChannelSystem(case.params, yp)
    phi_o = o.poisson(src)
    phi_g = g.poisson(src)
    e = rel_err(phi_g, phi_o)
    assert e <= TOL_POISSON, "poisson %s rel err %.3e" % (dims, e)


def test_poisson_manufactured():
    """phi = cos(2 pi x/Lx * 3) cos(2 pi z/Lz * 2) g(y): the source built with
    the discrete operator (4th-order x/z second derivative D4oD4, Neumann
    a?2ph in y) is inverted back to phi."""
    case = cases.small_channel(32, 24, 24)
    p = case.params
    yp = yp_of(case)
    o = ol.Oracle(p, yp)
    g = ChannelSystem(p, yp)
    nx, ny, nz = p.nxc, p.nyc, p.nzc
    x = np.arange(nx) * p.xlx / nx
    z = np.arange(nz) * p.zlz / nz
    yc = cases.cell_centres_y(yp)
    gy = np.cos(np.pi * yc / p.yly) + 0.3 * yc
    phi = np.cos(2 * np.pi * 3 * x / p.xlx)[None, None, :] * np.cos(2 * np.pi * 2 * z / p.zlz)[:, None, None] * gy[None, :, None]
    wx = o.metric("WaveNumX")[3]
    wz = o.metric("WaveNumZ")[2]
    am, ac, ap = o.metric("am2ph"), o.metric("ac2ph"), o.metric("ap2ph")
    Ly = np.diag(ac) + np.diag(am[1:], -1) + np.diag(ap[:-1], 1)
    lyphi = np.einsum("ij,kjl->kil", Ly, phi)
    src = lyphi + (wx + wz) * phi
    out = g.poisson(src)
    assert rel_err(out, phi) <= 1e-12


def test_project_divergence_and_parity():
    case = cases.small_channel(32, 24, 32)
    yp = yp_of(case)
    f = cases.initial_fields(case, yp)
    o = ol.Oracle(case.params, yp)
    g = ChannelSystem(case.params, yp)
    o.set_fields(f["ux"], f["uy"], f["uz"], f["p"])
    g.set_fields(f["ux"], f["uy"], f["uz"], f["p"])
    dmo = o.project()
    dmg = g.project()
    assert dmg < 1e-12 and dmo < 1e-12
    _cmp_fields(o, g, ["ux", "uy", "uz"], 1e-12, "project")


def test_poiseuille_fixed_point():
    case = cases.small_channel(16, 24, 16)
    p = case.params
    yp = yp_of(case)
    o = ol.Oracle(p, yp)
    u = discrete_poiseuille(o, p)
    shape = (p.nzc, p.nyc, p.nxc)
    ux = np.broadcast_to(u[None, :, None], shape).copy()
    z = np.zeros(shape)
    g = ChannelSystem(p, yp)
    g.set_fields(ux, z, z, z)
    g.iterate(3)
    fg = g.get_fields(["ux", "uy", "uz"])
    assert np.abs(fg["ux"] - ux).max() < 1e-13 * 10
    assert np.abs(fg["uy"]).max() < 1e-13 and np.abs(fg["uz"]).max() < 1e-13


def test_diagnostics_parity():
    case = variant("halfchannel_scalar")
    o, g, _ = _pair(case)
    do = o.diagnostics()
    dg = g.diagnostics()
    assert abs(dg.divmax - do.divmax) <= 1e-12 * max(do.divmax, 1e-300)
    for q in range(3):
        assert dg.vmax[q] == pytest.approx(do.vmax[q], rel=1e-14)
    assert dg.ux_mean == pytest.approx(do.ux_mean, rel=1e-12)
    assert dg.sc_mean == pytest.approx(do.sc_mean, rel=1e-12)
    assert dg.sc2_mean == pytest.approx(do.sc2_mean, rel=1e-12)


def test_restart_roundtrip_bytes():
    case = variant("channel_scalar_crf")
    o, g, _ = _pair(case)
    g.iterate(2)
    with tempfile.TemporaryDirectory() as d:
        a = os.path.join(d, "RestartForTest0000000002")
        b = os.path.join(d, "again")
        g.write_restart(a, with_hist=True)
        g2 = ChannelSystem(case.params, yp_of(case))
        g2.read_restart(a)
        g2.write_restart(b, with_hist=True)
        assert open(a, "rb").read() == open(b, "rb").read()
        n = case.params.nxc * case.params.nyc * case.params.nzc * 8
        assert os.path.getsize(a) == 9 * n
        # first record is ux + uCRF in Fortran order
        rec = np.fromfile(a, dtype=np.float64, count=n // 8).reshape(g.shape)
        assert rel_err(rec - case.params.ucrf, g.get_fields(["ux"])["ux"]) < 1e-15


def test_halo_layout_roundtrip():
    case = variant("channel")
    o, g, _ = _pair(case)
    g.iterate(1)
    o.step()
    from paratc_b200.abi import LAYOUT_HALO
    fh = g.get_fields(["ux", "p"], layout=LAYOUT_HALO)
    ho = o.get_halo("ux")
    inner = (slice(2, -2), slice(1, -1), slice(2, -2))
    assert rel_err(fh["ux"][inner], ho[inner]) < 1e-9


@pytest.mark.parametrize("name", ["channel", "channel_odd", "halfchannel_scalar", "channel_scalar_crf"])
def test_stats_accumulate(name):
    """clcStat accumulated over two steps on both sides: every moment of every
    row within 1e-11 (the per-routine tolerance) of the moment's largest
    magnitude over the rows; moments such as <w p> are small differences of
    large products, so the fields' rounding-level differences are amplified."""
    case = variant(name)
    o, g, _ = _pair(case)
    acc = None
    for _ in range(2):
        o.step()
        g.iterate(1, raise_on_guard=False)
        so = o.stats()
        acc = so if acc is None else acc + so
        g.stats_accumulate()
    sg, nf, pg = g.stats_get()
    assert nf == 2
    assert sg.shape == acc.shape
    for q in range(acc.shape[1]):
        scale = max(np.abs(acc[:, q]).max(), 1e-300)
        e = np.abs(sg[:, q] - acc[:, q]).max() / scale
        assert e <= TOL_STAGE or scale < 1e-14, "%s moment %d rel err %.3e" % (name, q + 1, e)
    g.stats_reset()
    sg, nf, pg = g.stats_get()
    assert nf == 0 and not sg.any() and pg == 0.0


@pytest.mark.parametrize("name", ["channel", "channel_odd", "halfchannel_scalar", "channel_scalar_crf"])
def test_spectra_accumulate(name):
    """clcStat's 1-D spectra (energy, cospectra, linear coherence) summed over
    two samples on both sides: every spectrum within 1e-11 of its largest
    magnitude (the fields already differ at rounding level after a step)."""
    case = variant(name)
    o, g, _ = _pair(case)
    ny = case.params.nyc
    acc = None
    for s, jl in enumerate((max(1, ny // 5), 1)):
        o.step()
        g.iterate(1, raise_on_guard=False)
        so = o.spectra(jl)
        acc = so if acc is None else (acc[0] + so[0], acc[1] + so[1])
        g.spectra_accumulate(jl)
    ex, ez, ns = g.spectra_get()
    assert ns == 2
    for got, ref in zip((ex, ez), acc):
        assert got.shape == ref.shape
        for m in range(ref.shape[0]):
            scale = max(np.abs(ref[m]).max(), 1e-300)
            e = np.abs(got[m] - ref[m]).max() / scale
            assert e <= TOL_STAGE, "%s spectrum %d rel err %.3e" % (name, m + 1, e)
    with pytest.raises(Exception):
        g.spectra_accumulate(0)
    with pytest.raises(Exception):
        g.spectra_accumulate(ny + 1)
    g.spectra_reset()
    ex, ez, ns = g.spectra_get()
    assert ns == 0 and not ex.any() and not ez.any()


@pytest.mark.parametrize("name", ["channel", "halfchannel_scalar"])
def test_spectra_same_fields(name):
    """On identical fields (the oracle's, after a step, loaded into the
    context) the spectra differ only by the transforms' rounding: 1e-12 of
    each spectrum's largest magnitude."""
    case = variant(name)
    o, g, _ = _pair(case)
    o.step()
    fo = o.get_fields()
    g.set_fields(fo["ux"], fo["uy"], fo["uz"], fo["p"], fo["c"])
    jl = max(1, case.params.nyc // 3)
    ref = o.spectra(jl)
    g.spectra_reset()
    g.spectra_accumulate(jl)
    ex, ez, ns = g.spectra_get()
    assert ns == 1
    for got, r in zip((ex, ez), ref):
        for m in range(r.shape[0]):
            e = np.abs(got[m] - r[m]).max() / max(np.abs(r[m]).max(), 1e-300)
            assert e <= 1e-12, "%s spectrum %d rel err %.3e" % (name, m + 1, e)


@pytest.mark.parametrize("name", ["channel", "halfchannel_scalar", "channel_odd"])
def test_spectra2d_accumulate(name):
    """clcStat's 2-D spectra (halfcomplex-of-halfcomplex x-z transforms at
    the rows iySpec2D) on identical fields, two samples: 1e-12 of each
    spectrum's largest magnitude; out-of-range rows are rejected."""
    case = variant(name)
    o, g, _ = _pair(case)
    ny = case.params.nyc
    iy = [2, ny // 2 - 1, ny // 2] if case.params.flow_type == cases.FT_CH else [2, ny // 2, ny]
    g.spectra2d_setup(iy[:1])  # then grown to the full row list
    g.spectra2d_setup(iy)
    acc = None
    for _ in range(2):
        o.step()
        fo = o.get_fields()
        g.set_fields(fo["ux"], fo["uy"], fo["uz"], fo["p"], fo["c"])
        r = o.spectra2d(iy)
        acc = r if acc is None else acc + r
        g.spectra2d_accumulate()
    got, ns = g.spectra2d_get()
    assert ns == 2 and got.shape == acc.shape
    for m in range(acc.shape[0]):
        e = np.abs(got[m] - acc[m]).max() / max(np.abs(acc[m]).max(), 1e-300)
        assert e <= 1e-12, "%s 2-D spectrum %d rel err %.3e" % (name, m + 1, e)
    bad = [1] if case.params.flow_type == cases.FT_HC else [ny // 2 + 1]
    with pytest.raises(Exception):
        g.spectra2d_setup(bad)
    g.spectra2d_reset()
    got, ns = g.spectra2d_get()
    assert ns == 0 and not got.any()


def _visu_names(p):
    return ["ux", "uy", "uz", "pr", "wx", "wy", "wz", "wMag", "Q", "lamda2"] + (["scalar"] if p.scalar_on else [])


@pytest.mark.parametrize("name", ["channel", "halfchannel_scalar", "channel_odd"])
def test_visu_quantities(name):
    """dump_visu's quantities on identical fields: the finite-difference ones
    within 1e-13 of their largest magnitude, lambda2 (closed-form cubic with
    CUDA's pow/acos/cos against the host's) within 1e-10; every skip pattern
    keeps the points 1, 1+skip, ..."""
    from paratc_b200.abi import VISU
    case = variant(name)
    o, g, _ = _pair(case)
    o.step()
    fo = o.get_fields()
    g.set_fields(fo["ux"], fo["uy"], fo["uz"], fo["p"], fo["c"])
    for n in _visu_names(case.params):
        for node in ((False, True) if n in ("ux", "uy", "uz") else (False,)):
            for skip in ((1, 1, 1), (2, 3, 2)):
                ref = o.visu(VISU[n], skip=skip, node=node)
                got = g.visu_quantity(n, skip=skip, node=node)
                assert got.shape == ref.shape
                tol = 1e-10 if n == "lamda2" else 1e-13
                e = np.abs(got - ref).max() / max(np.abs(ref).max(), 1e-300)
                assert e <= tol, "%s %s node=%s skip=%s rel err %.3e" % (name, n, node, skip, e)


def test_dump_visu_files():
    """paratc_dump_visu writes VisuFor<RunName>_<name>_<ntime> as raw
    Fortran-order REAL(8) (or REAL(4)) arrays of the kept points."""
    from paratc_b200.lib import visu_mask
    case = variant("halfchannel_scalar")
    o, g, _ = _pair(case)
    g.iterate(1)
    mask = visu_mask("ux", "uy", "pr", "wMag", "Q", "lamda2", "scalar")
    with tempfile.TemporaryDirectory() as d:
        for single in (False, True):
            g.dump_visu(d + "/", "Case", 7, mask, skip=(2, 1, 3), single=single)
            for n in ("ux", "uy", "pr", "wMag", "Q", "lamda2", "scalar"):
                ref = g.visu_quantity(n, skip=(2, 1, 3))
                path = os.path.join(d, "VisuForCase_%s_%010d" % (n, 7))
                got = np.fromfile(path, dtype=np.float32 if single else np.float64).reshape(ref.shape)
                if single:
                    assert np.array_equal(got, ref.astype(np.float32)), n
                else:
                    assert np.array_equal(got, ref), n
            assert not os.path.exists(os.path.join(d, "VisuForCase_wx_%010d" % 7))
