"""Pins of the CPU oracle (no GPU).

The reference ships no tests or golden vectors and cannot run here, so the
oracle is pinned by: numpy's FFT (FFTW's documented R2HC/HC2R convention),
scipy's banded solver (the Thomas sweeps), an independent numpy restatement
of the stencils, and discrete identities of the scheme.
"""
import numpy as np
import pytest
import scipy.linalg

from oracle import np_restate
from oracle import oracle_lib as ol
from paratc_b200 import cases

from .helpers import VARIANTS, discrete_poiseuille, fields_of, rel_err, variant, yp_of


@pytest.mark.parametrize("n", [4, 6, 8, 12, 30, 48, 96, 128, 160, 192, 250, 768])
def test_r2hc_matches_numpy(n):
    x = np.random.default_rng(n).standard_normal(n)
    X = np.fft.rfft(x)
    ref = np.zeros(n)
    ref[: n // 2 + 1] = X.real
    for k in range(1, (n + 1) // 2):
        ref[n - k] = X[k].imag
    hc = ol.r2hc(x)
    assert rel_err(hc, ref) < 1e-14
    assert rel_err(ol.hc2r(hc) / n, x) < 1e-14


def _padded(o, name):
    h = o.get_halo(name)  # (nz+4, ny+2, nx+4)
    return h[2:-2, :, 2:-2].copy()


def _metric(o):
    names = ["yp", "dyp", "rdyp", "rdyc", "YinterpCoe", "ap2c", "ac2c", "am2c", "ap2p", "ac2p", "am2p", "ap2cSc",
             "ac2cSc", "am2cSc"]
    return {n: o.metric(n) for n in names}


@pytest.mark.parametrize("name", VARIANTS)
def test_rhs_matches_numpy_restatement(name):
    case = variant(name)
    p = case.params
    yp = yp_of(case)
    o = ol.Oracle(p, yp, threads=2)
    f = fields_of(case, yp)
    o.set_fields(f["ux"], f["uy"], f["uz"], f["p"], f["c"])
    dt = p.dt_max
    o.substep(1, dt)  # histories non-zero
    st = {n: _padded(o, n) for n in (["ux", "uy", "uz", "p"] + (["c"] if p.scalar_on else []))}
    fo = o.get_fields()
    hist = {n: fo[n] for n in ("hx", "hy", "hz", "hc") if fo[n] is not None}
    ns = 2 if p.ischeme != 1 else 1
    o.substep(ns, dt, stop_stage=1)
    sim, dtt, pga = o.get_time()
    g = [8 / 15, 5 / 12, 3 / 4] if p.ischeme == 3 else ([0.5, 1.0, 0] if p.ischeme == 2 else [1.5, 0, 0])
    th = [0, -17 / 60, -5 / 12] if p.ischeme == 3 else ([0, -0.5, 0] if p.ischeme == 2 else [-0.5, 0, 0])
    al = g[ns - 1] + th[ns - 1]
    coef = dict(pmGamma=g[ns - 1] * dt, pmTheta=th[ns - 1] * dt, pmAlpha=al * dt, pmBeta=0.5 * al * p.xnu * dt,
                pmBetaSc=0.5 * al * p.sdiff * dt)
    out, newh, s3 = np_restate.rhs(p, _metric(o), coef, st, hist)
    # flow-rate constraint (src/m_TScheme.f90:269-300)
    if p.is_ux_const:
        if p.scalar_on:
            dpm = p.ubulk - p.ucrf - s3 / (p.nxc * p.nzc) / p.yly
            out["rhsx"] = out["rhsx"] + al * dpm
        else:
            dpm = p.xnu * s3 / (p.nxc * p.nzc) / p.yly
            out["rhsx"] = out["rhsx"] - al * dt * dpm
    for n in out:
        assert rel_err(o.get_work(n), out[n]) < 1e-12, n
    fo = o.get_fields()
    for n in newh:
        assert rel_err(fo[n], newh[n]) < 1e-12, n


@pytest.mark.parametrize("name", ["channel", "halfchannel_scalar", "channel_scalar_crf"])
def test_helmholtz_matches_banded_solver(name):
    case = variant(name)
    p = case.params
    yp = yp_of(case)
    o = ol.Oracle(p, yp, threads=2)
    f = fields_of(case, yp)
    o.set_fields(f["ux"], f["uy"], f["uz"], f["p"], f["c"])
    dt = p.dt_max
    o.substep(1, dt, stop_stage=1)
    rhs = {n: o.get_work(n) for n in ("rhsx", "rhsy", "rhsz", "rhsc") if n != "rhsc" or p.scalar_on}
    before = o.get_fields()
    beta = 0.5 * (8 / 15) * p.xnu * dt
    o2 = ol.Oracle(p, yp, threads=2)
    o2.set_fields(f["ux"], f["uy"], f["uz"], f["p"], f["c"])
    o2.substep(1, dt, stop_stage=2)
    after = o2.get_fields()
    ny = p.nyc

    def solve(am, ac, ap, rows):
        ab = np.zeros((3, ny))
        ab[0, 1:] = ap[:-1]
        ab[1, :] = ac
        ab[2, :-1] = am[1:]
        return scipy.linalg.solve_banded((1, 1), ab, rows)

    for comp, (u, r) in {"x": ("ux", "rhsx"), "z": ("uz", "rhsz")}.items():
        am = -beta * o.metric("am2cForCN")
        ap = -beta * o.metric("ap2cForCN")
        ac = -beta * o.metric("ac2cForCN") + 1.0
        rows = rhs[r].transpose(1, 0, 2).reshape(ny, -1)
        du = solve(am, ac, ap, rows).reshape(ny, p.nzc, p.nxc).transpose(1, 0, 2)
        assert rel_err(after[u] - before[u], du) < 1e-11, comp
    am = -beta * o.metric("am2p")
    ap = -beta * o.metric("ap2p")
    ac = -beta * o.metric("ac2p") + 1.0
    am[0], ac[0], ap[0] = 0.0, 1.0, 0.0
    rows = rhs["rhsy"].transpose(1, 0, 2).reshape(ny, -1).copy()
    rows[0] = 0.0
    dv = solve(am, ac, ap, rows).reshape(ny, p.nzc, p.nxc).transpose(1, 0, 2)
    assert rel_err(after["uy"][:, 1:] - before["uy"][:, 1:], dv[:, 1:]) < 1e-11
    if p.scalar_on:
        bs = 0.5 * (8 / 15) * p.sdiff * dt
        am = -bs * o.metric("am2cScCN")
        ap = -bs * o.metric("ap2cScCN")
        ac = -bs * o.metric("ac2cScCN") + 1.0
        rows = rhs["rhsc"].transpose(1, 0, 2).reshape(ny, -1)
        dc = solve(am, ac, ap, rows).reshape(ny, p.nzc, p.nxc).transpose(1, 0, 2)
        assert rel_err(after["c"] - before["c"], dc) < 1e-11


def test_poisson_manufactured_oracle():
    case = cases.small_channel(32, 24, 24)
    p = case.params
    yp = yp_of(case)
    o = ol.Oracle(p, yp, threads=2)
    nx, nz = p.nxc, p.nzc
    x = np.arange(nx) * p.xlx / nx
    z = np.arange(nz) * p.zlz / nz
    yc = cases.cell_centres_y(yp)
    gy = np.cos(np.pi * yc / p.yly) + 0.3 * yc
    phi = np.cos(2 * np.pi * 3 * x / p.xlx)[None, None, :] * np.cos(2 * np.pi * 2 * z / p.zlz)[:, None, None] * gy[None, :, None]
    wx = o.metric("WaveNumX")[3]
    wz = o.metric("WaveNumZ")[2]
    am, ac, ap = o.metric("am2ph"), o.metric("ac2ph"), o.metric("ap2ph")
    Ly = np.diag(ac) + np.diag(am[1:], -1) + np.diag(ap[:-1], 1)
    src = np.einsum("ij,kjl->kil", Ly, phi) + (wx + wz) * phi
    assert rel_err(o.poisson(src), phi) < 1e-12


def test_wavenumber_is_symbol_of_d4_squared():
    """lambda(w) = (1/dx^2)/288 (cos3w - 54cos2w + 783cosw - 730) is the symbol
    of D4 o D4 with D4 = (1/24, -9/8, 9/8, -1/24)/dx, so the discrete Poisson
    operator is div o grad and the projected field is divergence free."""
    case = cases.small_channel(32, 12, 24)
    p = case.params
    o = ol.Oracle(p, yp_of(case))
    dx = p.xlx / p.nxc
    w = 2 * np.pi * np.arange(p.nxc) / p.nxc
    d4 = np.array([1 / 24, -9 / 8, 9 / 8, -1 / 24]) / dx
    # D4 maps cell values to faces: symbol of D4(f)(i+1/2) = sum_m c_m e^{i w (m - 1/2)} with offsets -1,0,1,2
    offs = np.array([-1, 0, 1, 2]) - 0.5
    sym = np.array([np.sum(d4 * np.exp(1j * ww * offs)) for ww in w])
    lam = (sym * np.conj(sym)).real * -1.0
    assert rel_err(o.metric("WaveNumX"), lam) < 1e-13


def test_projection_divergence_oracle():
    case = cases.small_channel(32, 24, 16)
    yp = yp_of(case)
    o = ol.Oracle(case.params, yp, threads=2)
    f = cases.initial_fields(case, yp)
    o.set_fields(f["ux"], f["uy"], f["uz"], f["p"])
    assert o.diagnostics().divmax > 1.0
    assert o.project() < 1e-12
    st = {n: _padded(o, n) for n in ("ux", "uy", "uz")}
    assert np.abs(np_restate.divergence(case.params, _metric(o), st)).max() < 1e-12


def test_poiseuille_is_fixed_point_oracle():
    case = cases.small_channel(16, 24, 16)
    p = case.params
    yp = yp_of(case)
    o = ol.Oracle(p, yp, threads=2)
    u = discrete_poiseuille(o, p)
    shape = (p.nzc, p.nyc, p.nxc)
    ux = np.broadcast_to(u[None, :, None], shape).copy()
    z = np.zeros(shape)
    o.set_fields(ux, z, z, z)
    for _ in range(3):
        rc, d = o.step()
        assert rc == 0
    fo = o.get_fields()
    assert np.abs(fo["ux"] - ux).max() < 1e-12
    assert np.abs(fo["uy"]).max() < 1e-14 and np.abs(fo["uz"]).max() < 1e-14


def test_oracle_thread_count_invariance():
    case = variant("halfchannel_scalar")
    yp = yp_of(case)
    f = fields_of(case, yp)
    outs = []
    for t in (1, 3):
        ol.set_threads(t)
        o = ol.Oracle(case.params, yp)
        o.set_fields(f["ux"], f["uy"], f["uz"], f["p"], f["c"])
        o.step()
        outs.append(o.get_fields())
    ol.set_threads(0)
    for n in ("ux", "uy", "uz", "p", "c"):
        assert np.array_equal(outs[0][n], outs[1][n]), n


def test_stats_moments_pinned_by_numpy():
    """clcStat (src/m_FlowCase.f90:298-384) restated in the oracle: the point
    moments 1-8, 16, 19-23 are plain x-z means of the staggered values and are
    recomputed here from the fields; the rest follow the same expressions."""
    case = variant("channel")
    yp = yp_of(case)
    o = ol.Oracle(case.params, yp)
    f = fields_of(case, yp)
    o.set_fields(f["ux"], f["uy"], f["uz"], f["p"], f["c"])
    o.step()
    s = o.stats()
    g = o.get_fields()
    ux = g["ux"] + case.params.ucrf
    uy, uz, p = g["uy"], g["uz"], g["p"]
    checks = {0: ux, 1: uy, 2: uz, 3: p, 4: ux * ux, 5: uy * uy, 6: uz * uz, 7: p * p, 15: uy ** 3,
              18: ux ** 3, 19: uz ** 3, 20: ux ** 4, 21: uy ** 4, 22: uz ** 4}
    ny = case.params.nyc
    for q, a in checks.items():
        ref = a.mean(axis=(0, 2))  # fields are [z, y, x]
        scale = np.abs(a).mean(axis=(0, 2)).max()  # the v mean is zero up to rounding
        err = np.abs(s[:ny, q] - ref).max() / scale
        assert err < 1e-13, (q, err)
    # the top wall row carries only moments 27, 33 and 35
    assert np.count_nonzero(s[ny][[q for q in range(35) if q not in (26, 32, 34)]]) == 0


def numpy_spectra(params, g, jlcs):
    """clcStat's 1-D spectra (src/m_FlowCase.f90:430-806, :954-1180) in
    complex form with numpy's real FFT: E = w |X|^2 and the cospectra
    w Re(X conj Y) with w = 2 except at the mean and last mode, LCS =
    X conj(X_ref) (imaginary part zero at the end modes), all summed over the
    other homogeneous direction and times 1/(n_dir^2 n_other).  g: interior
    fields [z, y, x]."""
    p = params
    nx, ny, nz = p.nxc, p.nyc, p.nzc
    ux = g["ux"] + p.ucrf
    uy = g["uy"]
    top = p.uy_bc[3] if p.flow_type == cases.FT_CH else 0.0
    uyn = np.concatenate([uy, np.full((nz, 1, nx), top)], axis=1)
    uyc = 0.5 * (uyn[:, :-1] + uyn[:, 1:])
    ic = (-1 / 16, 9 / 16, 9 / 16, -1 / 16)
    u0 = g["ux"]
    uxc = ic[0] * np.roll(u0, 1, 2) + ic[1] * u0 + ic[2] * np.roll(u0, -1, 2) + ic[3] * np.roll(u0, -2, 2) + p.ucrf
    jr = np.array([jlcs if (p.flow_type == cases.FT_HC or jc <= ny // 2) else ny + 1 - jlcs
                   for jc in range(1, ny + 1)]) - 1
    fields = [ux, uy, g["uz"], g["p"]] + ([g["c"]] if p.scalar_on else [])
    out = []
    for axis, n, other in ((2, nx, nz), (0, nz, nx)):
        nh = n // 2
        w = np.full(nh + 1, 2.0)
        w[0] = w[nh] = 1.0
        norm = 1.0 / (n * n * other)
        sum_ax = 0 if axis == 2 else 1  # the other homogeneous direction

        def hat(a):
            # x: [z, y, kx]; z: [y, x, kz]
            return np.moveaxis(np.fft.rfft(a, axis=axis), axis, 2)

        def rsum(a):
            return a.sum(axis=sum_ax) * norm  # [y, k]

        X = hat(ux)
        Y = hat(uyc)
        spec = [rsum(w * np.abs(hat(f)) ** 2) for f in fields[:4]]
        spec.append(rsum(w * (X * np.conj(Y)).real))
        spec.append(rsum(w * (hat(uxc) * np.conj(Y)).real))
        lcs = X * np.conj(X[:, jr] if axis == 2 else X[jr])
        li = lcs.imag.copy()
        li[..., 0] = 0.0
        li[..., nh] = 0.0
        spec.append(rsum(lcs.real))
        spec.append(rsum(li))
        if p.scalar_on:
            spec.append(rsum(w * np.abs(hat(fields[4])) ** 2))
        out.append(np.stack(spec))
    return out


@pytest.mark.parametrize("name", ["channel", "halfchannel_scalar", "channel_scalar_crf", "channel_odd"])
def test_spectra_pinned_by_numpy(name):
    """The oracle's halfcomplex restatement of the 1-D energy spectra,
    cospectra and linear coherence spectra against numpy's complex FFT."""
    case = variant(name)
    yp = yp_of(case)
    o = ol.Oracle(case.params, yp)
    f = fields_of(case, yp)
    o.set_fields(f["ux"], f["uy"], f["uz"], f["p"], f["c"])
    o.step()
    jlcs = max(1, case.params.nyc // 5)
    ex, ez = o.spectra(jlcs)
    rx, rz = numpy_spectra(case.params, o.get_fields(), jlcs)
    for got, ref in ((ex, rx), (ez, rz)):
        assert got.shape == ref.shape
        for m in range(got.shape[0]):
            err = np.abs(got[m] - ref[m]).max() / max(np.abs(ref[m]).max(), 1e-300)
            assert err < 1e-12, (name, m, err)


def _hc(a, axis):
    """FFTW's R2HC along an axis with numpy: r_0..r_{n/2}, then i_k at n-k."""
    n = a.shape[axis]
    X = np.moveaxis(np.fft.rfft(a, axis=axis), axis, -1)
    out = np.zeros(X.shape[:-1] + (n,))
    out[..., : n // 2 + 1] = X.real
    for k in range(1, (n + 1) // 2):
        out[..., n - k] = X[..., k].imag
    return np.moveaxis(out, -1, axis)


def numpy_spectra2d(params, g, iy):
    """clcEnergySpectra2D / clcCosSpectra2D (src/m_FlowCase.f90:1186-1375)
    with numpy: R2HC along x then along z, squares at the rows iy (plus the
    mirrored row in a channel, the cospectrum subtracting it)."""
    p = params
    nx, ny, nz = p.nxc, p.nyc, p.nzc
    top = p.uy_bc[3] if p.flow_type == cases.FT_CH else 0.0
    uyn = np.concatenate([g["uy"], np.full((nz, 1, nx), top)], axis=1)
    uyc = 0.5 * (uyn[:, :-1] + uyn[:, 1:])
    ic = (-1 / 16, 9 / 16, 9 / 16, -1 / 16)
    u0 = g["ux"]
    uxc = ic[0] * np.roll(u0, 1, 2) + ic[1] * u0 + ic[2] * np.roll(u0, -1, 2) + ic[3] * np.roll(u0, -2, 2) + p.ucrf
    norm = (1.0 / (nx * nz)) ** 2 * (0.5 if p.flow_type == cases.FT_CH else 1.0)
    hc = p.flow_type == cases.FT_HC

    def H(a, j):  # j: 1-based row; a [z, y, x] (uy may carry the wall row)
        return _hc(_hc(a[:, j - 1, :], 1), 0)  # [z-hc, x-hc]

    out = []
    fields = [g["ux"], uyn, g["uz"], g["p"]] + ([g["c"]] if p.scalar_on else [])
    for m in range(6 if p.scalar_on else 5):
        planes = []
        for j in iy:
            if m == 4:
                v = H(uxc, j) * H(uyc, j)
                if not hc:
                    v = v - H(uxc, ny + 1 - j) * H(uyc, ny + 1 - j)
            else:
                a = fields[m if m < 4 else 4]
                js = (ny + 2 - j) if m == 1 else (ny + 1 - j)
                v = H(a, j) ** 2 + (0 if hc else H(a, js) ** 2)
            planes.append(norm * v)
        out.append(np.stack(planes, axis=1))  # [z, q, x]
    return np.stack(out)


@pytest.mark.parametrize("name", ["channel", "halfchannel_scalar", "channel_odd"])
def test_spectra2d_pinned_by_numpy(name):
    case = variant(name)
    yp = yp_of(case)
    o = ol.Oracle(case.params, yp)
    f = fields_of(case, yp)
    o.set_fields(f["ux"], f["uy"], f["uz"], f["p"], f["c"])
    o.step()
    ny = case.params.nyc
    iy = [2, ny // 2 - 1, ny // 2] if case.params.flow_type == cases.FT_CH else [2, ny // 2, ny]
    got = o.spectra2d(iy)
    ref = numpy_spectra2d(case.params, o.get_fields(), iy)
    assert got.shape == ref.shape
    for m in range(ref.shape[0]):
        err = np.abs(got[m] - ref[m]).max() / np.abs(ref[m]).max()
        assert err < 1e-12, (name, m, err)
    with pytest.raises(RuntimeError):
        o.spectra2d([1])


def numpy_visu(params, o, g, name, node=False):
    """dump_visu's quantities (src/m_IOAndVisu.f90:182-385, Clc_Q_vor and
    Clc_lamda2 of src/m_Tools.f90) with numpy on the halo'd fields; lambda2
    as the middle eigenvalue of the symmetric tensor by numpy's eigvalsh
    instead of the reference's closed-form cubic."""
    p = params
    H = {n: o.get_halo(n) for n in ("ux", "uy", "uz")}  # [z+4, y+2, x+4], interior at [2:-2, 1:-1, 2:-2]
    nz, ny, nx = p.nzc, p.nyc, p.nxc

    def sh(a, di=0, dj=0, dk=0):
        return a[2 + dk:2 + dk + nz, 1 + dj:1 + dj + ny, 2 + di:2 + di + nx]

    ux, uy, uz = H["ux"], H["uy"], H["uz"]
    if name == "ux":
        return sh(ux) + p.ucrf if node else 0.5 * (sh(ux, 1) + sh(ux)) + p.ucrf
    if name == "uy":
        return sh(uy) if node else 0.5 * (sh(uy, 0, 1) + sh(uy))
    if name == "uz":
        return sh(uz) if node else 0.5 * (sh(uz, 0, 0, 1) + sh(uz))
    if name == "pr":
        return g["p"]
    if name == "scalar":
        return g["c"]
    rdx, rdz = p.nxc / p.xlx, p.nzc / p.zlz
    rdyc = o.metric("rdyc")  # rdyc(1..nyp)
    rdyp = o.metric("rdyp")  # rdyp(0..nyp)
    c1 = rdyc[0:ny][None, :, None]
    c2 = rdyc[1:ny + 1][None, :, None]
    c12 = c1 - c2
    q4 = 0.25
    dudx = (sh(ux, 1) - sh(ux)) * rdx
    dudy = ((sh(ux, 1, 1) + sh(ux, 0, 1)) * c2 + (sh(ux, 1) + sh(ux)) * c12 - (sh(ux, 1, -1) + sh(ux, 0, -1)) * c1) * q4
    dudz = (sh(ux, 1, 0, 1) + sh(ux, 0, 0, 1) - sh(ux, 1, 0, -1) - sh(ux, 0, 0, -1)) * rdz * q4
    dvdx = (sh(uy, 1, 1) - sh(uy, -1, 1) + sh(uy, 1) - sh(uy, -1)) * rdx * q4
    dvdy = (sh(uy, 0, 1) - sh(uy)) * rdyp[1:ny + 1][None, :, None]
    dvdz = (sh(uy, 0, 1, 1) + sh(uy, 0, 0, 1) - sh(uy, 0, 1, -1) - sh(uy, 0, 0, -1)) * rdz * q4
    dwdx = (sh(uz, 1, 0, 1) - sh(uz, -1, 0, 1) + sh(uz, 1) - sh(uz, -1)) * rdx * q4
    dwdy = ((sh(uz, 0, 1, 1) + sh(uz, 0, 1)) * c2 + (sh(uz, 0, 0, 1) + sh(uz)) * c12 - (sh(uz, 0, -1, 1) + sh(uz, 0, -1)) * c1) * q4
    dwdz = (sh(uz, 0, 0, 1) - sh(uz)) * rdz
    wx, wy, wz = dwdy - dvdz, dudz - dwdx, dvdx - dudy
    if name == "wx":
        return wx
    if name == "wy":
        return wy
    if name == "wz":
        return wz
    if name == "wMag":
        return np.sqrt(wx * wx + wy * wy + wz * wz)
    G = np.stack([np.stack([dudx, dudy, dudz], -1), np.stack([dvdx, dvdy, dvdz], -1),
                  np.stack([dwdx, dwdy, dwdz], -1)], -2)  # G[..., i, j] = du_i/dx_j
    if name == "Q":
        return 0.5 * (np.trace(G, axis1=-2, axis2=-1) ** 2 - np.einsum("...ij,...ji->...", G, G))
    S = 0.5 * (G + np.swapaxes(G, -1, -2))
    W = 0.5 * (G - np.swapaxes(G, -1, -2))
    return np.linalg.eigvalsh(S @ S + W @ W)[..., 1]


@pytest.mark.parametrize("name", ["channel", "halfchannel_scalar"])
def test_visu_pinned_by_numpy(name):
    """The oracle's dump_visu quantities against numpy (Q as the invariant
    (tr(G)^2 - tr(G G))/2, lambda2 by eigvalsh), all points and a skipped
    sampling."""
    case = variant(name)
    yp = yp_of(case)
    o = ol.Oracle(case.params, yp)
    f = fields_of(case, yp)
    o.set_fields(f["ux"], f["uy"], f["uz"], f["p"], f["c"])
    o.step()
    g = o.get_fields()
    names = ["ux", "uy", "uz", "pr", "wx", "wy", "wz", "wMag", "Q", "lamda2"] + (["scalar"] if case.params.scalar_on else [])
    from paratc_b200.abi import VISU
    for n in names:
        for node in ((False, True) if n in ("ux", "uy", "uz") else (False,)):
            ref = numpy_visu(case.params, o, g, n, node)
            got = o.visu(VISU[n], node=node)
            tol = 1e-10 if n == "lamda2" else 1e-13
            err = np.abs(got - ref).max() / np.abs(ref).max()
            assert err < tol, (name, n, node, err)
            sk = o.visu(VISU[n], skip=(3, 2, 5), node=node)
            assert np.array_equal(sk, got[::5, ::2, ::3]), (n, "skip")
