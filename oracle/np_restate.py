"""Second, independent restatement of clcRhsXYZ / clcPrSrc / FluidVelUpdate /
PressureUpdate in vectorised numpy -- TEST INFRASTRUCTURE.

Written separately from the C oracle (periodic halos as np.roll instead of
halo copies, whole-array expressions instead of loops) so that a
transcription slip in one of the two shows up as a disagreement between
them.  Small grids only.

Fields are padded arrays of shape (nzc, nyc+2, nxc): y index j = 0..nyp as in
the reference (ghost rows 0 and nyp), x and z periodic.
"""
import numpy as np

I1, I2, I3, I4 = -1.0 / 16.0, 9.0 / 16.0, 9.0 / 16.0, -1.0 / 16.0


def _X(F, d):
    """F at x index i+d (periodic)."""
    return np.roll(F, -d, axis=2)


def _Z(F, d):
    """F at z index k+d (periodic)."""
    return np.roll(F, -d, axis=0)


def coefficients(params, metric):
    """4th-order constants of InitMeshAndMetries (src/m_MeshAndMetries.f90:96-101)."""
    rdx = params.nxc / params.xlx
    rdz = params.nzc / params.zlz
    c = {}
    c["dx"] = [rdx / 24.0, -rdx * 1.125, rdx * 1.125, -rdx / 24.0]
    c["dz"] = [rdz / 24.0, -rdz * 1.125, rdz * 1.125, -rdz / 24.0]
    c["dxx"] = [-rdx * rdx / 12.0, 4.0 / 3.0 * rdx * rdx, -2.5 * rdx * rdx, 4.0 / 3.0 * rdx * rdx, -rdx * rdx / 12.0]
    c["dzz"] = [-rdz * rdz / 12.0, 4.0 / 3.0 * rdz * rdz, -2.5 * rdz * rdz, 4.0 / 3.0 * rdz * rdz, -rdz * rdz / 12.0]
    return c


def _col(v, ny):
    """1-D metric over j = 1..ny broadcast to (1, ny, 1)."""
    return np.asarray(v, dtype=np.float64)[:ny].reshape(1, ny, 1)


def rhs(params, metric, coef, st, hist):
    """clcRhsXYZ (src/m_TScheme.f90:113-360) without the flow-rate term.

    metric: dict of 1-D arrays indexed as the oracle exports them (yp from 1,
    dyp/rdyp/yc from 0, the others from 1).  coef: pmGamma, pmTheta, pmAlpha,
    pmBeta, pmBetaSc.  st: padded ux, uy, uz, p (, c).  hist: interior hx, hy,
    hz (, hc).  Returns (rhs dict, new hist dict, s3tot)."""
    ny = params.nyc
    C = coefficients(params, metric)
    dX, dZ, dXX, dZZ = C["dx"], C["dz"], C["dxx"], C["dzz"]
    ux, uy, uz, pr = st["ux"], st["uy"], st["uz"], st["p"]
    uc = params.ucrf
    J, JM, JP = slice(1, ny + 1), slice(0, ny), slice(2, ny + 2)
    rdyp = _col(metric["rdyp"][1:], ny)
    rdyc = _col(metric["rdyc"], ny)
    dyp = _col(metric["dyp"][1:], ny)
    yi = np.asarray(metric["YinterpCoe"])  # j = 1..nyp
    IY1 = _col(yi[0:ny], ny)
    IY2 = 1.0 - IY1
    IY3 = _col(yi[1:ny + 1], ny)
    IY4 = 1.0 - IY3

    uxhx = I1 * _X(ux, -1) + I2 * ux + I3 * _X(ux, 1) + I4 * _X(ux, 2)
    uyhx = I1 * _X(uy, -2) + I2 * _X(uy, -1) + I3 * uy + I4 * _X(uy, 1)
    uzhx = I1 * _X(uz, -2) + I2 * _X(uz, -1) + I3 * uz + I4 * _X(uz, 1)
    uxhz = I1 * _Z(ux, -2) + I2 * _Z(ux, -1) + I3 * ux + I4 * _Z(ux, 1)
    uyhz = I1 * _Z(uy, -2) + I2 * _Z(uy, -1) + I3 * uy + I4 * _Z(uy, 1)
    uzhz = I1 * _Z(uz, -1) + I2 * uz + I3 * _Z(uz, 1) + I4 * _Z(uz, 2)
    uyhx[:, ny + 1, :] = 0.0
    uyhz[:, ny + 1, :] = 0.0

    def d1x(F):  # dxCoe on offsets -2..1
        return dX[0] * _X(F, -2) + dX[1] * _X(F, -1) + dX[2] * F + dX[3] * _X(F, 1)

    def dxx(F):
        return dXX[0] * _X(F, -2) + dXX[1] * _X(F, -1) + dXX[2] * F + dXX[3] * _X(F, 1) + dXX[4] * _X(F, 2)

    def dzz(F):
        return dZZ[0] * _Z(F, -2) + dZZ[1] * _Z(F, -1) + dZZ[2] * F + dZZ[3] * _Z(F, 1) + dZZ[4] * _Z(F, 2)

    g = params.gravity
    xnu = params.xnu
    # --- X
    uxhyc = IY1 * ux[:, JM] + IY2 * ux[:, J]
    uxhyp = IY3 * ux[:, J] + IY4 * ux[:, JP]
    q = uxhx * (uxhx + uc)
    h11 = (dX[0] * _X(q, -2) + dX[1] * _X(q, -1) + dX[2] * q + dX[3] * _X(q, 1))[:, J]
    h12 = (uyhx[:, JP] * uxhyp - uyhx[:, J] * uxhyc) * rdyp
    q = uxhz * uzhx
    h13 = (dZ[0] * _Z(q, -1) + dZ[1] * q + dZ[2] * _Z(q, 1) + dZ[3] * _Z(q, 2))[:, J]
    d11, d33 = dxx(ux)[:, J], dzz(ux)[:, J]
    d22 = _col(metric["ap2c"], ny) * ux[:, JP] + _col(metric["ac2c"], ny) * ux[:, J] + _col(metric["am2c"], ny) * ux[:, JM]
    if params.scalar_on:
        s3 = float(np.sum(ux[:, J] * dyp))
    else:
        s3 = float(np.sum((d11 + d33 + d22) * dyp))
    cx = -h11 - h12 - h13 + xnu * (d11 + d33) + g[0]
    rx = coef["pmGamma"] * cx + coef["pmTheta"] * hist["hx"] - coef["pmAlpha"] * d1x(pr)[:, J] + 2.0 * coef["pmBeta"] * d22
    # --- Y
    uxh = [IY1 * _X(ux, d)[:, JM] + IY2 * _X(ux, d)[:, J] + uc for d in (-1, 0, 1, 2)]
    uzh = [IY1 * _Z(uz, d)[:, JM] + IY2 * _Z(uz, d)[:, J] for d in (-1, 0, 1, 2)]
    h21 = sum(dX[n] * _X(uyhx, d)[:, J] * uxh[n] for n, d in enumerate((-1, 0, 1, 2)))
    vp, vc, vm = uy[:, JP], uy[:, J], uy[:, JM]
    h22 = ((vp + vc) ** 2 - (vc + vm) ** 2) * 0.25 * rdyc
    h23 = sum(dZ[n] * _Z(uyhz, d)[:, J] * uzh[n] for n, d in enumerate((-1, 0, 1, 2)))
    d22 = _col(metric["ap2p"], ny) * vp + _col(metric["ac2p"], ny) * vc + _col(metric["am2p"], ny) * vm
    cy = -h21 - h22 - h23 + xnu * (dxx(uy)[:, J] + dzz(uy)[:, J]) + g[1]
    ry = coef["pmGamma"] * cy + coef["pmTheta"] * hist["hy"] - coef["pmAlpha"] * (pr[:, J] - pr[:, JM]) * rdyc + 2.0 * coef["pmBeta"] * d22
    # --- Z
    uzhyc = IY1 * uz[:, JM] + IY2 * uz[:, J]
    uzhyp = IY3 * uz[:, J] + IY4 * uz[:, JP]
    q = uzhx * (uxhz + uc)
    h31 = (dX[0] * _X(q, -1) + dX[1] * q + dX[2] * _X(q, 1) + dX[3] * _X(q, 2))[:, J]
    h32 = (uyhz[:, JP] * uzhyp - uyhz[:, J] * uzhyc) * rdyp
    q = uzhz * uzhz
    h33 = (dZ[0] * _Z(q, -2) + dZ[1] * _Z(q, -1) + dZ[2] * q + dZ[3] * _Z(q, 1))[:, J]
    d22 = _col(metric["ap2c"], ny) * uz[:, JP] + _col(metric["ac2c"], ny) * uz[:, J] + _col(metric["am2c"], ny) * uz[:, JM]
    cz = -h31 - h32 - h33 + xnu * (dxx(uz)[:, J] + dzz(uz)[:, J]) + g[2]
    gp3 = (dZ[0] * _Z(pr, -2) + dZ[1] * _Z(pr, -1) + dZ[2] * pr + dZ[3] * _Z(pr, 1))[:, J]
    rz = coef["pmGamma"] * cz + coef["pmTheta"] * hist["hz"] - coef["pmAlpha"] * gp3 + 2.0 * coef["pmBeta"] * d22
    out = {"rhsx": rx, "rhsy": ry, "rhsz": rz}
    newh = {"hx": cx, "hy": cy, "hz": cz}
    if params.scalar_on:
        sc = st["c"]
        GE, FV = params.gravity_eff_vec, params.falling_vel_vec
        shx = I1 * _X(sc, -2) + I2 * _X(sc, -1) + I3 * sc + I4 * _X(sc, 1)
        shz = I1 * _Z(sc, -2) + I2 * _Z(sc, -1) + I3 * sc + I4 * _Z(sc, 1)
        shyc = IY1 * sc[:, JM] + IY2 * sc[:, J]
        shyp = IY3 * sc[:, J] + IY4 * sc[:, JP]
        c1, c2, c3 = GE[0] * shx[:, J], GE[1] * shyc, GE[2] * shz[:, J]
        out["rhsx"] = out["rhsx"] + coef["pmGamma"] * c1
        out["rhsy"] = out["rhsy"] + coef["pmGamma"] * c2
        out["rhsz"] = out["rhsz"] + coef["pmGamma"] * c3
        newh["hx"] = cx + c1
        newh["hy"] = cy + c2
        newh["hz"] = cz + c3
        q = (ux + FV[0]) * shx
        hc1 = (dX[0] * _X(q, -1) + dX[1] * q + dX[2] * _X(q, 1) + dX[3] * _X(q, 2))[:, J]
        hc2 = ((uy[:, JP] + FV[1]) * shyp - (uy[:, J] + FV[1]) * shyc) * rdyp
        q = (uz + FV[2]) * shz
        hc3 = (dZ[0] * _Z(q, -1) + dZ[1] * q + dZ[2] * _Z(q, 1) + dZ[3] * _Z(q, 2))[:, J]
        d22 = _col(metric["ap2cSc"], ny) * sc[:, JP] + _col(metric["ac2cSc"], ny) * sc[:, J] + _col(metric["am2cSc"], ny) * sc[:, JM]
        cc = -hc1 - hc2 - hc3 + params.sdiff * (dxx(sc)[:, J] + dzz(sc)[:, J])
        out["rhsc"] = coef["pmGamma"] * cc + coef["pmTheta"] * hist["hc"] + 2.0 * coef["pmBetaSc"] * d22
        newh["hc"] = cc
    return out, newh, s3


def divergence(params, metric, st):
    """dudx + dvdy + dwdz of clcPrSrc / CheckDivergence (src/m_TScheme.f90:60-75)."""
    ny = params.nyc
    C = coefficients(params, metric)
    dX, dZ = C["dx"], C["dz"]
    ux, uy, uz = st["ux"], st["uy"], st["uz"]
    J, JP = slice(1, ny + 1), slice(2, ny + 2)
    dudx = (dX[0] * _X(ux, -1) + dX[1] * ux + dX[2] * _X(ux, 1) + dX[3] * _X(ux, 2))[:, J]
    dvdy = (uy[:, JP] - uy[:, J]) * _col(metric["rdyp"][1:], ny)
    dwdz = (dZ[0] * _Z(uz, -1) + dZ[1] * uz + dZ[2] * _Z(uz, 1) + dZ[3] * _Z(uz, 2))[:, J]
    return dudx + dvdy + dwdz
