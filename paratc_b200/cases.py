"""Workload definitions and seeded initial fields.

Each case is a ParaTC input in the terms of its namelists (&BasicParam,
&MeshOptions, &ScalarFlowOptions; src/m_Parameters.f90:118-130,
src/m_MeshAndMetries.f90:77-80) with the derivations of ReadAndInitParameters
applied (src/m_Parameters.f90:144-187).  The initial fields replace
InitVelocity (src/m_FlowCase.f90:49-107), which seeds from system_clock and is
therefore not reproducible: here every field is drawn from a seeded numpy
PCG64 generator in Fortran order (x fastest).

Arrays are numpy float64 of shape (nzc, nyc, nxc).
"""
import math
from dataclasses import dataclass, field
from typing import List

import numpy as np

from .abi import FT_CH, FT_HC, RK3, ParatcParams


@dataclass
class Mesh:
    """&MeshSection / &MeshOptions."""

    section_length: List[float]
    section_cstret: List[float]
    nyc_section: List[int]
    stret_type: List[int]
    stret_option: List[int]


@dataclass
class Case:
    name: str
    params: ParatcParams
    mesh: Mesh
    init: str = "channel"          # "channel" | "lock" | "linear_c" | "gauss_src"
    seed: int = 1234
    noise: float = 0.3
    extra: dict = field(default_factory=dict)

    @property
    def n_cells(self):
        p = self.params
        return p.nxc * p.nyc * p.nzc


def retau_to_xnu(retau, ubulk=1.0, height=1.0):
    """Inverts retau = 0.1538*Re_b**0.887741, Re_b = ubulk*height/xnu
    (src/m_FlowCase.f90:63-64)."""
    rem = (retau / 0.1538) ** (1.0 / 0.887741)
    return ubulk * height / rem


def make_params(nxc, nyc, nzc, *, flow_type=FT_CH, xlx=4 * math.pi, yly=2.0, zlz=4 * math.pi / 3,
                xnu=2.0 * (2.0 / 3.0) / 5600.0, ubulk=2.0 / 3.0, dt_max=0.005, icfl=2, cflc=1.5,
                ischeme=RK3, is_ux_const=1, gravity=(0.0, 0.0, 0.0), scalar=None,
                vel_limit=1.0e9, div_limit=1.0e9, ucrf=0.0):
    """Builds a ParatcParams the way ReadAndInitParameters leaves m_Parameters.

    scalar: None or dict(schmidt, gravity_eff, gravity_dir, falling_vel,
    bc_option=(b,t), bc_values=(F_b,F_t,S_b,S_t), init_value)."""
    p = ParatcParams()
    p.nxc, p.nyc, p.nzc = nxc, nyc, nzc
    p.flow_type, p.ischeme, p.icfl = flow_type, ischeme, icfl
    p.is_ux_const = int(is_ux_const)
    p.xlx, p.yly, p.zlz = xlx, yly, zlz
    p.xnu, p.ubulk, p.ucrf = xnu, ubulk, ucrf
    p.dt_max, p.cflc = dt_max, cflc
    for i in range(3):
        p.gravity[i] = gravity[i]
    for i in range(6):
        p.ux_bc[i] = 0.0 - ucrf
        p.uy_bc[i] = 0.0
        p.uz_bc[i] = 0.0
    p.vel_limit, p.div_limit = vel_limit, div_limit
    p.scalar_on = 0
    if scalar is not None:
        p.scalar_on = 1
        gd = np.asarray(scalar.get("gravity_dir", (0.0, -1.0, 0.0)), dtype=np.float64)
        nrm = math.sqrt(gd[0] * gd[0] + gd[1] * gd[1] + gd[2] * gd[2])
        gd = gd / nrm if nrm > 1.0e-10 else np.array([0.0, -1.0, 0.0])
        p.sdiff = xnu / scalar.get("schmidt", 1.0)
        ge = scalar.get("gravity_eff", 1.0)
        fv = scalar.get("falling_vel", 0.0)
        for i in range(3):
            p.gravity_eff_vec[i] = gd[i] * ge
            p.falling_vel_vec[i] = gd[i] * fv
        p.falling_vel_vec[0] = p.falling_vel_vec[0] + ucrf
        bo = scalar.get("bc_option", (-2, -2))
        bv = scalar.get("bc_values", (0.0, 0.0, 0.0, 0.0))
        p.scalar_bc_option[0], p.scalar_bc_option[1] = bo
        for i in range(4):
            p.scalar_bc_values[i] = bv[i]
        p.scalar_init_value = scalar.get("init_value", 0.0)
    return p


def tanh_mesh(nyc, cstret=1.5, two_sided=True):
    if two_sided:
        h = nyc // 2
        return Mesh([1.0, 1.0], [cstret, cstret], [h, nyc - h], [1, 1], [0, 1])
    return Mesh([1.0], [cstret], [nyc], [1], [0])


# ---------------------------------------------------------------------------
# the five workloads
# ---------------------------------------------------------------------------

def channel_c1(nxc=128, nyc=96, nzc=128):
    """Closed turbulent channel, Re_b = 5600 (Re_tau ~ 180), 4pi x 2 x 4pi/3,
    tanh-stretched y (two sections, stretch 1.5), RK3, dt = 0.005 fixed,
    constant flow rate, no scalar."""
    p = make_params(nxc, nyc, nzc)
    return Case("channel_c1_%dx%dx%d" % (nxc, nyc, nzc), p, tanh_mesh(nyc), "channel", 1234, 0.3)


def poisson_c2(nxc=512, nyc=256, nzc=512):
    """Standalone pressure Poisson solve, stretched y with Neumann walls,
    periodic x/z, RHS = N(0,1) with seed 42 and the mean removed."""
    p = make_params(nxc, nyc, nzc)
    return Case("poisson_c2_%dx%dx%d" % (nxc, nyc, nzc), p, tanh_mesh(nyc), "gauss_src", 42, 1.0)


def lock_exchange_c3(nxc=1536, nyc=160, nzc=256):
    """Lock-exchange gravity current: 48 x 1 x 4, half channel (no-slip bottom,
    free-slip top), Re = 5000, Sc = 1, settling 0.02, g_eff = 1 along -y;
    scalar: bottom Robin with F = w_s/K (no net flux), top zero-flux Neumann;
    c = 1 for x < 1 else 0 plus U(-1e-3, 1e-3) noise (seed 7); u = 0."""
    xnu = 1.0 / 5000.0
    ws = 0.02
    sc = dict(schmidt=1.0, gravity_eff=1.0, gravity_dir=(0.0, -1.0, 0.0), falling_vel=ws,
              bc_option=(-3, -2), bc_values=(ws / xnu, 0.0, 0.0, 0.0), init_value=1.0)
    p = make_params(nxc, nyc, nzc, flow_type=FT_HC, xlx=48.0, yly=1.0, zlz=4.0, xnu=xnu, ubulk=0.0,
                    dt_max=0.005, icfl=1, cflc=0.8, is_ux_const=0, scalar=sc)
    return Case("lock_exchange_c3_%dx%dx%d" % (nxc, nyc, nzc), p, tanh_mesh(nyc, 1.5, False), "lock", 7, 1e-3)


def turbidity_c5(nxc=2304, nyc=192, nzc=768):
    """Turbidity-current channel, half channel 4pi x 1 x 4pi/3 (the domain of
    Input/GravityFlow/GravityFlow.prm), Re_tau = 550, Sc = 1, w_s = 0.01,
    bottom Robin with F = w_s/K (erosion-free, no net flux), top zero flux,
    constant flow rate, c linear in y plus 1e-3 noise (seed 11)."""
    xnu = retau_to_xnu(550.0, 1.0, 1.0)
    ws = 0.01
    sc = dict(schmidt=1.0, gravity_eff=1.0, gravity_dir=(0.0, -1.0, 0.0), falling_vel=ws,
              bc_option=(-3, -2), bc_values=(ws / xnu, 0.0, 0.0, 0.0), init_value=1.0)
    p = make_params(nxc, nyc, nzc, flow_type=FT_HC, xlx=4 * math.pi, yly=1.0, zlz=4 * math.pi / 3,
                    xnu=xnu, ubulk=1.0, dt_max=0.002, icfl=1, cflc=1.0, is_ux_const=1, scalar=sc)
    return Case("turbidity_c5_%dx%dx%d" % (nxc, nyc, nzc), p, tanh_mesh(nyc, 1.5, False), "linear_c", 11, 1e-3)


def ensemble_c4(n=32, seed=2024):
    """32 channel instances: (nx, nz) from {64,96,128,192}, ny from
    {48,64,96,128}, Re_tau from U[120, 395] (seed 2024)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    cases = []
    for i in range(n):
        nx = int(rng.choice([64, 96, 128, 192]))
        nz = int(rng.choice([64, 96, 128, 192]))
        ny = int(rng.choice([48, 64, 96, 128]))
        retau = float(rng.uniform(120.0, 395.0))
        xnu = retau_to_xnu(retau, 2.0 / 3.0, 1.0)
        p = make_params(nx, ny, nz, xnu=xnu)
        cases.append(Case("ensemble_%02d_%dx%dx%d" % (i, nx, ny, nz), p, tanh_mesh(ny), "channel", seed + i, 0.3))
    return cases


def small_channel(nxc=16, nyc=12, nzc=16, **kw):
    scalar = kw.pop("scalar", None)
    flow_type = kw.pop("flow_type", FT_CH)
    p = make_params(nxc, nyc, nzc, flow_type=flow_type, scalar=scalar, **kw)
    mesh = tanh_mesh(nyc, 1.5, flow_type == FT_CH)
    return Case("small_%dx%dx%d" % (nxc, nyc, nzc), p, mesh, "channel", 1234, 0.3)


# ---------------------------------------------------------------------------
# initial fields
# ---------------------------------------------------------------------------

def cell_centres_y(yp):
    yp = np.asarray(yp, dtype=np.float64)
    return 0.5 * (yp[:-1] + yp[1:])


def initial_fields(case, yp):
    """Seeded initial state (interior arrays) for a case.

    channel: u = 1.5*U_b*(1 - (y/h - 1)^2) (laminar Poiseuille, h = yly/2 for
    a channel, yly for a half channel) plus U(-a, a)*U_b noise on u, v, w;
    lock / linear_c: u = v = w = 0 (+ noise a on u,v,w for linear_c), scalar
    as documented on the case.  p = 0, histories 0.  The velocity is not yet
    solenoidal: ParaTC's projection (paratc_project) makes it so."""
    p = case.params
    shape = (p.nzc, p.nyc, p.nxc)
    rng = np.random.Generator(np.random.PCG64(case.seed))
    yc = cell_centres_y(yp)
    out = {"ux": np.zeros(shape), "uy": np.zeros(shape), "uz": np.zeros(shape), "p": np.zeros(shape), "c": None}
    if case.init in ("channel", "linear_c"):
        h = p.yly / 2.0 if p.flow_type == FT_CH else p.yly
        ub = p.ubulk
        eta = yc / h - 1.0
        prof = 1.5 * ub * (1.0 - eta * eta)
        out["ux"] = np.broadcast_to(prof[None, :, None], shape).copy()
        amp = case.noise if case.init == "channel" else 0.1
        out["ux"] += rng.uniform(-amp, amp, size=shape) * ub
        out["uy"] += rng.uniform(-amp, amp, size=shape) * ub
        out["uz"] += rng.uniform(-amp, amp, size=shape) * ub
    if p.scalar_on:
        if case.init == "lock":
            dx = p.xlx / p.nxc
            xc = (np.arange(p.nxc) + 0.5) * dx
            c = np.where(xc < 1.0, 1.0, 0.0)
            out["c"] = np.broadcast_to(c[None, None, :], shape).copy()
            out["c"] += rng.uniform(-case.noise, case.noise, size=shape)
        else:
            c = 1.0 - yc / p.yly
            out["c"] = np.broadcast_to(c[None, :, None], shape).copy()
            out["c"] += rng.uniform(-1e-3, 1e-3, size=shape)
    return out


def gaussian_source(case):
    """C2 right-hand side: N(0,1) with the given seed, mean removed exactly
    (compensated sum) so that the singular kx = kz = 0 mode is compatible."""
    p = case.params
    rng = np.random.Generator(np.random.PCG64(case.seed))
    src = rng.standard_normal((p.nzc, p.nyc, p.nxc))
    mean = math.fsum(src.ravel()) / src.size
    src -= mean
    return src
