"""Shared helpers of the test suite: cases, seeded fields, error norms."""
import numpy as np

from oracle import oracle_lib as ol
from paratc_b200 import cases
from paratc_b200.abi import FT_CH, FT_HC


def rel_err(a, b):
    """max|a - b| / max|b| (max|b| floored at 1e-300)."""
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def yp_of(case):
    m = case.mesh
    return ol.ycoord(m.section_length, m.section_cstret, m.nyc_section, m.stret_type, m.stret_option,
                     case.params.yly)


def scalar_opts(bc=(-3, -2), ws=0.02, ge=1.0, gdir=(0.0, -1.0, 0.0), vals=None, init=0.5):
    return dict(schmidt=1.0, gravity_eff=ge, gravity_dir=gdir, falling_vel=ws, bc_option=bc,
                bc_values=vals if vals is not None else (ws / 1e-3, 0.3, 0.0, 0.1), init_value=init)


def variant(name):
    """Small cases covering the option space of the hot path."""
    if name == "channel":
        return cases.small_channel(32, 24, 16)
    if name == "channel_odd":  # non-power-of-two x/z sizes (radix 3, 5)
        return cases.small_channel(24, 20, 30)
    if name == "channel_cfl":
        c = cases.small_channel(16, 16, 24, icfl=1, cflc=0.5, dt_max=0.02)
        return c
    if name == "channel_ab2":
        return cases.small_channel(16, 12, 16, ischeme=1)
    if name == "channel_rk2":
        return cases.small_channel(16, 12, 16, ischeme=2)
    if name == "halfchannel_scalar":
        c = cases.small_channel(32, 20, 16, flow_type=FT_HC, xnu=1e-3, yly=1.0, is_ux_const=0, icfl=1,
                                cflc=0.6, dt_max=0.01,
                                scalar=scalar_opts((-3, -2), 0.02, 1.0, (0.087, -0.996, 0.0)))
        return c
    if name == "channel_scalar_crf":
        c = cases.small_channel(16, 16, 16, xnu=1e-3, is_ux_const=1, ucrf=0.3,
                                scalar=scalar_opts((-1, -1), 0.0, 0.5, (1.0, 0.0, 0.0), (1.0, 0.2, 0.0, 0.0)))
        return c
    if name == "channel_scalar_neumann":
        c = cases.small_channel(16, 12, 16, xnu=1e-3, is_ux_const=0, gravity=(0.01, 0.0, 0.0),
                                scalar=scalar_opts((-2, -2), 0.01, 0.2, (0.0, -1.0, 0.0), (0.0, 0.0, 0.1, -0.1)))
        return c
    raise KeyError(name)


VARIANTS = ["channel", "channel_odd", "channel_cfl", "channel_ab2", "channel_rk2", "halfchannel_scalar",
            "channel_scalar_crf", "channel_scalar_neumann"]


def fields_of(case, yp):
    f = cases.initial_fields(case, yp)
    if case.params.scalar_on and f["c"] is None:
        rng = np.random.Generator(np.random.PCG64(99))
        f["c"] = 0.5 + 0.1 * rng.uniform(-1, 1, size=f["ux"].shape)
    rng = np.random.Generator(np.random.PCG64(7))
    f["p"] = 0.01 * rng.standard_normal(f["ux"].shape)
    return f


def discrete_poiseuille(o, params):
    """Laminar profile u(y) with L_y u = const for the operator the scheme
    uses (explicit a?2c stencil with the wall ghost u(0) = -u(1), i.e. the
    ForCN coefficients), scaled to the bulk velocity."""
    ny = params.nyc
    am = o.metric("am2cForCN")
    ac = o.metric("ac2cForCN")
    ap = o.metric("ap2cForCN")
    A = np.diag(ac) + np.diag(am[1:], -1) + np.diag(ap[:-1], 1)
    u = np.linalg.solve(A, -np.ones(ny))
    dyp = o.metric("dyp")[1:ny + 1]
    u *= params.ubulk / (np.sum(u * dyp) / params.yly)
    return u


def rel_l2(a, b):
    """||a - b||_2 / ||b||_2, the relative L2 error of a field."""
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def xprofile(q, dyp, yly):
    """Depth- and span-averaged x profile of an interior field [nz, ny, nx]:
    sum over y with the dyp weights, mean over z, divided by yly (the
    definition paratc_xprofile evaluates on the device)."""
    return np.einsum("kji,j->i", q, dyp) / q.shape[0] / yly


def front_position(prof, dx, x_from=1.0, level=0.5):
    """Nose of the current: the furthest cell centre (i + 0.5) dx right of
    x_from, within half the periodic domain, whose value is at least
    `level`, moved to the level's linear crossing with the next cell; -1 if
    no cell there reaches it (the definition paratc_front_position uses)."""
    n = len(prof)
    xlx = n * dx
    last = -1
    for i, v in enumerate(prof):
        x = (i + 0.5) * dx
        if x_from < x < x_from + 0.5 * xlx and v >= level:
            last = i
    if last < 0:
        return -1.0
    xl = (last + 0.5) * dx
    pn = prof[(last + 1) % n]
    return xl + (prof[last] - level) / (prof[last] - pn) * dx if pn < level else xl
