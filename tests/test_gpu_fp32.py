"""The FP32 storage form (PARATC_PREC_FP32) and the FP32 Poisson solve with
FP64 iterative refinement (paratc_poisson_refined), through the C ABI.

- Refined solve: on grids that take the one-CTA-per-plane transforms and the
  separate x / z transforms, the FP32-spectrum solve plus FP64-residual
  corrections reaches a relative residual max|r| / max|src| <= 1e-12 and
  agrees with the oracle's FP64 solve to 1e-12 of max|phi| (the FP64 path's
  own Poisson tolerance); one FP32 solve alone is far from it.
- FP32 storage step: from the same projected state, the FP32 form and the
  FP64 path after N steps differ by the FP32 rounding of the stored fields,
  amplified by the flow over the horizon; the bounds are stated per case.
  The divergence of the FP32-stored velocity is bounded by its rounding
  (about 1e-7 |u| / dx), checked against FP32_DIV.
- Switching the form converts the state: FP64 -> FP32 -> FP64 gives the
  FP32-rounded fields back.
"""
import numpy as np
import pytest

from oracle import oracle_lib as ol
from paratc_b200 import cases
from paratc_b200.abi import FT_HC
from paratc_b200.lib import ChannelSystem

from .helpers import fields_of, rel_err, variant, yp_of

pytestmark = pytest.mark.gpu

# relative error of the FP32 form against the FP64 path after NSTEP steps
# (max-norm, relative to the field's largest magnitude)
NSTEP = 10
FP32_VEL = 1e-5
FP32_PR = 1e-3
FP32_DIV = 1e-5


@pytest.mark.parametrize("dims,schedule", [((64, 48, 64), 0), ((64, 48, 64), 3), ((48, 40, 96), 3)])
def test_poisson_refined_matches_oracle(dims, schedule):
    import torch

    case = cases.small_channel(*dims)
    p = case.params
    yp = yp_of(case)
    g = ChannelSystem(p, yp)
    g.schedule = schedule
    src = cases.gaussian_source(cases.Case("src", p, case.mesh, "gauss_src", 42, 1.0))
    o = ol.Oracle(p, yp)
    ref = o.poisson(src)
    o.close()
    d_src = torch.from_numpy(src).cuda()
    d_phi = torch.empty_like(d_src)
    # one FP32-spectrum solve alone
    n0, r0 = g.poisson_refined(d_src.data_ptr(), d_phi.data_ptr(), rtol=1e-12, max_corr=0)
    e0 = rel_err(d_phi.cpu().numpy(), ref)
    n, r = g.poisson_refined(d_src.data_ptr(), d_phi.data_ptr(), rtol=1e-12, max_corr=4)
    e = rel_err(d_phi.cpu().numpy(), ref)
    print("refined %s sched %d: one solve rel err %.2e relres %.2e; %d corrections rel err %.2e relres %.2e"
          % (dims, schedule, e0, r0, n, e, r))
    assert n0 == 0 and r0 > 1e-10 and e0 > 1e-10
    assert r <= 1e-12 and 1 <= n <= 3
    assert e <= 1e-12
    # the asynchronous form with the same count gives the same potential
    d_phi2 = torch.empty_like(d_src)
    g.poisson_refined_async(d_src.data_ptr(), d_phi2.data_ptr(), n)
    torch.cuda.synchronize()
    assert torch.equal(d_phi, d_phi2)
    g.close()


def _pair(case):
    yp = yp_of(case)
    f = fields_of(case, yp)
    a = ChannelSystem(case.params, yp)
    b = ChannelSystem(case.params, yp)
    for x in (a, b):
        x.set_fields(f["ux"], f["uy"], f["uz"], f["p"], f["c"])
        x.project()
    return a, b


def _case(name):
    if name == "channel_64":
        return cases.small_channel(64, 48, 64)
    if name == "channel_z128":  # TMA-fed z transforms (nz >= 128) on the float2 spectrum
        return cases.small_channel(32, 24, 128)
    if name == "channel_z128_odd":  # ny * (nx/2+1) odd (a half channel): no float2 map, register-fed z
        return cases.small_channel(32, 25, 128, flow_type=FT_HC, xnu=1e-3, yly=1.0, is_ux_const=0)
    return variant(name)


# the plane transforms (schedule 0), the separate x / z transforms (3), the
# divergence-fed x transform (8), the TMA-fed z transforms (6), and the
# default schedule of smaller variants (scalar, CFL-controlled dt, AB2)
@pytest.mark.parametrize("name,schedule", [("channel_64", 0), ("channel_64", 3), ("channel_64", 8), ("channel_z128", 6),
                                           ("channel_z128_odd", 6), ("channel", -1),
                                           ("halfchannel_scalar", -1), ("channel_cfl", -1), ("channel_ab2", -1)])
def test_fp32_storage_steps_track_fp64(name, schedule):
    case = _case(name)
    g64, g32 = _pair(case)
    if schedule >= 0:
        g64.schedule = schedule
        g32.schedule = schedule
    g32.precision = "fp32"
    assert g32.precision == "fp32"
    worst_div = 0.0
    for _ in range(NSTEP):
        d64 = g64.iterate(1)
        d32 = g32.iterate(1)
        assert d64.divmax <= 1e-10
        worst_div = max(worst_div, d32.divmax)
        assert abs(d32.dt - d64.dt) <= 1e-4 * d64.dt
    f64, f32 = g64.get_fields(), g32.get_fields()
    errs = {n: rel_err(f32[n], f64[n]) for n in f64 if n in ("ux", "uy", "uz", "p", "c")}
    print("fp32 %s after %d steps: %s, max div %.2e" % (name, NSTEP, {n: "%.2e" % v for n, v in errs.items()},
                                                        worst_div))
    for n in ("ux", "uy", "uz", "c"):
        if n in errs:
            assert errs[n] <= FP32_VEL, (n, errs[n])
    assert errs["p"] <= FP32_PR
    assert worst_div <= FP32_DIV
    g64.close()
    g32.close()


@pytest.mark.parametrize("shape", [(1, 0), (0, 2), (1, 2)])
@pytest.mark.parametrize("name", ["channel_64", "halfchannel_scalar", "channel_cfl"])
def test_fp32_launch_shapes(name, shape):
    """The FP32 storage form's other launch shapes, (rhs_var, helm_var):
    the right-hand side with two z-adjacent cells per thread (rhs_var 1) and
    the Helmholtz sweeps in float arithmetic (helm_var 2).  Each keeps the
    form's bounds against the FP64 path and agrees with the default shapes
    (0, 0) within them."""
    case = _case(name)
    g64, g32 = _pair(case)
    gb = ChannelSystem(case.params, yp_of(case))
    f = fields_of(case, yp_of(case))
    gb.set_fields(f["ux"], f["uy"], f["uz"], f["p"], f["c"])
    gb.project()
    for g in (g32, gb):
        g.precision = "fp32"
    t = gb.tuning
    t.rhs_var, t.helm_var = shape
    gb.tuning = t
    assert (gb.tuning.rhs_var, gb.tuning.helm_var) == shape
    assert (g32.tuning.rhs_var, g32.tuning.helm_var) == (0, 0)
    worst_div = 0.0
    for _ in range(NSTEP):
        g64.iterate(1)
        g32.iterate(1)
        worst_div = max(worst_div, gb.iterate(1).divmax)
    f64, f32, fb = g64.get_fields(), g32.get_fields(), gb.get_fields()
    for n in ("ux", "uy", "uz", "p", "c"):
        if f64.get(n) is None:
            continue
        tol = FP32_PR if n == "p" else FP32_VEL
        assert rel_err(fb[n], f64[n]) <= tol, (n, rel_err(fb[n], f64[n]))
        assert rel_err(fb[n], f32[n]) <= tol, (n, rel_err(fb[n], f32[n]))
    assert worst_div <= FP32_DIV
    for g in (g64, g32, gb):
        g.close()


def test_fp32_switch_round_trip():
    case = variant("channel")
    yp = yp_of(case)
    f = fields_of(case, yp)
    g = ChannelSystem(case.params, yp)
    g.set_fields(f["ux"], f["uy"], f["uz"], f["p"])
    h64 = g.get_fields(["ux", "uy", "uz", "p"])  # as loaded (wall rows set)
    g.precision = "fp32"
    h = g.get_fields(["ux", "uy", "uz", "p"])
    for n in ("ux", "uy", "uz"):
        assert np.array_equal(h[n], h64[n].astype(np.float32).astype(np.float64)), n
    assert np.array_equal(h["p"], h64["p"])  # the pressure stays FP64
    g.precision = "fp64"
    h2 = g.get_fields(["ux"])
    assert np.array_equal(h2["ux"], h["ux"])
    g.close()
