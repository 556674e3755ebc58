"""The mixed-precision step (PARATC_PREC_MIXED): the explicit right-hand
side in FP32 arithmetic, everything else FP64.  Against the FP64 oracle:
the right-hand side itself within FP32 rounding (1e-5 of its largest
magnitude), the velocities and the scalar after 10 steps within 1e-6, the
pressure within 1e-5 (it accumulates the potential, whose source is the
divergence of the FP32-rounded u*), the divergence after every step at the
FP64 level (1e-10), the mean pressure gradient of the flow-rate forcing (the
FP64 s3tot sum of fields that differ at 1e-7) within 1e-6 of the oracle's
PrGradAver."""
import numpy as np
import pytest

from oracle import oracle_lib as ol
from paratc_b200 import cases
from paratc_b200.lib import ChannelSystem

from .helpers import fields_of, rel_err, variant, yp_of

pytestmark = pytest.mark.gpu


def _pair(case):
    yp = yp_of(case)
    f = fields_of(case, yp)
    o = ol.Oracle(case.params, yp)
    g = ChannelSystem(case.params, yp)
    o.set_fields(f["ux"], f["uy"], f["uz"], f["p"], f["c"])
    g.set_fields(f["ux"], f["uy"], f["uz"], f["p"], f["c"])
    g.precision = "mixed"
    assert g.precision == "mixed"
    return o, g


@pytest.mark.parametrize("name", ["channel", "halfchannel_scalar", "channel_scalar_crf", "channel_odd"])
def test_mixed_rhs_stage(name):
    case = variant(name)
    o, g = _pair(case)
    dt = case.params.dt_max
    o.substep(1, dt, stop_stage=1)
    g.substep_stage(1, dt, 1)
    for n in ["rhsx", "rhsy", "rhsz"] + (["rhsc"] if case.params.scalar_on else []):
        e = rel_err(g.get_work(n), o.get_work(n))
        assert e <= 1e-5, "%s %s rel err %.3e" % (name, n, e)


@pytest.mark.parametrize("name", ["channel", "halfchannel_scalar", "channel_scalar_crf"])
def test_mixed_steps(name):
    case = variant(name)
    o, g = _pair(case)
    for s in range(10):
        rc, do = o.step()
        assert rc == 0
        dg = g.iterate(1, raise_on_guard=False)
        assert dg.divmax <= 1e-10, "%s step %d divmax %.3e" % (name, s + 1, dg.divmax)
        assert abs(dg.pr_grad_aver - do.pr_grad_aver) <= 1e-6 * max(abs(do.pr_grad_aver), 1e-6)
    fo, fg = o.get_fields(), g.get_fields()
    for n in ("ux", "uy", "uz", "p", "c"):
        if fo.get(n) is None:
            continue
        e = rel_err(fg[n], fo[n])
        tol = 1e-5 if n == "p" else 1e-6
        assert e <= tol, "%s %s rel err after 10 steps %.3e" % (name, n, e)
    g.precision = "fp64"
    assert g.precision == "fp64"
