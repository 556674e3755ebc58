"""Failure paths of a step, driven from the host or by a test setting: no
kernel is made to fault, trap or wait without bound.

- The guards of ChannelIterate (src/m_ChannelSystem.f90:143,145): a step
  whose max|div u| exceeds div_limit returns PARATC_ERR_DIV_LIMIT, one whose
  smallest velocity maximum exceeds vel_limit returns PARATC_ERR_VEL_LIMIT;
  the fields then hold the state after the step.
- A NaN or an Inf placed in one cell of a field on the host makes the step
  return PARATC_ERR_NONFINITE (the grid maxima keep a NaN), through the
  synchronous call and through the asynchronous one with its step index.
- The bounded waits of the TMA-fed kernels: with the poll limit of their
  pipeline waits set to zero, every such wait gives up at once, the CTA waits
  (with the full limit) for its own copies in flight and returns, and the next
  synchronising call returns PARATC_ERR_TIMEOUT.  A fresh context on the same
  GPU then solves the Poisson equation to 1e-12 of the oracle.
"""
import numpy as np
import pytest

from oracle import oracle_lib as ol
from paratc_b200 import abi, cases
from paratc_b200.lib import ChannelSystem, ParatcError

from .helpers import fields_of, rel_err, variant, yp_of

pytestmark = pytest.mark.gpu


def _ctx(case, **limits):
    p = case.params.copy()
    for k, v in limits.items():
        setattr(p, k, v)
    yp = yp_of(case)
    return ChannelSystem(p, yp), fields_of(case, yp)


@pytest.mark.parametrize("name,field,value", [
    ("channel", "ux", np.nan), ("channel", "uz", np.inf), ("channel", "uy", -np.inf),
    ("halfchannel_scalar", "c", np.nan), ("halfchannel_scalar", "p", np.nan),
])
def test_nonfinite_cell_stops_the_step(name, field, value):
    case = variant(name)
    g, f = _ctx(case)
    bad = {k: (None if v is None else v.copy()) for k, v in f.items()}
    bad[field][3, 5, 7] = value
    g.set_fields(bad["ux"], bad["uy"], bad["uz"], bad["p"], bad["c"])
    with pytest.raises(ParatcError) as e:
        g.iterate(1)
    assert e.value.code == abi.PARATC_ERR_NONFINITE
    # the asynchronous form reports the first failing step of the batch
    g.set_fields(bad["ux"], bad["uy"], bad["uz"], bad["p"], bad["c"])
    g.iterate_async(3)
    with pytest.raises(ParatcError) as e:
        g.last_diag()
    assert e.value.code == abi.PARATC_ERR_NONFINITE
    assert "at step 1" in str(e.value)
    # the context stays usable: clean fields step normally
    g.set_fields(f["ux"], f["uy"], f["uz"], f["p"], f["c"])
    g.project()
    d = g.iterate(2)
    assert np.isfinite(d.divmax) and d.divmax <= 1e-10
    g.close()


def test_div_limit_guard():
    case = variant("channel")
    g, f = _ctx(case, div_limit=1e-30)
    ref, _ = _ctx(case)
    for x in (g, ref):
        x.set_fields(f["ux"], f["uy"], f["uz"], f["p"])
        x.project()
    with pytest.raises(ParatcError) as e:
        g.iterate(1)
    assert e.value.code == abi.PARATC_ERR_DIV_LIMIT
    d = ref.iterate(1)
    assert 1e-30 < d.divmax <= 1e-10
    # the fields hold the state after the step, as in a run without the limit
    fg, fr = g.get_fields(), ref.get_fields()
    for n in ("ux", "uy", "uz", "p"):
        assert np.array_equal(fg[n], fr[n]), n
    # raise_on_guard=False hands back the step's diagnostics instead
    d2 = g.iterate(1, raise_on_guard=False)
    assert d2.divmax > 1e-30
    g.close()
    ref.close()


def test_vel_limit_guard():
    case = variant("channel")
    g, f = _ctx(case, vel_limit=1e-3)
    g.set_fields(f["ux"], f["uy"], f["uz"], f["p"])
    g.project()
    with pytest.raises(ParatcError) as e:
        g.iterate(1)
    assert e.value.code == abi.PARATC_ERR_VEL_LIMIT
    d = g.iterate(1, raise_on_guard=False)
    assert min(d.vmax) > 1e-3
    g.close()
    # just above the smallest velocity maximum: no stop
    g, f = _ctx(case, vel_limit=1e3)
    g.set_fields(f["ux"], f["uy"], f["uz"], f["p"])
    g.project()
    g.iterate(1)
    g.close()


# grids and schedules whose Poisson solve runs the TMA-fed kernels:
# 7 TMA z transforms + bulk-copy x transforms, 8 divergence-fed x transform,
# 11 both (choice = 2 * s + y-solve variant)
@pytest.mark.parametrize("schedule", [7, 8, 11])
def test_bounded_wait_timeout(schedule):
    case = cases.small_channel(64, 24, 128)
    g, f = _ctx(case)
    g.set_fields(f["ux"], f["uy"], f["uz"], f["p"])
    g.schedule = schedule
    g.set_wait_limit(0)
    rng = np.random.Generator(np.random.PCG64(3))
    src = rng.standard_normal(g.shape)
    src -= src.mean()
    with pytest.raises(ParatcError) as e:
        if schedule == 8:
            g.iterate(1)  # the divergence-fed transform runs inside a step
        else:
            g.poisson(src)
    assert e.value.code == abi.PARATC_ERR_TIMEOUT
    # the context keeps reporting it; a new one on the same GPU works
    with pytest.raises(ParatcError):
        g.sync()
    g.close()
    yp = yp_of(case)
    h = ChannelSystem(case.params, yp)
    h.schedule = schedule
    phi = h.poisson(src)
    o = ol.Oracle(case.params, yp)
    assert rel_err(phi, o.poisson(src)) <= 1e-12
    # restoring the default limit on a context keeps it working
    h.set_wait_limit(None)
    h.set_fields(f["ux"], f["uy"], f["uz"], f["p"])
    h.project()
    assert h.iterate(1).divmax <= 1e-10
    h.close()
    o.close()

