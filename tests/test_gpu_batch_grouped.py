"""Grouped launches of an ensemble (paratc_batch_set_mode(PARATC_BATCH_GROUPED)).

Every stage of a batch step is one launch per kernel instantiation over the
members that share it; each member's CTAs run that member's own launch shape
on its own fields.  So a grouped batch must give exactly (bitwise) the fields
and diagnostics of the same cases stepped one by one with the same Poisson
schedule (the separate compile-time-length transforms): members of uneven
sizes, a CFL-controlled dt, a scalar, RK2 / AB2 members with fewer substeps,
FP32-storage members next to FP64 ones.  The x inverse of a single context
is the plain kernel here (PARATC_XT_TMA=0), the one the grouped step runs.

One exception: a member with FP32 right-hand-side arithmetic (the FP32
storage form) rounds its RHS as the grouped kernel's compilation does, which
may differ from its own launch's in the last float bit (the one-context
kernel takes its constants from the parameter bank, the grouped one from the
member's record); those members are held to FP32_REL (velocity, scalar) and
FP32_REL_P (pressure, histories) of each field's largest magnitude after
the steps of a test, the bounds of the FP32 form against the FP64 path, and
their diagnostics to DIAG32_REL.
"""
import numpy as np
import pytest

from paratc_b200 import cases
from paratc_b200.lib import BatchSystem, ChannelSystem, ParatcError

from .helpers import fields_of, variant, yp_of

pytestmark = pytest.mark.gpu

NAMES = ("ux", "uy", "uz", "p", "c", "hx", "hy", "hz", "hc")
FP32_REL = 1e-5
FP32_REL_P = 1e-3
DIAG32_REL = 1e-5


def _members():
    return [cases.small_channel(16, 12, 16), cases.small_channel(24, 20, 30), variant("channel_cfl"),
            variant("halfchannel_scalar"), cases.small_channel(32, 24, 16), variant("channel_ab2"),
            variant("channel_rk2"), cases.small_channel(64, 48, 64)]


def _setup(cs, monkeypatch, precisions=None):
    monkeypatch.setenv("PARATC_XT_TMA", "0")
    yps = [yp_of(c) for c in cs]
    init = [fields_of(c, y) for c, y in zip(cs, yps)]
    b = BatchSystem([c.params for c in cs], yps)
    singles = [ChannelSystem(c.params, y) for c, y in zip(cs, yps)]
    for i, (m, s, f) in enumerate(zip(b.members, singles, init)):
        for g in (m, s):
            g.set_fields(f["ux"], f["uy"], f["uz"], f["p"], f["c"])
            if precisions is not None:
                g.precision = precisions[i]
    return b, singles, init


def _group(b, singles):
    b.mode = "grouped"
    assert b.mode == "grouped"
    # the batch put every member on the separate transforms; the singles follow
    for m, s in zip(b.members, singles):
        assert m.schedule in (2, 3)
        s.tuning = m.tuning


def _f32(m):
    return m.precision == "fp32"


def _same(b, singles):
    for i, (m, s) in enumerate(zip(b.members, singles)):
        fm, fs = m.get_fields(), s.get_fields()
        for n in NAMES:
            if fm.get(n) is None:
                continue
            if _f32(m):
                e = float(np.abs(fm[n] - fs[n]).max() / max(np.abs(fs[n]).max(), 1e-300))
                tol = FP32_REL if n in ("ux", "uy", "uz", "c") else FP32_REL_P
                assert e <= tol, "member %d field %s differs by %.2e" % (i, n, e)
            else:
                assert np.array_equal(fm[n], fs[n]), "member %d field %s differs" % (i, n)


def _same_diag(b, d, ds):
    for i in range(len(d)):
        if _f32(b.members[i]):
            for x, y in ((d[i].dt, ds[i].dt), (d[i].sim_time, ds[i].sim_time), (d[i].cfl, ds[i].cfl)):
                assert abs(x - y) <= DIAG32_REL * abs(y), i
            continue
        assert d[i].dt == ds[i].dt and d[i].divmax == ds[i].divmax and d[i].sim_time == ds[i].sim_time, i
        assert d[i].cfl == ds[i].cfl and list(d[i].vmax) == list(ds[i].vmax), i
        assert d[i].pr_grad_aver == ds[i].pr_grad_aver and d[i].ux_mean == ds[i].ux_mean, i


@pytest.mark.parametrize("use_graph", [True, False])
def test_grouped_equals_single_contexts(use_graph, monkeypatch):
    cs = _members()
    b, singles, init = _setup(cs, monkeypatch)
    _group(b, singles)
    d = b.iterate(4, use_graph=use_graph)
    ds = [s.iterate(4) for s in singles]
    _same(b, singles)
    _same_diag(b, d, ds)
    n_grouped = b.step_launches
    assert n_grouped > 0
    if use_graph:
        assert b.graph_kernels == n_grouped
    # a member whose state is reset takes an ordinary step before the grouped ones
    f = init[2]
    for g in (b.members[2], singles[2]):
        g.set_fields(f["ux"], f["uy"], f["uz"], f["p"], f["c"])
    d = b.iterate(3, use_graph=use_graph)
    ds = [s.iterate(3) for s in singles]
    _same(b, singles)
    _same_diag(b, d, ds)
    # the same members one launch per member and stage: more launches per step
    b.mode = "streams"
    b.iterate(2, use_graph=True)
    for s in singles:
        s.iterate(2)
    _same(b, singles)
    print("launches per step: grouped %d, streams %d" % (n_grouped, b.graph_kernels))
    assert n_grouped < b.graph_kernels
    b.close()


def test_grouped_fp32_and_fp64_members(monkeypatch):
    cs = [cases.small_channel(32, 24, 16), cases.small_channel(32, 24, 16), variant("halfchannel_scalar"),
          cases.small_channel(64, 48, 64), cases.small_channel(48, 40, 96)]
    prec = ["fp32", "fp64", "fp32", "fp32", "fp64"]
    b, singles, _ = _setup(cs, monkeypatch, prec)
    _group(b, singles)
    d = b.iterate(5, use_graph=True)
    ds = [s.iterate(5) for s in singles]
    _same(b, singles)
    _same_diag(b, d, ds)
    b.close()


def test_grouped_tables_follow_member_changes(monkeypatch):
    """A member re-tuned, or switched to the FP32 storage form, while the
    batch is grouped: the next batch call rebuilds the tables (and puts the
    member back on the separate transforms)."""
    cs = [cases.small_channel(32, 24, 16), cases.small_channel(64, 48, 64)]
    b, singles, _ = _setup(cs, monkeypatch)
    _group(b, singles)
    b.iterate(2)
    for s in singles:
        s.iterate(2)
    _same(b, singles)
    b.members[1].schedule = 0  # the plane transforms: not a grouped form
    for g in (b.members[0], singles[0]):
        g.precision = "fp32"
    b.iterate(3)
    assert b.members[1].schedule in (2, 3)
    singles[1].tuning = b.members[1].tuning
    for s in singles:
        s.iterate(3)
    _same(b, singles)
    b.close()


def test_grouped_refuses_generic_lengths(monkeypatch):
    # nxc = 20: no compile-time-length x transform for 10 points (the
    # generic mixed-radix one serves it)
    cs = [cases.small_channel(16, 12, 16), cases.small_channel(20, 12, 16)]
    b, _, _ = _setup(cs, monkeypatch)
    with pytest.raises(ParatcError):
        b.mode = "grouped"
    assert b.mode == "streams"
    b.iterate(1)
    b.close()
