"""The ensemble API (paratc_batch_*): members of uneven sizes and options
advanced together, with and without the captured CUDA graph, must give
exactly the fields and diagnostics of the same cases stepped one by one
(same kernels on the same inputs; every reduction has a fixed order)."""
import numpy as np
import pytest

from paratc_b200 import cases
from paratc_b200.lib import BatchSystem, ChannelSystem

from .helpers import fields_of, variant, yp_of

pytestmark = pytest.mark.gpu

NAMES = ("ux", "uy", "uz", "p", "c", "hx", "hy", "hz", "hc")


def _members():
    # uneven grids, a CFL-controlled dt, a scalar with a half channel
    return [cases.small_channel(16, 12, 16), cases.small_channel(24, 20, 30), variant("channel_cfl"),
            variant("halfchannel_scalar"), cases.small_channel(32, 24, 16)]


def _setup(cs):
    yps = [yp_of(c) for c in cs]
    init = [fields_of(c, y) for c, y in zip(cs, yps)]
    b = BatchSystem([c.params for c in cs], yps)
    singles = [ChannelSystem(c.params, y) for c, y in zip(cs, yps)]
    for m, s, f in zip(b.members, singles, init):
        for g in (m, s):
            g.set_fields(f["ux"], f["uy"], f["uz"], f["p"], f["c"])
    return b, singles, init


def _same(b, singles):
    for i, (m, s) in enumerate(zip(b.members, singles)):
        fm, fs = m.get_fields(), s.get_fields()
        for n in NAMES:
            if fm.get(n) is None:
                continue
            assert np.array_equal(fm[n], fs[n]), "member %d field %s differs" % (i, n)


@pytest.mark.parametrize("use_graph", [True, False])
def test_batch_equals_single_contexts(use_graph):
    cs = _members()
    b, singles, init = _setup(cs)
    d = b.iterate(4, use_graph=use_graph)
    ds = [s.iterate(4) for s in singles]
    _same(b, singles)
    for i in range(len(cs)):
        assert d[i].dt == ds[i].dt and d[i].divmax == ds[i].divmax and d[i].sim_time == ds[i].sim_time, i
        assert d[i].cfl == ds[i].cfl and list(d[i].vmax) == list(ds[i].vmax), i
    if use_graph:
        assert b.graph_kernels > 0
    # a member whose state is reset takes an ordinary step before the graph runs again
    f = init[2]
    for g in (b.members[2], singles[2]):
        g.set_fields(f["ux"], f["uy"], f["uz"], f["p"], f["c"])
    b.iterate(3, use_graph=use_graph)
    for s in singles:
        s.iterate(3)
    _same(b, singles)
    b.close()


def test_batch_members_are_contexts():
    cs = [cases.small_channel(16, 12, 16), cases.small_channel(32, 24, 16)]
    b, singles, _ = _setup(cs)
    for m, s in zip(b.members, singles):
        assert m.get_time() == s.get_time()
        m.project()
        s.project()
    _same(b, singles)
    b.iterate(2)
    for s in singles:
        s.iterate(2)
    _same(b, singles)
    b.close()


def test_async_transfers_equal_sync():
    """paratc_set_fields_async / steps_async / get_fields_async on pinned
    buffers give the fields of the synchronous calls."""
    import torch

    case = cases.small_channel(32, 24, 16)
    yp = yp_of(case)
    f = fields_of(case, yp)
    a = ChannelSystem(case.params, yp)
    s = ChannelSystem(case.params, yp)
    pin = {n: torch.empty(a.shape, dtype=torch.float64, pin_memory=True).numpy() for n in ("ux", "uy", "uz", "p")}
    for n in pin:
        pin[n][...] = f[n]
    for _ in range(3):
        a.set_fields_async(pin["ux"], pin["uy"], pin["uz"], pin["p"])
        a.iterate_async(1)
        a.get_fields_into_async(pin)
        a.sync()
        s.set_fields(f["ux"], f["uy"], f["uz"], f["p"])
        s.iterate(1)
        f = s.get_fields()
        for n in pin:
            assert np.array_equal(pin[n], f[n]), n
    a.last_diag()


def test_batch_recaptures_after_schedule_change():
    """A member whose Poisson schedule changes after the graph was captured
    (auto-tuning, or a pinned choice) is stepped with the new kernels: the
    graph is captured again."""
    cs = [cases.small_channel(16, 12, 16), cases.small_channel(32, 24, 16)]
    b, singles, _ = _setup(cs)
    b.iterate(3, use_graph=True)
    for s in singles:
        s.iterate(3)
    _same(b, singles)
    for g in (b.members[1], singles[1]):
        g.schedule = 5  # generic transforms, streaming y-solve
    b.iterate(3, use_graph=True)
    for s in singles:
        s.iterate(3)
    _same(b, singles)
    b.close()
