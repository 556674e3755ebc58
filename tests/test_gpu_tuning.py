"""The tuner of launch shapes (paratc_autotune_all) and its cache.

Every compiled launch shape of the right-hand side (FP64: rows prefetched 1
or 2 ahead, 2 or 1 cells per thread) and of the Helmholtz sweeps (8 or 4 rows
per register chunk) must give the oracle's fields (1e-10 after one step,
1e-8 after two, as the other parity tests); the tuner picks one of them,
writes the picks to a JSON cache, and a second context on the same grid (or
paratc_create with PARATC_TUNE_CACHE naming the file) applies them without
searching.
"""
import json
import os

import numpy as np
import pytest

from oracle import oracle_lib as ol
from paratc_b200 import abi, cases
from paratc_b200.lib import ChannelSystem

from .helpers import fields_of, rel_err, variant, yp_of

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["channel", "halfchannel_scalar"])
@pytest.mark.parametrize("rhs_var", [0, 1, 2])
@pytest.mark.parametrize("helm_var", [0, 1])
def test_launch_shapes_match_oracle(name, rhs_var, helm_var):
    case = variant(name)
    yp = yp_of(case)
    f = fields_of(case, yp)
    o = ol.Oracle(case.params, yp)
    g = ChannelSystem(case.params, yp)
    t = g.tuning
    t.rhs_var, t.helm_var = rhs_var, helm_var
    g.tuning = t
    assert (g.tuning.rhs_var, g.tuning.helm_var) == (rhs_var, helm_var)
    for x in (o, g):
        x.set_fields(f["ux"], f["uy"], f["uz"], f["p"], f["c"])
    for s, tol in ((1, 1e-10), (2, 1e-8)):
        rc, _ = o.step()
        assert rc == 0
        g.iterate(1)
        fo, fg = o.get_fields(), g.get_fields()
        for n in ("ux", "uy", "uz", "p", "c"):
            if n in fo and fo[n] is not None and n in fg:
                e = rel_err(fg[n], fo[n])
                assert e <= tol, (name, rhs_var, helm_var, s, n, e)
    g.close()
    o.close()


def test_autotune_all_writes_and_reads_the_cache(tmp_path, monkeypatch):
    case = cases.small_channel(64, 48, 64)
    yp = yp_of(case)
    f = fields_of(case, yp)
    path = str(tmp_path / "tune.json")
    a = ChannelSystem(case.params, yp)
    a.set_fields(f["ux"], f["uy"], f["uz"], f["p"])
    a.project()
    before = a.get_fields()
    ta = a.autotune_all(nrep=2, cache_path=path)
    assert ta.from_cache == 0 and ta.step_ms > 0
    assert 0 <= ta.rhs_var < 3 and 0 <= ta.helm_var < 2 and 0 <= ta.schedule < abi.SCHED_NCHOICES
    # the search puts the state back
    after = a.get_fields()
    for n in ("ux", "uy", "uz", "p", "hx"):
        assert np.array_equal(before[n], after[n]), n
    entries = json.load(open(path))
    assert len(entries) == 1
    (key, val), = entries.items()
    assert "64x48x64" in key and val["rhs_var"] == ta.rhs_var and val["helm_var"] == ta.helm_var
    # a second context on the same grid reads the picks and skips the search
    b = ChannelSystem(case.params, yp)
    tb = b.autotune_all(nrep=2, cache_path=path)
    assert tb.from_cache == 1
    assert (tb.schedule, tb.rhs_var, tb.helm_var) == (ta.schedule, ta.rhs_var, ta.helm_var)
    # and so does paratc_create when PARATC_TUNE_CACHE names the file
    monkeypatch.setenv("PARATC_TUNE_CACHE", path)
    c = ChannelSystem(case.params, yp)
    tc = c.tuning
    assert tc.from_cache == 1 and (tc.schedule, tc.rhs_var, tc.helm_var) == (ta.schedule, ta.rhs_var, ta.helm_var)
    # another grid has no entry: a fresh search, and the file keeps both
    other = cases.small_channel(32, 24, 16)
    d = ChannelSystem(other.params, yp_of(other))
    td = d.autotune_all(nrep=2, cache_path=path)
    assert td.from_cache == 0
    assert len(json.load(open(path))) == 2
    for x in (a, b, c, d):
        x.close()
    # the tuned context still steps like the oracle
    o = ol.Oracle(case.params, yp)
    g = ChannelSystem(case.params, yp)
    assert g.tuning.from_cache == 1
    for x in (o, g):
        x.set_fields(f["ux"], f["uy"], f["uz"], f["p"])
    o.step()
    g.iterate(1)
    fo, fg = o.get_fields(), g.get_fields()
    for n in ("ux", "uy", "uz", "p"):
        assert rel_err(fg[n], fo[n]) <= 1e-10
    g.close()
    o.close()
    os.environ.pop("PARATC_TUNE_CACHE", None)
