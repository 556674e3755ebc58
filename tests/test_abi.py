"""The C ABI boundary (include/paratc.h) on the CPU: the library loads, exports
every declared entry point, and its host-side set-up (y-grid, namelist
reader, argument checks) matches the oracle.  No kernel is launched."""
import ctypes
import os
import re

import numpy as np
import pytest

from oracle import oracle_lib as ol
from paratc_b200 import abi, cases, lib

from .helpers import rel_err, yp_of

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")


def _declared():
    txt = open(os.path.join(ROOT, "include", "paratc.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(paratc_[a-z_0-9]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    L = lib.load()
    names = _declared()
    assert len(names) >= 20
    for n in names:
        assert hasattr(L, n), n
    assert set(lib.EXPORTED) <= set(names)


def test_header_constants_match_python():
    # the #define PARATC_* integers that the Python side mirrors
    hdr = open(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "paratc.h")).read()
    defs = dict(re.findall(r"#define\s+(PARATC_\w+)\s+(-?\d+)", hdr))
    assert int(defs["PARATC_SCHED_NCHOICES"]) == abi.SCHED_NCHOICES
    for n in ("PARATC_OK", "PARATC_ERR_BAD_ARG", "PARATC_ERR_TIMEOUT", "PARATC_ERR_NUMERIC"):
        assert int(defs[n]) == getattr(abi, n), n


def test_header_structs_match_ctypes():
    # offsets that a C compiler gives the structs, checked with a tiny probe
    assert ctypes.sizeof(abi.ParatcParams) % 8 == 0
    assert abi.ParatcParams.xlx.offset == 32
    assert ctypes.sizeof(abi.ParatcDiag) == 12 * 8


@pytest.mark.parametrize("mesh", [
    cases.Mesh([1.0, 1.0], [1.5, 1.5], [48, 48], [1, 1], [0, 1]),
    cases.Mesh([1.0], [0.9], [40], [2], [0]),
    cases.Mesh([1.0, 3.0], [0.0, 1.05], [10, 30], [0, 3], [0, 1]),
    cases.Mesh([2.0, 1.0, 1.0], [1.0, 2.0, 0.7], [16, 8, 9], [3, 1, 2], [1, 0, 1]),
])
def test_ycoord_library_matches_oracle(mesh):
    a = lib.mesh_ycoord(mesh, 2.0)
    b = ol.ycoord(mesh.section_length, mesh.section_cstret, mesh.nyc_section, mesh.stret_type, mesh.stret_option, 2.0)
    assert np.array_equal(a, b)
    assert a[0] == 0.0 and a[-1] == 2.0 and np.all(np.diff(a) > 0)


def test_namelist_reader():
    p, yp = lib.params_from_namelist(os.path.join(GOLD, "channel_small.prm"), scalar_on=True)
    assert (p.nxc, p.nyc, p.nzc) == (32, 24, 16)
    assert p.flow_type == 1 and p.is_ux_const == 1 and p.ischeme == 3 and p.icfl == 2
    assert p.ucrf == 0.25 and p.ux_bc[2] == -0.25 and p.ux_bc[3] == -0.25
    assert p.xnu == 2.381e-4 and p.dt_max == 0.005
    assert p.sdiff == pytest.approx(2.381e-4 / 2.0, rel=1e-15)
    assert list(p.gravity_eff_vec) == [0.0, -3.0, 0.0]
    assert p.falling_vel_vec[0] == 0.25 and p.falling_vel_vec[1] == -0.02
    assert list(p.scalar_bc_option) == [-3, -2] and p.scalar_bc_values[3] == 0.25
    ref = cases.tanh_mesh(24, 1.5, True)
    assert np.array_equal(yp, lib.mesh_ycoord(ref, 2.0))
    L = lib.load()
    ro = abi_run_options()
    assert L.paratc_run_options_from_namelist(os.path.join(GOLD, "channel_small.prm").encode(), ctypes.byref(ro)) == 0
    assert ro.run_name == b"Small/Chan" and ro.restart_dir == b"./restart/" and ro.ilast == 10
    assert ro.backup_freq == 5 and ro.cmd_lfile_freq == 2


# The reference's own input decks (copied verbatim by
# tests/golden/make_reference_inputs.py): every value below is the one
# written in the file, passed through ReadAndInitParameters'
# derivations (src/m_Parameters.f90:143-187: nxc = nxp - 1, uxBcValue -= uCRF
# under IsUseCRF else uCRF = 0, GravityDir normalised, SDiffCoe = xnu/Sc,
# GravityEffVec = GravityDir*GravityEff, FallingVelVec = GravityDir*FallingVel
# + (uCRF, 0, 0)).
REF_INPUTS = {
    "TurbCha0180_4th.standard": dict(
        scalar=False, grid=(384, 192, 256), flow_type=1, ischeme=3, icfl=2, is_ux_const=1, xnu=2.3310e-4,
        dt_max=0.02, cflc=1.5, ubulk=0.666666666666666666666666666667, ucrf=0.0, dom=(12.56637061, 2.0, 6.283185307),
        limits=(2.0, 0.2), gravity=(0.0, 0.0, 0.0), mesh=([1.0, 1.0], [1.0, 1.0], [96, 96], [2, 2], [0, 1]),
        run=(1, 27000, 0, 9000, 5, b"Cha180_4th", b"./CFD/Results/", b"./CFD/Restart/"),
        io=(20, 3000, 3000, 1, ("ux", "uy", "uz"), (1, 20, 20), (1, [10, 20, 30, 40, 50, 60, 70, 80, 90]))),
    "GravityFlow.prm": dict(
        scalar=True, grid=(192, 96, 128), flow_type=2, ischeme=3, icfl=1, is_ux_const=0, xnu=4.66591665597541e-04,
        dt_max=0.015, cflc=1.5, ubulk=1.4352, ucrf=0.0, dom=(12.56637061, 1.0, 4.188790205), limits=(4.0, 0.2),
        gravity=(0.0, 0.0, 0.0), mesh=([1.0, 1.0], [1.0, 1.0], [48, 48], [2, 2], [0, 1]),
        sc=dict(schmidt=1.0, geff=16.1865, gdir=(8.71557427476582e-02, -9.961946980917460e-01, 0.0),
                ws=1.679729996151150e-03, bc=(-3, -3), vals=(3.58630091313028, 3.58630091313028, 0.0, 0.0),
                init=5.0e-3),
        run=(1, 40000, 1, 10000, 5, b"TurbidityCurrent", b"./CFD/Results/", b"./CFD/Restart/"),
        io=(20, 5000, 5000, 1, ("ux", "uy", "uz", "scalar"), (1, 20, 10), (0, [5, 10, 15, 20, 25, 30, 35, 40, 45]))),
    "GravityFlow.small": dict(
        scalar=True, grid=(96, 96, 96), flow_type=2, ischeme=3, icfl=1, is_ux_const=0, xnu=4.66591665597541e-04,
        dt_max=0.03, cflc=1.5, ubulk=1.4352, ucrf=0.0, dom=(12.56637061, 1.0, 4.188790205), limits=(4.0, 0.2),
        gravity=(0.0, 0.0, 0.0), mesh=([1.0, 1.0], [1.0, 1.0], [48, 48], [2, 2], [0, 1]),
        sc=dict(schmidt=1.0, geff=16.1865, gdir=(8.71557427476582e-02, -9.961946980917460e-01, 0.0),
                ws=1.679729996151150e-03, bc=(-3, -3), vals=(3.58630091313028, 3.58630091313028, 0.0, 0.0),
                init=5.0e-3),
        run=(1, 200, 0, 10000, 5, b"TurbidityCurrent", b"./CFD/Results/", b"./CFD/Restart/"),
        io=(10, 50, 5000, 1, (), (1, 10, 10), (0, [5, 10, 15, 20, 25, 30, 35, 40, 45]))),
    "SF_Ri000.prm": dict(
        scalar=True, grid=(512, 128, 512), flow_type=1, ischeme=3, icfl=1, is_ux_const=0, xnu=2.3310e-4,
        dt_max=0.03, cflc=1.7, ubulk=0.65, ucrf=0.6, dom=(25.13274123, 2.0, 12.56637061), limits=None,
        gravity=(1.760473764e-3, 0.0, 0.0), mesh=([1.0, 1.0], [1.0, 1.0], [64, 64], [2, 2], [0, 1]),
        sc=dict(schmidt=0.7, geff=0.0, gdir=(0.0, 1.0, 0.0), ws=0.0, bc=(-1, -1), vals=(0.0, 1.0, 0.0, 0.0),
                init=0.5),
        run=(1, 60000, 0, 12000, 5, b"Ri000_", b"./CFD/Results1/", b"./CFD/Restart1/"), io=None),
}


def _sf(ubulk, ucrf, dom, grid, geff, ilast, name, k):
    """A stratified-flow deck: SF_Ri000's values with the ones that deck changes."""
    d = dict(REF_INPUTS["SF_Ri000.prm"])
    d.update(ubulk=ubulk, ucrf=ucrf, dom=dom, grid=grid)
    d["sc"] = dict(d["sc"], geff=geff)
    d["run"] = (1, ilast, 0, 12000, 5, name, b"./CFD/Results%d/" % k, b"./CFD/Restart%d/" % k)
    return d


REF_INPUTS["SF_Ri018.prm"] = _sf(0.75, 0.6, (25.13274123, 2.0, 12.56637061), (512, 128, 512), 0.03168852775, 60000,
                                 b"Ri018_", 2)
REF_INPUTS["SF_Ri120.prm"] = _sf(1.0, 0.6, (25.13274123, 2.0, 12.56637061), (512, 128, 512), 0.2112568517, 60000,
                                 b"Ri120_", 3)
REF_INPUTS["SF_Ri480.prm"] = _sf(1.6, 1.0, (56.54866776, 2.0, 25.13274123), (1152, 128, 1024), 0.8450274067, 90000,
                                 b"Ri480_", 4)


@pytest.mark.parametrize("fname", sorted(REF_INPUTS))
def test_namelist_reader_on_reference_inputs(fname):
    """paratc_params_from_namelist, paratc_run_options_from_namelist and
    paratc_io_options_from_namelist read the reference's own input files
    unchanged and give the values written in them."""
    ex = REF_INPUTS[fname]
    path = os.path.join(GOLD, fname)
    p, yp = lib.params_from_namelist(path, scalar_on=ex["scalar"])
    assert (p.nxc, p.nyc, p.nzc) == ex["grid"]
    assert (p.flow_type, p.ischeme, p.icfl, p.is_ux_const) == (ex["flow_type"], ex["ischeme"], ex["icfl"],
                                                               ex["is_ux_const"])
    assert p.xnu == ex["xnu"] and p.dt_max == ex["dt_max"] and p.cflc == ex["cflc"] and p.ubulk == ex["ubulk"]
    assert (p.xlx, p.yly, p.zlz) == ex["dom"] and tuple(p.gravity) == ex["gravity"]
    assert p.ucrf == ex["ucrf"]
    assert list(p.ux_bc) == [0.0 - ex["ucrf"]] * 6
    if ex["limits"]:
        assert (p.vel_limit, p.div_limit) == ex["limits"]
    sl, cs, nys, st, so = ex["mesh"]
    ref = cases.Mesh(sl, cs, nys, st, so)
    assert np.array_equal(yp, lib.mesh_ycoord(ref, p.yly))
    assert np.array_equal(yp, ol.ycoord(sl, cs, nys, st, so, p.yly))
    if ex["scalar"]:
        s = ex["sc"]
        g = np.array(s["gdir"])
        g = g / np.sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2])
        assert p.sdiff == pytest.approx(ex["xnu"] / s["schmidt"], rel=1e-15)
        assert np.allclose(list(p.gravity_eff_vec), g * s["geff"], rtol=1e-15, atol=0)
        fv = g * s["ws"]
        fv[0] += ex["ucrf"]
        assert np.allclose(list(p.falling_vel_vec), fv, rtol=1e-15, atol=0)
        assert tuple(p.scalar_bc_option) == s["bc"] and tuple(p.scalar_bc_values) == s["vals"]
        assert p.scalar_init_value == s["init"]
    L = lib.load()
    ro = abi_run_options()
    assert L.paratc_run_options_from_namelist(path.encode(), ctypes.byref(ro)) == 0
    assert (ro.ifirst, ro.ilast, ro.restart_flag, ro.backup_freq, ro.cmd_lfile_freq, ro.run_name, ro.res_dir,
            ro.restart_dir) == ex["run"]
    if ex["io"]:
        ivs, sstat, svisu, skip, saved, sp1, sp2 = ex["io"]
        o = lib.io_options_from_namelist(path, scalar_on=ex["scalar"])
        assert (o.ivstats, o.save_stat, o.save_visu) == (ivs, sstat, svisu)
        assert (o.iskip, o.jskip, o.kskip, o.xdmf_set_type) == (skip, skip, skip, 1)
        assert o.save_mask == lib.visu_mask(*saved)
        assert (o.clc_spectra1d, o.iv_spec, o.j_for_lcs) == sp1
        assert o.clc_spectra2d == sp2[0] and o.ny_spec2d == len(sp2[1])
        # &Spectra2DOpt is read only when clcSpectra2D is set (src/m_FlowCase.f90:209-214)
        if sp2[0]:
            assert list(o.iy_spec2d[:len(sp2[1])]) == sp2[1]


class abi_run_options(ctypes.Structure):
    _fields_ = [("ifirst", ctypes.c_int32), ("ilast", ctypes.c_int32), ("restart_flag", ctypes.c_int32),
                ("backup_freq", ctypes.c_int32), ("cmd_lfile_freq", ctypes.c_int32),
                ("run_name", ctypes.c_char * 64), ("res_dir", ctypes.c_char * 256),
                ("restart_dir", ctypes.c_char * 256)]


def test_namelist_errors(tmp_path):
    src = open(os.path.join(GOLD, "channel_small.prm")).read()
    bad = tmp_path / "odd.prm"
    bad.write_text(src.replace("nxp = 33", "nxp = 32"))
    with pytest.raises(lib.ParatcError) as e:
        lib.params_from_namelist(str(bad))
    assert e.value.code == abi.PARATC_ERR_BAD_ARG
    with pytest.raises(lib.ParatcError) as e:
        lib.params_from_namelist(str(tmp_path / "missing.prm"))
    assert e.value.code == abi.PARATC_ERR_IO
    bad2 = tmp_path / "ny.prm"
    bad2.write_text(src.replace("nycSection    =  12    12", "nycSection    =  12    11"))
    with pytest.raises(lib.ParatcError):
        lib.params_from_namelist(str(bad2))


def test_create_rejects_bad_arguments():
    L = lib.load()
    case = cases.small_channel(16, 12, 16)
    yp = yp_of(case)
    h = ctypes.c_void_p()
    for field, val in (("nxc", 15), ("nzc", 2), ("ischeme", 4), ("flow_type", 3), ("icfl", 0), ("nyc", 300)):
        p = case.params.copy()
        setattr(p, field, val)
        ypp = yp if field != "nyc" else np.linspace(0, 2, 301)
        rc = L.paratc_create(ctypes.byref(p), ypp.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 0, ctypes.byref(h))
        assert rc == abi.PARATC_ERR_BAD_ARG, field
    p = case.params.copy()
    p.nyc = 13  # channel needs an even nyc
    rc = L.paratc_create(ctypes.byref(p), np.linspace(0, 2, 14).ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 0,
                         ctypes.byref(h))
    assert rc == abi.PARATC_ERR_BAD_ARG
    assert L.paratc_strerror(abi.PARATC_ERR_DIV_LIMIT) == b"too big div"


def test_no_cpu_fallback_without_device():
    """Without a GPU the library refuses to create a context (it never falls
    back to a CPU path)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    case = cases.small_channel(16, 12, 16)
    with pytest.raises(lib.ParatcError) as e:
        lib.ChannelSystem(case.params, yp_of(case))
    assert e.value.code == abi.PARATC_ERR_NO_DEVICE


def test_io_options_reader():
    o = lib.io_options_from_namelist(os.path.join(GOLD, "channel_small.prm"), scalar_on=True)
    assert (o.ivstats, o.save_stat, o.save_visu) == (20, 200, 5)
    assert (o.iskip, o.jskip, o.kskip, o.xdmf_set_type) == (2, 1, 3, 1)
    assert o.save_mask == lib.visu_mask("ux", "uz", "wz", "pr", "Q", "scalar")
    assert (o.write_hist_old, o.read_hist_old) == (1, 0)
    assert (o.clc_spectra1d, o.iv_spec, o.j_for_lcs, o.clc_spectra2d, o.ny_spec2d) == (1, 40, 5, 1, 3)
    assert list(o.iy_spec2d[:3]) == [2, 6, 12]
    o2 = lib.io_options_from_namelist(os.path.join(GOLD, "channel_small.prm"), scalar_on=False)
    assert not o2.save_mask & lib.visu_mask("scalar")


@pytest.mark.parametrize("edit", [("ivSpec   = 40", "ivSpec   = 30"),     # mod(SaveStat, ivSpec) /= 0
                                  ("SaveStat = 200", "SaveStat = 210"),    # mod(SaveStat, ivstats) /= 0
                                  ("&IO_Options", "&IO_Optionz")])         # InitVisu reads it unconditionally
def test_io_options_errors(tmp_path, edit):
    txt = open(os.path.join(GOLD, "channel_small.prm")).read().replace(*edit)
    bad = tmp_path / "bad.prm"
    bad.write_text(txt)
    with pytest.raises(lib.ParatcError):
        lib.io_options_from_namelist(str(bad), scalar_on=True)


@pytest.mark.parametrize("set_type,single", [(0, False), (1, True)])
def test_xdmf_index(tmp_path, set_type, single):
    """InitVisu's XDMF index (src/m_IOAndVisu.f90:56-175): a well-formed
    XDMF file with the rectilinear grid written in Fortran's E14.7, the time
    list and one binary attribute per saved quantity and output step."""
    import xml.etree.ElementTree as ET

    p, yp = lib.params_from_namelist(os.path.join(GOLD, "channel_small.prm"), scalar_on=True)
    mask = lib.visu_mask("ux", "Q", "scalar")
    lib.write_xdmf(p, yp, str(tmp_path) + "/", "Run", 1, 10, 5, mask, set_type, single)
    path = tmp_path / "VisuForRun.xmf"
    txt = path.read_text()
    root = ET.fromstring(txt.split("\n", 2)[2])  # past the xml and DOCTYPE lines
    dom = root.find("Domain")
    nxo, nyo, nzo = (33, 25, 17) if set_type == 0 else (32, 24, 16)
    assert dom.find("Topology").get("Dimensions") == "%5d%5d%5d" % (nzo, nyo, nxo)
    axes = dom.find("Geometry").findall("DataItem")
    vals = [np.array([float(v) for v in re.findall(r"-?\d\.\d{7}E[+-]\d\d", a.text)]) for a in axes]
    assert [len(v) for v in vals] == [nxo, nyo, nzo]
    assert all(a.get("Precision") == ("4" if single else "8") for a in axes)
    dx = p.xlx / p.nxc
    xs = np.arange(nxo) * dx + (0 if set_type == 0 else dx / 2)
    ys = yp if set_type == 0 else 0.5 * (yp[:-1] + yp[1:])
    assert np.allclose(vals[0], xs, rtol=6e-7, atol=1e-7) and np.allclose(vals[1], ys, rtol=6e-7, atol=1e-7)
    # E14.7: 14 characters, 0.ddddddd mantissa
    if set_type == 0:
        assert "         0.0000000E+00 0.3926991E+00" in txt and " 0.2000000E+01 \n" in txt
    else:
        assert "         0.1963495E+00 0.5890486E+00" in txt
    coll = dom.find("Grid")
    times = coll.find("Time").find("DataItem")
    assert times.get("Dimensions") == "%6d" % 3 and times.text.split() == ["0", "5", "10"]
    steps = coll.findall("Grid")
    assert [g.get("Name") for g in steps] == ["T0000000000", "T0000000005", "T0000000010"]
    for g, t in zip(steps, (0, 5, 10)):
        at = g.findall("Attribute")
        assert [a.get("Name") for a in at] == ["ux", "Q", "scalar"]
        assert all(a.get("Center") == ("Cell" if set_type == 0 else "Node") for a in at)
        di = at[1].find("DataItem")
        assert di.get("Dimensions") == "%5d%5d%5d" % (16, 24, 32) and di.get("Format") == "Binary"
        assert di.text.strip() == "VisuForRun_Q_%010d" % t
