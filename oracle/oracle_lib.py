"""ctypes wrapper of the C oracle (oracle/paratc_oracle.c) -- TEST INFRASTRUCTURE.

The oracle restates ParaTC's Fortran hot path on the CPU; the CUDA library is
checked against it.  Arrays are numpy float64 of shape (nzc, nyc, nxc),
C-contiguous, i.e. the Fortran (x fastest) order of the reference.
"""
import ctypes
import os
import subprocess

import numpy as np

from paratc_b200.abi import ParatcDiag, ParatcParams

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libparatc_oracle.so")
_lib = None

_dp = ctypes.POINTER(ctypes.c_double)


def build(force=False):
    """Compile the oracle with its Makefile (gcc + OpenMP)."""
    if force or not os.path.exists(_LIB_PATH):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        L.orc_create.argtypes = [ctypes.POINTER(ParatcParams), _dp, ctypes.POINTER(ctypes.c_void_p)]
        L.orc_destroy.argtypes = [ctypes.c_void_p]
        L.orc_destroy.restype = None
        L.orc_set_threads.argtypes = [ctypes.c_int]
        L.orc_set_threads.restype = None
        L.orc_set_fields.argtypes = [ctypes.c_void_p] + [_dp] * 9
        L.orc_get_fields.argtypes = [ctypes.c_void_p] + [_dp] * 9
        L.orc_get_halo.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp]
        L.orc_get_work.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp]
        L.orc_set_time.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double]
        L.orc_get_time.argtypes = [ctypes.c_void_p, _dp, _dp, _dp]
        L.orc_step.argtypes = [ctypes.c_void_p, ctypes.POINTER(ParatcDiag)]
        L.orc_substep.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_int, _dp]
        L.orc_poisson.argtypes = [ctypes.c_void_p, _dp, _dp]
        L.orc_project.argtypes = [ctypes.c_void_p, _dp]
        L.orc_diagnostics.argtypes = [ctypes.c_void_p, ctypes.POINTER(ParatcDiag)]
        L.orc_metric.argtypes = [ctypes.c_void_p, ctypes.c_char_p, _dp, ctypes.c_int]
        L.orc_stats.argtypes = [ctypes.c_void_p, _dp]
        L.orc_spectra.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp]
        L.orc_spectra2d.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int32), _dp]
        L.orc_visu.argtypes = [ctypes.c_void_p] + [ctypes.c_int] * 5 + [_dp]
        L.orc_r2hc.argtypes = [ctypes.c_int, _dp, _dp]
        L.orc_hc2r.argtypes = [ctypes.c_int, _dp, _dp]
        L.orc_ycoord.argtypes = [ctypes.c_int, _dp, _dp, ctypes.POINTER(ctypes.c_int32),
                                 ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32),
                                 ctypes.c_double, _dp]
        _lib = L
    return _lib


def _ptr(a):
    if a is None:
        return None
    return a.ctypes.data_as(_dp)


def _f64(a, shape=None):
    if a is None:
        return None
    a = np.ascontiguousarray(a, dtype=np.float64)
    if shape is not None:
        a = a.reshape(shape)
    return a


def set_threads(n):
    lib().orc_set_threads(int(n))


def r2hc(x):
    x = _f64(x)
    out = np.empty_like(x)
    lib().orc_r2hc(len(x), _ptr(x), _ptr(out))
    return out


def hc2r(x):
    x = _f64(x)
    out = np.empty_like(x)
    lib().orc_hc2r(len(x), _ptr(x), _ptr(out))
    return out


def ycoord(section_length, section_cstret, nyc_section, stret_type, stret_option, yly):
    sl = _f64(section_length)
    sc = _f64(section_cstret)
    ny = np.ascontiguousarray(nyc_section, dtype=np.int32)
    st = np.ascontiguousarray(stret_type, dtype=np.int32)
    so = np.ascontiguousarray(stret_option, dtype=np.int32)
    out = np.zeros(int(ny.sum()) + 1)
    i32 = ctypes.POINTER(ctypes.c_int32)
    rc = lib().orc_ycoord(len(sl), _ptr(sl), _ptr(sc), ny.ctypes.data_as(i32), st.ctypes.data_as(i32),
                          so.ctypes.data_as(i32), float(yly), _ptr(out))
    if rc != 0:
        raise ValueError("orc_ycoord failed: %d" % rc)
    return out


class Oracle:
    """One oracle context = the module state of one ParaTC rank."""

    WORK = {"rhsx": 0, "rhsy": 1, "rhsz": 2, "rhsc": 3, "prsrc": 4, "phi": 5}
    HALO = {"ux": 0, "uy": 1, "uz": 2, "p": 3, "c": 4, "phi": 5}

    def __init__(self, params, yp, threads=None):
        if threads:
            set_threads(threads)
        self.params = params.copy()
        self.shape = (params.nzc, params.nyc, params.nxc)
        self.hshape = (params.nzc + 4, params.nyc + 2, params.nxc + 4)
        self._yp = _f64(yp)
        h = ctypes.c_void_p()
        rc = lib().orc_create(ctypes.byref(self.params), _ptr(self._yp), ctypes.byref(h))
        if rc != 0:
            raise ValueError("orc_create failed: %d" % rc)
        self._h = h

    def close(self):
        if self._h:
            lib().orc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_fields(self, ux, uy, uz, p, c=None, hx=None, hy=None, hz=None, hc=None):
        arrs = [_f64(a, self.shape) for a in (ux, uy, uz, p, c, hx, hy, hz, hc)]
        self._keep = arrs
        rc = lib().orc_set_fields(self._h, *[_ptr(a) for a in arrs])
        if rc != 0:
            raise ValueError("orc_set_fields failed: %d" % rc)

    def get_fields(self, names=None):
        """The interior fields; `names` selects some of them (the others are
        not copied)."""
        allnames = ["ux", "uy", "uz", "p", "c", "hx", "hy", "hz", "hc"]
        want = set(allnames if names is None else names)
        out = {}
        for n in allnames:
            if n not in want or (n in ("c", "hc") and not self.params.scalar_on):
                out[n] = None
            else:
                out[n] = np.empty(self.shape)
        lib().orc_get_fields(self._h, *[_ptr(out[n]) for n in allnames])
        return {n: v for n, v in out.items() if names is None or n in want}

    def get_halo(self, name):
        out = np.empty(self.hshape)
        rc = lib().orc_get_halo(self._h, self.HALO[name], _ptr(out))
        if rc != 0:
            raise ValueError("orc_get_halo(%s) failed" % name)
        return out

    def get_work(self, name):
        out = np.empty(self.shape)
        rc = lib().orc_get_work(self._h, self.WORK[name], _ptr(out))
        if rc != 0:
            raise ValueError("orc_get_work(%s) failed" % name)
        return out

    def set_time(self, sim_time, dt):
        lib().orc_set_time(self._h, float(sim_time), float(dt))

    def get_time(self):
        a, b, c = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        lib().orc_get_time(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c))
        return a.value, b.value, c.value

    def step(self):
        d = ParatcDiag()
        rc = lib().orc_step(self._h, ctypes.byref(d))
        return rc, d

    def substep(self, ns, dt, stop_stage=5):
        dm = ctypes.c_double()
        rc = lib().orc_substep(self._h, int(ns), float(dt), int(stop_stage), ctypes.byref(dm))
        if rc != 0:
            raise ValueError("orc_substep failed: %d" % rc)
        return dm.value

    def poisson(self, src):
        src = _f64(src, self.shape)
        phi = np.empty(self.shape)
        rc = lib().orc_poisson(self._h, _ptr(src), _ptr(phi))
        if rc != 0:
            raise ValueError("orc_poisson failed: %d" % rc)
        return phi

    def project(self):
        dm = ctypes.c_double()
        lib().orc_project(self._h, ctypes.byref(dm))
        return dm.value

    def diagnostics(self):
        d = ParatcDiag()
        lib().orc_diagnostics(self._h, ctypes.byref(d))
        return d

    def stats(self):
        """clcStat's contribution of the current fields: array [nyp, nstat]
        (SumVec/(nx nz) per row jc = 1..nyp)."""
        nst = 40 if self.params.scalar_on else 35
        out = np.zeros((self.params.nyc + 1, nst))
        rc = lib().orc_stats(self._h, _ptr(out))
        if rc != 0:
            raise RuntimeError("orc_stats rc=%d" % rc)
        return out

    def spectra(self, jlcs):
        """clcStat's 1-D spectra of the current fields (one sample, already
        times normEgy): (x spectra [nsp, nyc, nxc/2+1], z spectra [nsp, nyc,
        nzc/2+1]), nsp = 8, or 9 with the scalar."""
        p = self.params
        nsp = 9 if p.scalar_on else 8
        ex = np.zeros((nsp, p.nyc, p.nxc // 2 + 1))
        ez = np.zeros((nsp, p.nyc, p.nzc // 2 + 1))
        rc = lib().orc_spectra(self._h, int(jlcs), _ptr(ex), _ptr(ez))
        if rc != 0:
            raise RuntimeError("orc_spectra rc=%d" % rc)
        return ex, ez

    def spectra2d(self, iy):
        """clcStat's 2-D spectra of the current fields at the rows iy
        (iySpec2D, 1-based): one sample, [nsp2, nzc, nsel, nxc] (EnergySpec2D's
        Fortran order reversed), nsp2 = 5, or 6 with the scalar."""
        p = self.params
        iy = np.ascontiguousarray(iy, dtype=np.int32)
        nsp = 6 if p.scalar_on else 5
        out = np.zeros((nsp, p.nzc, len(iy), p.nxc))
        rc = lib().orc_spectra2d(self._h, len(iy), iy.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), _ptr(out))
        if rc != 0:
            raise RuntimeError("orc_spectra2d rc=%d" % rc)
        return out

    def visu(self, q, skip=(1, 1, 1), node=False):
        """dump_visu's quantity q (PARATC_VISU_* number) at the kept points
        1, 1+skip, ...: [nzo, nyo, nxo]; raises on complex lambda2 roots."""
        p = self.params
        shape = tuple(-(-a // s) for a, s in zip((p.nzc, p.nyc, p.nxc), (skip[2], skip[1], skip[0])))
        out = np.zeros(shape)
        rc = lib().orc_visu(self._h, int(q), int(skip[0]), int(skip[1]), int(skip[2]), int(bool(node)), _ptr(out))
        if rc != 0:
            raise RuntimeError("orc_visu rc=%d" % rc)
        return out

    def metric(self, name):
        buf = np.empty(max(self.params.nxc, self.params.nyc, self.params.nzc) + 8)
        n = lib().orc_metric(self._h, name.encode(), _ptr(buf), len(buf))
        if n < 0:
            raise KeyError(name)
        return buf[:n].copy()
