"""ctypes binding of libparatc_gpu.so (include/paratc.h) and a thin host-side
mirror of ParaTC's channel interface.

ChannelSystem follows m_ChannelSystem (src/m_ChannelSystem.f90): construction
is ChannelInitialize minus file IO, iterate() is ChannelIterate, and the
Poisson entry point mirrors the clcPPE procedure pointer
(src/m_Poisson.f90:16).  Every call goes through the CUDA library; there is no
CPU fallback -- a missing library or device raises.
"""
import ctypes
import os

import numpy as np

from .abi import (BATCH_GROUPED, BATCH_STREAMS, ParatcTuning, LAYOUT_INTERIOR, SCHED_NCHOICES, VISU, VISU_NAMES, ParatcIoOptions, PARATC_ERR_DIV_LIMIT, PARATC_ERR_VEL_LIMIT, PARATC_OK, ParatcDiag,
                  ParatcParams)

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libparatc_gpu.so")
_lib = None
_dp = ctypes.POINTER(ctypes.c_double)
_i32p = ctypes.POINTER(ctypes.c_int32)

EXPORTED = [
    "paratc_mesh_ycoord", "paratc_params_from_namelist", "paratc_run_options_from_namelist", "paratc_create",
    "paratc_destroy", "paratc_stream", "paratc_set_fields", "paratc_get_fields", "paratc_set_fields_device",
    "paratc_get_fields_device", "paratc_set_time", "paratc_get_time", "paratc_step", "paratc_steps",
    "paratc_substep", "paratc_substep_stage", "paratc_get_work", "paratc_poisson", "paratc_poisson_device", "paratc_poisson_device_async", "paratc_project", "paratc_diagnostics",
    "paratc_write_restart", "paratc_read_restart", "paratc_strerror", "paratc_last_error", "paratc_launch_count",
    "paratc_profile_enable", "paratc_profile_get", "paratc_profile_name", "paratc_steps_async", "paratc_last_diag",
    "paratc_poisson_noalloc", "paratc_batch_create", "paratc_batch_destroy", "paratc_batch_member",
    "paratc_batch_steps", "paratc_batch_graph_kernels", "paratc_batch_stream", "paratc_stats_reset",
    "paratc_stats_accumulate", "paratc_stats_get", "paratc_set_fields_async", "paratc_get_fields_async",
    "paratc_sync", "paratc_spectra_reset", "paratc_spectra_accumulate", "paratc_spectra_get",
    "paratc_spectra2d_setup", "paratc_spectra2d_reset", "paratc_spectra2d_accumulate", "paratc_spectra2d_get",
    "paratc_visu_name", "paratc_visu_quantity", "paratc_dump_visu", "paratc_write_xdmf",
    "paratc_io_options_from_namelist", "paratc_visu_quantity_device", "paratc_autotune", "paratc_get_schedule",
    "paratc_set_schedule", "paratc_set_precision", "paratc_get_precision", "paratc_set_wait_limit",
    "paratc_xprofile", "paratc_front_position", "paratc_poisson_refined", "paratc_poisson_refined_async",
    "paratc_autotune_all", "paratc_get_tuning", "paratc_set_tuning", "paratc_batch_set_mode",
    "paratc_batch_get_mode", "paratc_batch_step_launches", "paratc_slab_partition", "paratc_slab_create",
    "paratc_slab_destroy", "paratc_slab_counts", "paratc_slab_forward", "paratc_slab_middle", "paratc_slab_backward",
    "paratc_slab_sync", "paratc_slab_xslab", "paratc_slab_forward_peers", "paratc_slab_backward_peers",
    "paratc_ipc_get_handle", "paratc_ipc_open", "paratc_ipc_close",
]
PROF_NKERNELS = 16


class ParatcError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("paratc error %d (%s): %s" % (code, _strerror(code), msg))
        self.code = code


def load(path=None):
    """Loads the library (building it first if it is missing and nvcc exists)."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or LIB_PATH
    if not os.path.exists(path):
        from . import build as _build
        _build.build()
    L = ctypes.CDLL(path)
    L.paratc_mesh_ycoord.argtypes = [ctypes.c_int, _dp, _dp, _i32p, _i32p, _i32p, ctypes.c_double, _dp]
    L.paratc_params_from_namelist.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(ParatcParams), _dp,
                                              ctypes.c_int]
    L.paratc_create.argtypes = [ctypes.POINTER(ParatcParams), _dp, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
    L.paratc_destroy.argtypes = [ctypes.c_void_p]
    L.paratc_stream.argtypes = [ctypes.c_void_p]
    L.paratc_stream.restype = ctypes.c_void_p
    L.paratc_set_fields.argtypes = [ctypes.c_void_p] + [_dp] * 9 + [ctypes.c_int]
    L.paratc_get_fields.argtypes = [ctypes.c_void_p] + [_dp] * 9 + [ctypes.c_int]
    L.paratc_set_fields_async.argtypes = [ctypes.c_void_p] + [_dp] * 9 + [ctypes.c_int]
    L.paratc_get_fields_async.argtypes = [ctypes.c_void_p] + [_dp] * 9 + [ctypes.c_int]
    L.paratc_sync.argtypes = [ctypes.c_void_p]
    L.paratc_set_fields_device.argtypes = [ctypes.c_void_p] + [ctypes.c_void_p] * 9
    L.paratc_get_fields_device.argtypes = [ctypes.c_void_p] + [ctypes.c_void_p] * 9
    L.paratc_set_time.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double]
    L.paratc_visu_name.argtypes = [ctypes.c_int]
    L.paratc_visu_name.restype = ctypes.c_char_p
    L.paratc_visu_quantity.argtypes = [ctypes.c_void_p] + [ctypes.c_int] * 5 + [_dp, ctypes.POINTER(ctypes.c_int64)]
    L.paratc_visu_quantity_device.argtypes = [ctypes.c_void_p] + [ctypes.c_int] * 5 + [ctypes.c_void_p] * 2
    L.paratc_autotune.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int), _dp]
    L.paratc_get_schedule.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]
    L.paratc_set_schedule.argtypes = [ctypes.c_void_p, ctypes.c_int]
    L.paratc_set_precision.argtypes = [ctypes.c_void_p, ctypes.c_int]
    L.paratc_get_precision.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]
    L.paratc_set_wait_limit.argtypes = [ctypes.c_void_p, ctypes.c_longlong]
    L.paratc_xprofile.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp]
    L.paratc_autotune_all.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_char_p, ctypes.POINTER(ParatcTuning)]
    L.paratc_get_tuning.argtypes = [ctypes.c_void_p, ctypes.POINTER(ParatcTuning)]
    L.paratc_set_tuning.argtypes = [ctypes.c_void_p, ctypes.POINTER(ParatcTuning)]
    L.paratc_poisson_refined.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double,
                                         ctypes.c_int, ctypes.POINTER(ctypes.c_int), _dp]
    L.paratc_poisson_refined_async.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
    L.paratc_front_position.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, _dp]
    L.paratc_dump_visu.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_char_p] + [ctypes.c_int] * 7
    L.paratc_write_xdmf.argtypes = [ctypes.POINTER(ParatcParams), _dp, ctypes.c_char_p, ctypes.c_char_p] + \
        [ctypes.c_int] * 6
    L.paratc_io_options_from_namelist.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(ParatcIoOptions)]
    L.paratc_get_time.argtypes = [ctypes.c_void_p, _dp, _dp]
    L.paratc_step.argtypes = [ctypes.c_void_p, ctypes.POINTER(ParatcDiag)]
    L.paratc_steps.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ParatcDiag)]
    L.paratc_substep.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, _dp]
    L.paratc_substep_stage.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_int, _dp]
    L.paratc_get_work.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp]
    L.paratc_poisson.argtypes = [ctypes.c_void_p, _dp, _dp]
    L.paratc_poisson_device.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    L.paratc_poisson_device_async.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    L.paratc_project.argtypes = [ctypes.c_void_p, _dp]
    L.paratc_diagnostics.argtypes = [ctypes.c_void_p, ctypes.POINTER(ParatcDiag)]
    L.paratc_write_restart.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int]
    L.paratc_read_restart.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
    L.paratc_strerror.argtypes = [ctypes.c_int]
    L.paratc_strerror.restype = ctypes.c_char_p
    L.paratc_last_error.argtypes = [ctypes.c_void_p]
    L.paratc_last_error.restype = ctypes.c_char_p
    L.paratc_launch_count.argtypes = [ctypes.c_void_p]
    L.paratc_launch_count.restype = ctypes.c_int64
    L.paratc_poisson_noalloc.argtypes = [ctypes.POINTER(ParatcParams), _dp, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_void_p]
    L.paratc_steps_async.argtypes = [ctypes.c_void_p, ctypes.c_int]
    L.paratc_last_diag.argtypes = [ctypes.c_void_p, ctypes.POINTER(ParatcDiag)]
    L.paratc_profile_enable.argtypes = [ctypes.c_void_p, ctypes.c_int]
    L.paratc_profile_get.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, ctypes.POINTER(ctypes.c_int64)]
    L.paratc_profile_name.argtypes = [ctypes.c_int]
    L.paratc_profile_name.restype = ctypes.c_char_p
    L.paratc_batch_create.argtypes = [ctypes.c_int, ctypes.POINTER(ParatcParams), ctypes.POINTER(_dp), ctypes.c_int,
                                      ctypes.POINTER(ctypes.c_void_p)]
    L.paratc_batch_destroy.argtypes = [ctypes.c_void_p]
    L.paratc_batch_member.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
    L.paratc_batch_steps.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ParatcDiag)]
    L.paratc_batch_graph_kernels.argtypes = [ctypes.c_void_p]
    L.paratc_batch_graph_kernels.restype = ctypes.c_int64
    L.paratc_stats_reset.argtypes = [ctypes.c_void_p]
    L.paratc_stats_accumulate.argtypes = [ctypes.c_void_p]
    L.paratc_stats_get.argtypes = [ctypes.c_void_p, _dp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                   _dp]
    L.paratc_batch_stream.argtypes = [ctypes.c_void_p]
    L.paratc_batch_stream.restype = ctypes.c_void_p
    L.paratc_batch_set_mode.argtypes = [ctypes.c_void_p, ctypes.c_int]
    L.paratc_batch_get_mode.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]
    L.paratc_batch_step_launches.argtypes = [ctypes.c_void_p]
    L.paratc_batch_step_launches.restype = ctypes.c_int64
    L.paratc_slab_partition.argtypes = [ctypes.c_int] * 3 + [_i32p] * 2
    L.paratc_slab_create.argtypes = [ctypes.POINTER(ParatcParams), _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                     ctypes.POINTER(ctypes.c_void_p)]
    L.paratc_slab_destroy.argtypes = [ctypes.c_void_p]
    L.paratc_slab_counts.argtypes = [ctypes.c_void_p] + [ctypes.POINTER(ctypes.c_int64)] * 2
    L.paratc_slab_forward.argtypes = [ctypes.c_void_p] * 4
    L.paratc_slab_middle.argtypes = [ctypes.c_void_p] * 3
    L.paratc_slab_backward.argtypes = [ctypes.c_void_p] * 4
    L.paratc_slab_sync.argtypes = [ctypes.c_void_p] * 2
    L.paratc_slab_xslab.argtypes = [ctypes.c_void_p]
    L.paratc_slab_xslab.restype = ctypes.c_void_p
    L.paratc_slab_forward_peers.argtypes = [ctypes.c_void_p] * 4
    L.paratc_slab_backward_peers.argtypes = [ctypes.c_void_p] * 4
    L.paratc_ipc_get_handle.argtypes = [ctypes.c_void_p] * 2
    L.paratc_ipc_open.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]
    L.paratc_ipc_close.argtypes = [ctypes.c_void_p]
    L.paratc_spectra_reset.argtypes = [ctypes.c_void_p]
    L.paratc_spectra_accumulate.argtypes = [ctypes.c_void_p, ctypes.c_int]
    L.paratc_spectra_get.argtypes = [ctypes.c_void_p, _dp, _dp, ctypes.POINTER(ctypes.c_int),
                                     ctypes.POINTER(ctypes.c_int)]
    L.paratc_spectra2d_setup.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    L.paratc_spectra2d_reset.argtypes = [ctypes.c_void_p]
    L.paratc_spectra2d_accumulate.argtypes = [ctypes.c_void_p]
    L.paratc_spectra2d_get.argtypes = [ctypes.c_void_p, _dp, ctypes.POINTER(ctypes.c_int),
                                       ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
    _lib = L
    return L


def _strerror(code):
    try:
        return load().paratc_strerror(int(code)).decode()
    except Exception:
        return "?"


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_dp)


def _f64(a, shape):
    if a is None:
        return None
    return np.ascontiguousarray(a, dtype=np.float64).reshape(shape)


def mesh_ycoord(mesh, yly):
    """yp(1..nyp) for a cases.Mesh (clcYcoord, src/m_MeshAndMetries.f90:340-408)."""
    L = load()
    sl = np.ascontiguousarray(mesh.section_length, dtype=np.float64)
    cs = np.ascontiguousarray(mesh.section_cstret, dtype=np.float64)
    ny = np.ascontiguousarray(mesh.nyc_section, dtype=np.int32)
    st = np.ascontiguousarray(mesh.stret_type, dtype=np.int32)
    so = np.ascontiguousarray(mesh.stret_option, dtype=np.int32)
    out = np.zeros(int(ny.sum()) + 1)
    rc = L.paratc_mesh_ycoord(len(sl), _ptr(sl), _ptr(cs), ny.ctypes.data_as(_i32p), st.ctypes.data_as(_i32p),
                              so.ctypes.data_as(_i32p), float(yly), _ptr(out))
    if rc != PARATC_OK:
        raise ParatcError(rc, "paratc_mesh_ycoord")
    return out


def params_from_namelist(path, scalar_on=False, nyp_cap=8192):
    L = load()
    p = ParatcParams()
    yp = np.zeros(nyp_cap)
    rc = L.paratc_params_from_namelist(path.encode(), int(bool(scalar_on)), ctypes.byref(p), _ptr(yp), nyp_cap)
    if rc != PARATC_OK:
        raise ParatcError(rc, "paratc_params_from_namelist(%s)" % path)
    return p, yp[: p.nyc + 1].copy()


def io_options_from_namelist(path, scalar_on=False):
    """&IO_Options, &SpectraOptions (+ &Spectra2DOpt, &SaveScalarOption) and
    the output cadences of &BasicParam."""
    o = ParatcIoOptions()
    rc = load().paratc_io_options_from_namelist(path.encode(), int(bool(scalar_on)), ctypes.byref(o))
    if rc != PARATC_OK:
        raise ParatcError(rc, "paratc_io_options_from_namelist(%s)" % path)
    return o


def write_xdmf(params, yp, res_dir, run_name, ifirst, ilast, save_visu, save_mask, xdmf_set_type=0, single=False):
    """InitVisu's XDMF index res_dir + "VisuFor" + run_name + ".xmf"."""
    yp = np.ascontiguousarray(yp, dtype=np.float64)
    p = params.copy()
    rc = load().paratc_write_xdmf(ctypes.byref(p), _ptr(yp), res_dir.encode(), run_name.encode(), int(ifirst),
                                  int(ilast), int(save_visu), int(save_mask), int(xdmf_set_type), int(bool(single)))
    if rc != PARATC_OK:
        raise ParatcError(rc, "paratc_write_xdmf")


def visu_mask(*names):
    m = 0
    for n in names:
        m |= 1 << VISU[n]
    return m


class ChannelSystem:
    """One B200 context: the module state of a ParaTC run on one GPU."""

    FIELDS = ("ux", "uy", "uz", "p", "c", "hx", "hy", "hz", "hc")

    def __init__(self, params, yp, device=-1, _borrowed=None):
        L = load()
        self.params = params.copy()
        self.shape = (params.nzc, params.nyc, params.nxc)
        self._yp = np.ascontiguousarray(yp, dtype=np.float64)
        self._L = L
        self._owner = _borrowed is None
        if _borrowed is not None:  # a member of a BatchSystem, destroyed with it
            self._h = _borrowed
            return
        h = ctypes.c_void_p()
        rc = L.paratc_create(ctypes.byref(self.params), _ptr(self._yp), int(device), ctypes.byref(h))
        if rc != PARATC_OK:
            raise ParatcError(rc, "paratc_create")
        self._h = h

    # -- lifetime
    def close(self):
        if getattr(self, "_h", None):
            if self._owner:
                self._L.paratc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc, what):
        if rc != PARATC_OK:
            raise ParatcError(rc, "%s: %s" % (what, self._L.paratc_last_error(self._h).decode()))

    @property
    def handle(self):
        return self._h

    @property
    def stream(self):
        return self._L.paratc_stream(self._h)

    @property
    def launches(self):
        return int(self._L.paratc_launch_count(self._h))

    # -- state
    def set_fields(self, ux, uy, uz, p, c=None, hx=None, hy=None, hz=None, hc=None, layout=LAYOUT_INTERIOR):
        shape = self.shape if layout == LAYOUT_INTERIOR else (self.params.nzc + 4, self.params.nyc + 2, self.params.nxc + 4)
        arrs = [_f64(a, shape) for a in (ux, uy, uz, p, c, hx, hy, hz, hc)]
        self._check(self._L.paratc_set_fields(self._h, *[_ptr(a) for a in arrs], int(layout)), "paratc_set_fields")

    def get_fields(self, names=None, layout=LAYOUT_INTERIOR):
        names = names or self.FIELDS
        shape = self.shape if layout == LAYOUT_INTERIOR else (self.params.nzc + 4, self.params.nyc + 2, self.params.nxc + 4)
        out = {}
        ptrs = []
        for n in self.FIELDS:
            if n in names and (n not in ("c", "hc") or self.params.scalar_on):
                out[n] = np.zeros(shape)
                ptrs.append(_ptr(out[n]))
            else:
                ptrs.append(None)
        self._check(self._L.paratc_get_fields(self._h, *ptrs, int(layout)), "paratc_get_fields")
        return out

    def get_fields_into(self, out, layout=LAYOUT_INTERIOR):
        """Copies the fields named in `out` into its (C-contiguous float64) arrays."""
        ptrs = [_ptr(out[n]) if n in out and out[n] is not None else None for n in self.FIELDS]
        self._check(self._L.paratc_get_fields(self._h, *ptrs, int(layout)), "paratc_get_fields")

    def set_fields_async(self, ux, uy, uz, p, c=None, hx=None, hy=None, hz=None, hc=None):
        """Queues the copies; the (C-contiguous float64, ideally pinned) arrays
        must stay alive until sync()."""
        arrs = [None if a is None else a for a in (ux, uy, uz, p, c, hx, hy, hz, hc)]
        for a in arrs:
            if a is not None and not (a.flags.c_contiguous and a.dtype == np.float64 and a.shape == self.shape):
                raise ValueError("set_fields_async needs C-contiguous float64 arrays of shape %s" % (self.shape,))
        self._check(self._L.paratc_set_fields_async(self._h, *[_ptr(a) for a in arrs], LAYOUT_INTERIOR),
                    "paratc_set_fields_async")

    def get_fields_into_async(self, out):
        ptrs = [_ptr(out[n]) if n in out and out[n] is not None else None for n in self.FIELDS]
        self._check(self._L.paratc_get_fields_async(self._h, *ptrs, LAYOUT_INTERIOR), "paratc_get_fields_async")

    def sync(self):
        self._check(self._L.paratc_sync(self._h), "paratc_sync")

    def set_time(self, sim_time, dt):
        self._check(self._L.paratc_set_time(self._h, float(sim_time), float(dt)), "paratc_set_time")

    def get_time(self):
        a, b = ctypes.c_double(), ctypes.c_double()
        self._check(self._L.paratc_get_time(self._h, ctypes.byref(a), ctypes.byref(b)), "paratc_get_time")
        return a.value, b.value

    # -- hot path
    def iterate(self, nsteps=1, raise_on_guard=True):
        """ChannelIterate nsteps times; returns the last step's ParatcDiag."""
        d = ParatcDiag()
        rc = self._L.paratc_steps(self._h, int(nsteps), ctypes.byref(d))
        if rc in (PARATC_ERR_DIV_LIMIT, PARATC_ERR_VEL_LIMIT) and not raise_on_guard:
            return d
        self._check(rc, "paratc_steps")
        return d

    def iterate_async(self, nsteps=1):
        """Enqueues nsteps steps on the context stream without waiting."""
        self._check(self._L.paratc_steps_async(self._h, int(nsteps)), "paratc_steps_async")

    def last_diag(self, raise_on_guard=True):
        d = ParatcDiag()
        rc = self._L.paratc_last_diag(self._h, ctypes.byref(d))
        if rc in (PARATC_ERR_DIV_LIMIT, PARATC_ERR_VEL_LIMIT) and not raise_on_guard:
            return d
        self._check(rc, "paratc_last_diag")
        return d

    def substep(self, ns, dt):
        dm = ctypes.c_double()
        self._check(self._L.paratc_substep(self._h, int(ns), float(dt), ctypes.byref(dm)), "paratc_substep")
        return dm.value

    WORK = {"rhsx": 0, "rhsy": 1, "rhsz": 2, "rhsc": 3, "prsrc": 4, "phi": 5}

    def substep_stage(self, ns, dt, stop_stage):
        dm = ctypes.c_double()
        self._check(self._L.paratc_substep_stage(self._h, int(ns), float(dt), int(stop_stage), ctypes.byref(dm)),
                    "paratc_substep_stage")
        return dm.value

    def get_work(self, name):
        out = np.empty(self.shape)
        self._check(self._L.paratc_get_work(self._h, self.WORK[name], _ptr(out)), "paratc_get_work")
        return out

    def poisson(self, src):
        src = _f64(src, self.shape)
        phi = np.empty(self.shape)
        self._check(self._L.paratc_poisson(self._h, _ptr(src), _ptr(phi)), "paratc_poisson")
        return phi

    def poisson_device(self, d_src_ptr, d_phi_ptr):
        self._check(self._L.paratc_poisson_device(self._h, ctypes.c_void_p(d_src_ptr), ctypes.c_void_p(d_phi_ptr)),
                    "paratc_poisson_device")

    def poisson_device_async(self, d_src_ptr, d_phi_ptr):
        self._check(self._L.paratc_poisson_device_async(self._h, ctypes.c_void_p(d_src_ptr), ctypes.c_void_p(d_phi_ptr)),
                    "paratc_poisson_device_async")

    def poisson_refined(self, d_src_ptr, d_phi_ptr, rtol=1e-12, max_corr=4):
        """FP32 solves with FP64 iterative refinement (device pointers);
        returns (corrections, final max|r| / max|src|)."""
        n, r = ctypes.c_int(), ctypes.c_double()
        self._check(self._L.paratc_poisson_refined(self._h, ctypes.c_void_p(d_src_ptr), ctypes.c_void_p(d_phi_ptr),
                                                   float(rtol), int(max_corr), ctypes.byref(n), ctypes.byref(r)),
                    "paratc_poisson_refined")
        return n.value, r.value

    def poisson_refined_async(self, d_src_ptr, d_phi_ptr, ncorr):
        self._check(self._L.paratc_poisson_refined_async(self._h, ctypes.c_void_p(d_src_ptr),
                                                         ctypes.c_void_p(d_phi_ptr), int(ncorr)),
                    "paratc_poisson_refined_async")

    # -- statistics (clcStat)
    def stats_reset(self):
        self._check(self._L.paratc_stats_reset(self._h), "paratc_stats_reset")

    def stats_accumulate(self):
        self._check(self._L.paratc_stats_accumulate(self._h), "paratc_stats_accumulate")

    def stats_get(self):
        """(SumStat [nyp, nstat], nfstime, PrGradsum)."""
        nst = 40 if self.params.scalar_on else 35
        out = np.zeros((self.params.nyc + 1, nst))
        n, nf, pg = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        self._check(self._L.paratc_stats_get(self._h, _ptr(out), ctypes.byref(n), ctypes.byref(nf), ctypes.byref(pg)),
                    "paratc_stats_get")
        return out, nf.value, pg.value

    # -- 1-D spectra (clcStat's spectra section)
    def spectra_reset(self):
        self._check(self._L.paratc_spectra_reset(self._h), "paratc_spectra_reset")

    def spectra_accumulate(self, jlcs):
        self._check(self._L.paratc_spectra_accumulate(self._h, int(jlcs)), "paratc_spectra_accumulate")

    def spectra_get(self):
        """(x spectra [nsp, nyc, nxc/2+1], z spectra [nsp, nyc, nzc/2+1],
        nSpectime): the sums of EgyX*normEgy and EgyZ*normEgy over the samples."""
        p = self.params
        nsp = 9 if p.scalar_on else 8
        ex = np.zeros((nsp, p.nyc, p.nxc // 2 + 1))
        ez = np.zeros((nsp, p.nyc, p.nzc // 2 + 1))
        n, ns = ctypes.c_int(), ctypes.c_int()
        self._check(self._L.paratc_spectra_get(self._h, _ptr(ex), _ptr(ez), ctypes.byref(n), ctypes.byref(ns)),
                    "paratc_spectra_get")
        return ex, ez, ns.value

    # -- 2-D spectra at the rows iySpec2D
    def spectra2d_setup(self, iy):
        iy = np.ascontiguousarray(iy, dtype=np.int32)
        self._check(self._L.paratc_spectra2d_setup(self._h, len(iy), iy.ctypes.data_as(ctypes.POINTER(ctypes.c_int))),
                    "paratc_spectra2d_setup")

    def spectra2d_reset(self):
        self._check(self._L.paratc_spectra2d_reset(self._h), "paratc_spectra2d_reset")

    def spectra2d_accumulate(self):
        self._check(self._L.paratc_spectra2d_accumulate(self._h), "paratc_spectra2d_accumulate")

    def spectra2d_get(self):
        """(EnergySpec2D sums [nsp2, nzc, nsel, nxc], nSpectime)."""
        p = self.params
        nsp, nsel, ns = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self._check(self._L.paratc_spectra2d_get(self._h, None, ctypes.byref(nsp), ctypes.byref(nsel),
                                                 ctypes.byref(ns)), "paratc_spectra2d_get")
        out = np.zeros((nsp.value, p.nzc, nsel.value, p.nxc))
        self._check(self._L.paratc_spectra2d_get(self._h, _ptr(out), None, None, None), "paratc_spectra2d_get")
        return out, ns.value

    # -- visualisation dumps (dump_visu)
    def visu_quantity(self, name, skip=(1, 1, 1), node=False):
        """dump_visu's quantity `name` at the kept points, [nzo, nyo, nxo]."""
        q = VISU[name] if isinstance(name, str) else int(name)
        n = ctypes.c_int64()
        self._check(self._L.paratc_visu_quantity(self._h, q, skip[0], skip[1], skip[2], int(bool(node)), None,
                                                 ctypes.byref(n)), "paratc_visu_quantity")
        p = self.params
        shape = tuple(-(-a // s) for a, s in zip((p.nzc, p.nyc, p.nxc), (skip[2], skip[1], skip[0])))
        out = np.zeros(shape)
        assert out.size == n.value
        self._check(self._L.paratc_visu_quantity(self._h, q, skip[0], skip[1], skip[2], int(bool(node)), _ptr(out),
                                                 None), "paratc_visu_quantity")
        return out

    # -- precision: "fp64" (default), "mixed" (FP32 right-hand side) or
    #    "fp32" (FP32 storage of everything but the pressure)
    @property
    def precision(self):
        v = ctypes.c_int()
        self._check(self._L.paratc_get_precision(self._h, ctypes.byref(v)), "paratc_get_precision")
        return ("fp64", "mixed", "fp32")[v.value]

    @precision.setter
    def precision(self, name):
        self._check(self._L.paratc_set_precision(self._h, {"fp64": 0, "mixed": 1, "fp32": 2}[name]),
                    "paratc_set_precision")

    def set_wait_limit(self, polls):
        """Poll limit of the TMA-fed kernels' pipeline waits (None or < 0:
        the default); a wait that runs out makes the next synchronising call
        raise PARATC_ERR_TIMEOUT."""
        self._check(self._L.paratc_set_wait_limit(self._h, -1 if polls is None else int(polls)),
                    "paratc_set_wait_limit")

    # -- Poisson schedule (InitPoissonSolver's auto-tuning)
    def autotune(self, nrep=15):
        """Times every supported schedule and keeps the fastest: (choice, ms
        for nrep solves per choice, -1 where unsupported)."""
        ch = ctypes.c_int()
        t = np.zeros(SCHED_NCHOICES)
        self._check(self._L.paratc_autotune(self._h, int(nrep), ctypes.byref(ch), _ptr(t)), "paratc_autotune")
        return ch.value, t

    def autotune_all(self, nrep=5, cache_path=None):
        """Poisson schedule, then the right-hand-side and Helmholtz launch
        shapes by whole steps; picks cached in cache_path (JSON) when given.
        Returns the ParatcTuning applied."""
        t = ParatcTuning()
        self._check(self._L.paratc_autotune_all(self._h, int(nrep), None if cache_path is None else cache_path.encode(),
                                                ctypes.byref(t)), "paratc_autotune_all")
        return t

    @property
    def tuning(self):
        t = ParatcTuning()
        self._check(self._L.paratc_get_tuning(self._h, ctypes.byref(t)), "paratc_get_tuning")
        return t

    @tuning.setter
    def tuning(self, t):
        self._check(self._L.paratc_set_tuning(self._h, ctypes.byref(t)), "paratc_set_tuning")

    @property
    def schedule(self):
        ch = ctypes.c_int()
        self._check(self._L.paratc_get_schedule(self._h, ctypes.byref(ch)), "paratc_get_schedule")
        return ch.value

    @schedule.setter
    def schedule(self, choice):
        self._check(self._L.paratc_set_schedule(self._h, int(choice)), "paratc_set_schedule")

    def visu_quantity_device_async(self, name, d_out, skip=(1, 1, 1), node=False, d_nbad=None):
        """Into a device pointer (int), asynchronous on the context's stream."""
        q = VISU[name] if isinstance(name, str) else int(name)
        self._check(self._L.paratc_visu_quantity_device(self._h, q, skip[0], skip[1], skip[2], int(bool(node)),
                                                        ctypes.c_void_p(d_out),
                                                        None if d_nbad is None else ctypes.c_void_p(d_nbad)),
                    "paratc_visu_quantity_device")

    def dump_visu(self, res_dir, run_name, ntime, save_mask, skip=(1, 1, 1), node=False, single=False):
        self._check(self._L.paratc_dump_visu(self._h, res_dir.encode(), run_name.encode(), int(ntime), int(save_mask),
                                             skip[0], skip[1], skip[2], int(bool(node)), int(bool(single))),
                    "paratc_dump_visu")

    def xprofile(self, name="c"):
        """The field averaged over the depth (dyp weights) and the span, one
        value per x cell."""
        out = np.zeros(self.params.nxc)
        q = {"ux": 0, "uy": 1, "uz": 2, "p": 3, "c": 4}[name]
        self._check(self._L.paratc_xprofile(self._h, q, _ptr(out)), "paratc_xprofile")
        return out

    def front_position(self, x_from=1.0, level=0.5):
        """x where the depth-averaged scalar first drops below `level` to the
        right of x_from (-1 if nowhere)."""
        x = ctypes.c_double()
        self._check(self._L.paratc_front_position(self._h, float(x_from), float(level), ctypes.byref(x)),
                    "paratc_front_position")
        return x.value

    def project(self):
        dm = ctypes.c_double()
        self._check(self._L.paratc_project(self._h, ctypes.byref(dm)), "paratc_project")
        return dm.value

    def diagnostics(self):
        d = ParatcDiag()
        self._check(self._L.paratc_diagnostics(self._h, ctypes.byref(d)), "paratc_diagnostics")
        return d

    def profile(self, on):
        self._check(self._L.paratc_profile_enable(self._h, int(bool(on))), "paratc_profile_enable")

    def profile_read(self):
        """{kernel class: (total ms, launches)} since profile(True)."""
        out = {}
        for k in range(PROF_NKERNELS):
            ms = ctypes.c_double()
            n = ctypes.c_int64()
            self._check(self._L.paratc_profile_get(self._h, k, ctypes.byref(ms), ctypes.byref(n)), "paratc_profile_get")
            if n.value:
                out[self._L.paratc_profile_name(k).decode()] = (ms.value, n.value)
        return out

    def write_restart(self, path, with_hist=False):
        self._check(self._L.paratc_write_restart(self._h, path.encode(), int(bool(with_hist))), "paratc_write_restart")

    def read_restart(self, path):
        self._check(self._L.paratc_read_restart(self._h, path.encode()), "paratc_read_restart")


class BatchSystem:
    """An ensemble of independent contexts that advance together
    (paratc_batch_*): members[i] is a ChannelSystem view of member i."""

    def __init__(self, params_list, yp_list, device=-1):
        L = load()
        n = len(params_list)
        self._L = L
        self._params = (ParatcParams * n)(*[p.copy() for p in params_list])
        self._yps = [np.ascontiguousarray(y, dtype=np.float64) for y in yp_list]
        ptrs = (_dp * n)(*[_ptr(y) for y in self._yps])
        h = ctypes.c_void_p()
        rc = L.paratc_batch_create(n, self._params, ptrs, int(device), ctypes.byref(h))
        if rc != PARATC_OK:
            raise ParatcError(rc, "paratc_batch_create")
        self._h = h
        self.members = []
        for i in range(n):
            m = ctypes.c_void_p()
            rc = L.paratc_batch_member(h, i, ctypes.byref(m))
            if rc != PARATC_OK:
                raise ParatcError(rc, "paratc_batch_member")
            self.members.append(ChannelSystem(params_list[i], yp_list[i], _borrowed=m))

    def __len__(self):
        return len(self.members)

    def close(self):
        if getattr(self, "_h", None):
            for m in self.members:
                m.close()
            self._L.paratc_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def iterate(self, nsteps=1, use_graph=True, raise_on_guard=True):
        """nsteps ChannelIterate steps of every member; returns the members'
        last-step diagnostics."""
        n = len(self.members)
        d = (ParatcDiag * n)()
        rc = self._L.paratc_batch_steps(self._h, int(nsteps), int(bool(use_graph)), d)
        if rc != PARATC_OK and (raise_on_guard or rc not in (PARATC_ERR_DIV_LIMIT, PARATC_ERR_VEL_LIMIT)):
            raise ParatcError(rc, "paratc_batch_steps")
        return list(d)

    @property
    def graph_kernels(self):
        return int(self._L.paratc_batch_graph_kernels(self._h))

    @property
    def mode(self):
        """'streams' (every member launches its own kernels on its own
        stream) or 'grouped' (one launch per kernel instantiation over the
        members, paratc_batch_set_mode)."""
        v = ctypes.c_int()
        rc = self._L.paratc_batch_get_mode(self._h, ctypes.byref(v))
        if rc != PARATC_OK:
            raise ParatcError(rc, "paratc_batch_get_mode")
        return {BATCH_STREAMS: "streams", BATCH_GROUPED: "grouped"}[v.value]

    @mode.setter
    def mode(self, name):
        v = {"streams": BATCH_STREAMS, "grouped": BATCH_GROUPED}[name]
        rc = self._L.paratc_batch_set_mode(self._h, v)
        if rc != PARATC_OK:
            raise ParatcError(rc, "paratc_batch_set_mode")

    @property
    def step_launches(self):
        """Kernel launches of one steady step in the batch's mode."""
        return int(self._L.paratc_batch_step_launches(self._h))

    @property
    def stream(self):
        return self._L.paratc_batch_stream(self._h)

