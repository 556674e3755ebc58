"""ctypes mirror of the structs and constants in include/paratc.h.

Plain data only: importing this module loads no shared library.
"""
import ctypes

PARATC_OK = 0
PARATC_ERR_BAD_ARG = -1
PARATC_ERR_OOM = -2
PARATC_ERR_CUDA = -3
PARATC_ERR_NONFINITE = -4
PARATC_ERR_DIV_LIMIT = -5
PARATC_ERR_VEL_LIMIT = -6
PARATC_ERR_TIMEOUT = -7
PARATC_ERR_IO = -8
PARATC_ERR_NO_DEVICE = -9
PARATC_ERR_NUMERIC = -10

FT_CH = 1
FT_HC = 2
AB2, RK2, RK3 = 1, 2, 3
LAYOUT_INTERIOR = 0
LAYOUT_HALO = 1

# Poisson schedule choices (PARATC_SCHED_NCHOICES of include/paratc.h)
SCHED_NCHOICES = 12

# launch modes of an ensemble (PARATC_BATCH_*)
BATCH_STREAMS = 0
BATCH_GROUPED = 1

# dump_visu quantities (PARATC_VISU_*)
VISU_NAMES = ("ux", "uy", "uz", "pr", "wx", "wy", "wz", "wMag", "Q", "lamda2", "scalar")
VISU = {n: q for q, n in enumerate(VISU_NAMES)}
MAX_SPEC2D = 64

_d3 = ctypes.c_double * 3
_d6 = ctypes.c_double * 6


class ParatcParams(ctypes.Structure):
    """struct paratc_params (include/paratc.h)."""

    _fields_ = [
        ("nxc", ctypes.c_int32), ("nyc", ctypes.c_int32), ("nzc", ctypes.c_int32),
        ("flow_type", ctypes.c_int32), ("ischeme", ctypes.c_int32), ("icfl", ctypes.c_int32),
        ("is_ux_const", ctypes.c_int32), ("scalar_on", ctypes.c_int32),
        ("xlx", ctypes.c_double), ("yly", ctypes.c_double), ("zlz", ctypes.c_double),
        ("xnu", ctypes.c_double), ("ubulk", ctypes.c_double), ("ucrf", ctypes.c_double),
        ("dt_max", ctypes.c_double), ("cflc", ctypes.c_double),
        ("gravity", _d3), ("ux_bc", _d6), ("uy_bc", _d6), ("uz_bc", _d6),
        ("vel_limit", ctypes.c_double), ("div_limit", ctypes.c_double),
        ("sdiff", ctypes.c_double), ("gravity_eff_vec", _d3), ("falling_vel_vec", _d3),
        ("scalar_bc_option", ctypes.c_int32 * 2), ("scalar_bc_values", ctypes.c_double * 4),
        ("scalar_init_value", ctypes.c_double),
    ]

    def copy(self):
        out = ParatcParams()
        ctypes.pointer(out)[0] = self
        return out

    def as_dict(self):
        d = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            d[name] = list(v) if hasattr(v, "__len__") else v
        return d


class ParatcDiag(ctypes.Structure):
    """struct paratc_diag (include/paratc.h)."""

    _fields_ = [
        ("dt", ctypes.c_double), ("cfl", ctypes.c_double), ("sim_time", ctypes.c_double),
        ("divmax_src", ctypes.c_double), ("divmax", ctypes.c_double), ("vmax", _d3),
        ("pr_grad_aver", ctypes.c_double), ("ux_mean", ctypes.c_double),
        ("sc_mean", ctypes.c_double), ("sc2_mean", ctypes.c_double),
    ]

    def as_dict(self):
        return {
            "dt": self.dt, "cfl": self.cfl, "sim_time": self.sim_time,
            "divmax_src": self.divmax_src, "divmax": self.divmax, "vmax": list(self.vmax),
            "pr_grad_aver": self.pr_grad_aver, "ux_mean": self.ux_mean,
            "sc_mean": self.sc_mean, "sc2_mean": self.sc2_mean,
        }


class ParatcIoOptions(ctypes.Structure):
    """struct paratc_io_options (include/paratc.h)."""

    _fields_ = [
        ("ivstats", ctypes.c_int32), ("save_stat", ctypes.c_int32), ("save_visu", ctypes.c_int32),
        ("iskip", ctypes.c_int32), ("jskip", ctypes.c_int32), ("kskip", ctypes.c_int32),
        ("xdmf_set_type", ctypes.c_int32), ("save_mask", ctypes.c_int32),
        ("write_hist_old", ctypes.c_int32), ("read_hist_old", ctypes.c_int32),
        ("clc_spectra1d", ctypes.c_int32), ("iv_spec", ctypes.c_int32), ("j_for_lcs", ctypes.c_int32),
        ("clc_spectra2d", ctypes.c_int32), ("ny_spec2d", ctypes.c_int32),
        ("iy_spec2d", ctypes.c_int32 * MAX_SPEC2D),
    ]


class ParatcTuning(ctypes.Structure):
    """paratc_tuning of include/paratc.h."""
    _fields_ = [("schedule", ctypes.c_int32), ("rhs_var", ctypes.c_int32), ("helm_var", ctypes.c_int32),
                ("from_cache", ctypes.c_int32), ("step_ms", ctypes.c_double)]
