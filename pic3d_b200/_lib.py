"""ctypes binding of libpic3d_b200.so (include/pic3d_gpu.h).

The library is built in-tree by ``pic3d_b200.build``.  There is no CPU
fallback: if the library cannot be loaded, importing the binding raises.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# PIC3D_LIBRARY may point at another build of the same sources (tuning builds)
LIB_PATH = os.environ.get("PIC3D_LIBRARY", os.path.join(HERE, "libpic3d_b200.so"))

(PIC_OK, PIC_EINVAL, PIC_ENOMEM, PIC_EOOB, PIC_ENAN, PIC_ETIMEOUT, PIC_ECUDA, PIC_EOVERFLOW, PIC_ERANGE,
 PIC_ENOCONV) = range(10)
STATUS_NAMES = {0: "PIC_OK", 1: "PIC_EINVAL", 2: "PIC_ENOMEM", 3: "PIC_EOOB", 4: "PIC_ENAN", 5: "PIC_ETIMEOUT",
                6: "PIC_ECUDA", 7: "PIC_EOVERFLOW", 8: "PIC_ERANGE", 9: "PIC_ENOCONV"}
ARRAYS = ["ex", "ey", "ez", "bx", "by", "bz", "jx", "jy", "jz", "rho0", "rho1"]
NDIAG = 6
NPOISSON = 4

_I32, _I64, _D = ctypes.c_int32, ctypes.c_int64, ctypes.c_double


class PicParams(ctypes.Structure):
    _fields_ = [
        ("local_xcells", _I32), ("local_ycells", _I32), ("local_zcells", _I32), ("mem", _I32),
        ("rank_period", _I32 * 3), ("laser_polarization", _I32),
        ("Pi", _D), ("omega", _D), ("l0", _D), ("Lx", _D),
        ("dx", _D), ("dy", _D), ("dz", _D), ("dt", _D), ("dt_half", _D),
        ("laser_amplitude", _D), ("laser_pulse_duration", _D), ("laser_start_time", _D),
        ("waist", _D), ("xfocus", _D), ("yfocus", _D), ("zfocus", _D), ("phase", _D),
        ("E_schwinger", _D),
        ("charge", _D * 2), ("mass", _D * 2),
        ("capacity", _I64 * 2),
        ("precision", _I32), ("spin", _I32), ("deposit_rho", _I32),
        ("laser_envelope", _I32), ("laser_profile", _I32), ("tile", _I32), ("sort_interval", _I32), ("adjoint", _I32),
        ("absorbing", _I32),
    ]


class PicDensity(ctypes.Structure):
    _fields_ = [("kind", _I32), ("nknots", _I32), ("value", _D), ("lo", _D * 3), ("hi", _D * 3),
                ("knot_x", ctypes.POINTER(_D)), ("knot_v", ctypes.POINTER(_D))]


DENSITY_UNIFORM, DENSITY_BOX, DENSITY_XPROFILE = range(3)


class PicError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


_lib = None

EXPORTS = [
    "pic_default_params", "pic_create", "pic_destroy", "pic_last_error", "pic_array_len", "pic_upload_array",
    "pic_download_array", "pic_upload_particles", "pic_download_particles", "pic_num_particles",
    "pic_set_g_table", "pic_set_laser_profile", "pic_radiating_boundary", "pic_update_fields_first",
    "pic_update_fields_second", "pic_clear_currents", "pic_update_particles", "pic_exchange_particles",
    "pic_exchange_currents", "pic_initial_push", "pic_run_steps", "pic_get_step", "pic_set_step",
    "pic_synchronize", "pic_get_stream", "pic_diagnostics", "pic_profile_enable", "pic_profile_read",
    "pic_profile_reset", "pic_save", "pic_load", "pic_field_diagnostics_noalloc", "pic_checkpoint_save",
    "pic_checkpoint_restore", "pic_adjoint_tape", "pic_adjoint_record", "pic_adjoint_seed_kinetic",
    "pic_adjoint_backward", "pic_adjoint_weight_grad", "pic_adjoint_profile_grad", "pic_adjoint_release",
    "pic_update_fields_full", "pic_exchange_boundary", "pic_exchange_current", "pic_filter_current",
    "pic_binomial_filter_currents", "pic_deposit_particle", "pic_eval", "pic_solve_initial_field",
    "pic_initialize_particles", "pic_generate_thermal", "pic_particle_order_stats",
]

# pic_eval selectors (include/pic3d_gpu.h)
EVAL_SHAPE2, EVAL_SHAPE4, EVAL_G_FACTOR, EVAL_LASER_PULSE, EVAL_GPULSE = range(5)


def load(path: str = LIB_PATH):
    """Load the CUDA library; raises if it is missing (no fallback path)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"{path} is not built; run `python -m pic3d_b200.build`")
    lib = ctypes.CDLL(path)
    P, V = ctypes.POINTER, ctypes.c_void_p
    lib.pic_default_params.argtypes = [P(PicParams)]
    lib.pic_default_params.restype = None
    lib.pic_create.argtypes = [P(PicParams), ctypes.c_int, P(V)]
    lib.pic_destroy.argtypes = [V]
    lib.pic_last_error.argtypes = [V]
    lib.pic_last_error.restype = ctypes.c_char_p
    lib.pic_array_len.argtypes = [V, ctypes.c_int, P(_I64)]
    lib.pic_upload_array.argtypes = [V, ctypes.c_int, V]
    lib.pic_download_array.argtypes = [V, ctypes.c_int, V]
    lib.pic_upload_particles.argtypes = [V, ctypes.c_int, V, _I64]
    lib.pic_download_particles.argtypes = [V, ctypes.c_int, V, _I64, P(_I64)]
    lib.pic_num_particles.argtypes = [V, ctypes.c_int, P(_I64)]
    lib.pic_set_g_table.argtypes = [V, V, ctypes.c_int]
    lib.pic_set_laser_profile.argtypes = [V, V, ctypes.c_int]
    lib.pic_radiating_boundary.argtypes = [V, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    for n in ["pic_update_fields_first", "pic_update_fields_second", "pic_clear_currents", "pic_exchange_currents",
              "pic_initial_push", "pic_synchronize", "pic_profile_reset", "pic_update_fields_full",
              "pic_binomial_filter_currents"]:
        getattr(lib, n).argtypes = [V]
    lib.pic_update_particles.argtypes = [V, ctypes.c_int]
    lib.pic_exchange_particles.argtypes = [V, ctypes.c_int]
    lib.pic_run_steps.argtypes = [V, ctypes.c_int]
    lib.pic_get_step.argtypes = [V, P(ctypes.c_int)]
    lib.pic_set_step.argtypes = [V, ctypes.c_int]
    lib.pic_get_stream.argtypes = [V, P(V)]
    lib.pic_diagnostics.argtypes = [V, V, ctypes.c_int]
    lib.pic_profile_enable.argtypes = [V, ctypes.c_int]
    lib.pic_profile_read.argtypes = [V, P(ctypes.c_char_p), P(_D), P(_I64), ctypes.c_int, P(ctypes.c_int)]
    lib.pic_field_diagnostics_noalloc.argtypes = [P(PicParams)] + [V] * 10
    lib.pic_checkpoint_save.argtypes = [V, ctypes.c_int]
    lib.pic_checkpoint_restore.argtypes = [V, ctypes.c_int]
    lib.pic_adjoint_tape.argtypes = [V, ctypes.c_int]
    lib.pic_adjoint_record.argtypes = [V, ctypes.c_int]
    lib.pic_adjoint_seed_kinetic.argtypes = [V, ctypes.c_int, _D, _D, _D, P(_D)]
    lib.pic_adjoint_backward.argtypes = [V, ctypes.c_int]
    lib.pic_adjoint_weight_grad.argtypes = [V, ctypes.c_int, V, _I64]
    lib.pic_adjoint_profile_grad.argtypes = [V, V, ctypes.c_int]
    lib.pic_adjoint_release.argtypes = [V]
    lib.pic_exchange_boundary.argtypes = [V, ctypes.c_int]
    lib.pic_exchange_current.argtypes = [V, ctypes.c_int]
    lib.pic_filter_current.argtypes = [V, ctypes.c_int]
    lib.pic_deposit_particle.argtypes = [V, ctypes.c_int, V]
    lib.pic_eval.argtypes = [V, ctypes.c_int, P(_D), ctypes.c_int, P(_D), ctypes.c_int]
    lib.pic_save.argtypes = [V, ctypes.c_char_p]
    lib.pic_load.argtypes = [V, ctypes.c_char_p]
    lib.pic_solve_initial_field.argtypes = [V, _D, ctypes.c_int, P(_D), ctypes.c_int]
    lib.pic_initialize_particles.argtypes = [V, ctypes.c_int, P(PicDensity), ctypes.c_int, P(_D), P(_D)]
    lib.pic_generate_thermal.argtypes = [V, ctypes.c_int, ctypes.c_int, _D, _D, ctypes.c_uint64]
    lib.pic_particle_order_stats.argtypes = [V, ctypes.c_int, P(_I64), ctypes.c_int]
    _lib = lib
    return lib
