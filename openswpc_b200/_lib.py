"""ctypes binding of ``lib/libswpc_gpu.so`` (include/swpc_gpu.h, include/swpc_setup.h).

The library is the product: every time-step computation happens in its CUDA
kernels.  Loading fails loudly when the shared library is missing; there is no
CPU fallback.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libswpc_gpu.so"

SWPC_OK = 0
SWPC_ERR_ARG = 1
SWPC_ERR_CUDA = 2
SWPC_ERR_STATE = 3
SWPC_ERR_DIVERGED = 4
SWPC_ERR_NOMEM = 5
SWPC_ERR_LIMIT = 6
PREC_F32, PREC_BF16_R, PREC_F16_SR, PREC_F16_R = 0, 1, 2, 3
PRECISIONS = {"f32": PREC_F32, "bf16r": PREC_BF16_R, "f16sr": PREC_F16_SR, "f16r": PREC_F16_R}
SWPC_NOALLOC_MAX_NY = 16384

KIND_3D, KIND_PSV, KIND_SH = 3, 2, 1
STF_CODES = {"kupper": 0, "boxcar": 1, "triangle": 2, "herrmann": 3, "cosine": 4, "scosine": 4, "texp": 5}

F_VX, F_VY, F_VZ, F_SXX, F_SYY, F_SZZ, F_SYZ, F_SXZ, F_SXY = range(9)
F_R = 10
F_AUX = 40
F_MED = 60
WAV_V, WAV_U, WAV_STRESS, WAV_STRAIN = 1, 2, 4, 8

# every symbol the headers in include/ declare
EXPORTS = [
    "swpc_create", "swpc_destroy", "swpc_last_error", "swpc_stream", "swpc_sync", "swpc_upload_medium",
    "swpc_vmodel_lhm_device", "swpc_vmodel_lhm_device_opt", "swpc_vmodel_upload", "swpc_medium_setup_device", "swpc_medium_setup_device_opt", "swpc_absorb_setup_cerjan",
    "swpc_green_store_setup", "swpc_green_store", "swpc_green_fetch", "swpc_fbatch_green_fetch",
    "swpc_kernel_setup", "swpc_absorb_setup", "swpc_source_setup", "swpc_bodyforce_setup", "swpc_green_setup",
    "swpc_wav_setup", "swpc_kernel_update_stress", "swpc_absorb_update_stress", "swpc_kernel_update_vel",
    "swpc_absorb_update_vel", "swpc_update_stress", "swpc_update_vel", "swpc_source_stressglut",
    "swpc_source_bodyforce", "swpc_green_source", "swpc_comm_stress", "swpc_comm_vel", "swpc_wav_store",
    "swpc_vmax", "swpc_vmax_noalloc", "swpc_step", "swpc_run", "swpc_time_steps", "swpc_wav_fetch", "swpc_wav_dims",
    "swpc_snap_setup", "swpc_snap_write", "swpc_snap_dims", "swpc_snap_fetch", "swpc_snap_fetch_max",
    "swpc_adj_reset", "swpc_adj_step_linear", "swpc_adj_upload", "swpc_adj_download", "swpc_gradient",
    "swpc_gradient_set_slot_memory", "swpc_gradient_memory", "swpc_gradient_segment_bytes",
    "swpc_gradient_model_device",
    "swpc_vmodel_velocity_device",
    "swpc_gradient_fetch", "swpc_gradient_model", "swpc_reset_state",
    "swpc_download_field", "swpc_upload_field", "swpc_rescale", "swpc_device_bytes", "swpc_set_launch",
    # swpc_setup.h
    "swpc_x2i", "swpc_i2x", "swpc_momentrate", "swpc_sdr2moment", "swpc_visco_setup", "swpc_kbeg_a",
    "swpc_vmodel_lhm", "swpc_vmodel_lhm_opt", "swpc_seawater_vel", "swpc_setup_medium", "swpc_damping_profiles", "swpc_setup_medium_2d", "swpc_cerjan_profiles",
    "swpc_setup_medium_opt", "swpc_setup_medium_2d_opt", "swpc_rmedia_generate", "swpc_pw_setup", "swpc_set_pw_mode", "swpc_clear_error", "swpc_raise_copy_error",
    "swpc_set_subdomain", "swpc_step_half", "swpc_halo_count", "swpc_halo_pack", "swpc_halo_unpack",
    "swpc_enable_peer_access",
    "swpc_batch_create", "swpc_batch_step", "swpc_batch_run", "swpc_batch_sync", "swpc_batch_time_steps", "swpc_batch_autotune",
    "swpc_batch_set_shape", "swpc_batch_set_staged", "swpc_batch_get_launch",
    "swpc_fbatch_create", "swpc_fbatch_destroy", "swpc_fbatch_green_source", "swpc_fbatch_set_strip",
    "swpc_fbatch_autotune", "swpc_fbatch_step", "swpc_fbatch_run", "swpc_fbatch_time_steps", "swpc_fbatch_sync",
    "swpc_fbatch_wav_fetch", "swpc_fbatch_download_field", "swpc_fbatch_device_bytes", "swpc_fbatch_set_launch",
    "swpc_fbatch_get_launch",
    "swpc_batch_last_error", "swpc_batch_destroy",
]


class SwpcError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"swpc error {code}: {msg}")
        self.code = code


class Desc(C.Structure):
    _fields_ = [("kind", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("na", C.c_int),
                ("nm", C.c_int), ("nt", C.c_int), ("dx", C.c_float), ("dy", C.c_float), ("dz", C.c_float),
                ("dt", C.c_float), ("tbeg", C.c_float), ("device", C.c_int), ("precision", C.c_int)]


_FP = C.POINTER(C.c_float)
_IP = C.POINTER(C.c_int)


class MediumView(C.Structure):
    _fields_ = [("rho", _FP), ("lam", _FP), ("mu", _FP), ("taup", _FP), ("taus", _FP), ("bx", _FP),
                ("by", _FP), ("bz", _FP), ("muyz", _FP), ("muxz", _FP), ("muxy", _FP), ("ld_k", C.c_int),
                ("ld_i", C.c_int), ("kfs", _IP), ("kob", _IP), ("kfs_top", _IP), ("kfs_bot", _IP),
                ("kob_top", _IP), ("kob_bot", _IP), ("kbeg_a", _IP), ("ld_i2", C.c_int)]


class SnapDesc(C.Structure):
    _fields_ = [("planes", C.c_int), ("idec", C.c_int), ("jdec", C.c_int), ("kdec", C.c_int),
                ("ntdec_s", C.c_int), ("i0_yz", C.c_int), ("j0_xz", C.c_int), ("k0_xy", C.c_int),
                ("M0", C.c_float), ("UC", C.c_float)]


class Grid(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("na", C.c_int), ("nm", C.c_int),
                ("dx", C.c_float), ("dy", C.c_float), ("dz", C.c_float), ("dt", C.c_float),
                ("xbeg", C.c_float), ("ybeg", C.c_float), ("zbeg", C.c_float), ("tbeg", C.c_float)]


class RmediaDesc(C.Structure):
    """swpc_rmedia_desc of swpc_setup.h."""
    _fields_ = [("ptype", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("dx", C.c_float),
                ("dy", C.c_float), ("dz", C.c_float), ("a", C.c_float), ("epsil", C.c_float), ("kappa", C.c_float),
                ("seed", C.c_ulonglong)]


_lib = None


def fptr(a):
    if a is None:
        return None
    assert a.dtype == np.float32 and a.flags["C_CONTIGUOUS"] or a.flags["F_CONTIGUOUS"]
    return a.ctypes.data_as(_FP)


def iptr(a):
    if a is None:
        return None
    assert a.dtype == np.int32
    return a.ctypes.data_as(_IP)


def load():
    """Load the shared library (once).  Raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: run `python -m openswpc_b200.build` (needs nvcc)")
    lib = C.CDLL(str(LIB_PATH))
    vp = C.c_void_p
    i = C.c_int
    f = C.c_float
    sig = {
        "swpc_create": (i, [C.POINTER(Desc), C.POINTER(vp)]),
        "swpc_destroy": (i, [vp]),
        "swpc_last_error": (C.c_char_p, [vp]),
        "swpc_stream": (vp, [vp]),
        "swpc_sync": (i, [vp]),
        "swpc_upload_medium": (i, [vp, C.POINTER(MediumView)]),
        "swpc_vmodel_lhm_device": (i, [vp, i, _FP, _FP, _FP, _FP, _FP, _FP, f, f, f, _FP, i, i]),
        "swpc_vmodel_lhm_device_opt": (i, [vp, i, _FP, _FP, _FP, _FP, _FP, _FP, f, f, f, _FP, i, i, i]),
        "swpc_vmodel_upload": (i, [vp, _FP, _FP, _FP, _FP, _FP, i, i]),
        "swpc_vmodel_velocity_device": (i, [vp, vp, vp, vp, vp, vp, i, i]),
        "swpc_medium_setup_device": (i, [vp, f, f, f, _FP, _FP, _IP, _IP, _IP, _IP, _IP, _IP, _IP, i]),
        "swpc_medium_setup_device_opt": (i, [vp, f, f, f, _FP, _FP, _IP, _IP, _IP, _IP, _IP, _IP, _IP, i, i]),
        "swpc_kernel_setup": (i, [vp, _FP]),
        "swpc_absorb_setup": (i, [vp, _FP, _FP, _FP, _FP, _FP, _FP]),
        "swpc_absorb_setup_cerjan": (i, [vp, _FP, _FP, _FP, _FP, _FP, _FP]),
        "swpc_green_store_setup": (i, [vp, i, _IP, _IP, _IP, i, i]),
        "swpc_green_store": (i, [vp, i]),
        "swpc_green_fetch": (i, [vp, _FP]),
        "swpc_fbatch_green_fetch": (i, [vp, i, _FP]),
        "swpc_cerjan_profiles": (None, [C.POINTER(Grid), _FP, _FP, _FP, _FP, _FP, _FP]),
        "swpc_source_setup": (i, [vp, i, _IP, _IP, _IP, _FP, _FP, _FP, i]),
        "swpc_bodyforce_setup": (i, [vp, i, _IP, _IP, _IP, _FP, _FP, i]),
        "swpc_green_setup": (i, [vp, i, i, i, C.c_char, f, f, i]),
        "swpc_wav_setup": (i, [vp, i, _IP, _IP, _IP, i, i, f, f]),
        "swpc_vmax": (i, [vp, _FP]),
        "swpc_vmax_noalloc": (i, [vp, vp, vp, vp, i, i, i, i, i, i, f, vp, _FP]),
        "swpc_step": (i, [vp, i]),
        "swpc_run": (i, [vp, i, i]),
        "swpc_time_steps": (i, [vp, i, i, _FP]),
        "swpc_wav_fetch": (i, [vp, i, _FP]),
        "swpc_wav_dims": (i, [vp, _IP, _IP]),
        "swpc_snap_setup": (i, [vp, C.POINTER(SnapDesc)]),
        "swpc_snap_write": (i, [vp, i]),
        "swpc_snap_dims": (i, [vp, i, _IP, _IP, _IP, _IP]),
        "swpc_snap_fetch": (i, [vp, i, _FP]),
        "swpc_snap_fetch_max": (i, [vp, i, _FP]),
        "swpc_download_field": (i, [vp, i, _FP, i, i]),
        "swpc_upload_field": (i, [vp, i, _FP, i, i]),
        "swpc_rescale": (i, [vp, _IP]),
        "swpc_adj_reset": (i, [vp]),
        "swpc_reset_state": (i, [vp]),
        "swpc_adj_step_linear": (i, [vp]),
        "swpc_adj_upload": (i, [vp, i, _FP, i, i]),
        "swpc_adj_download": (i, [vp, i, _FP, i, i]),
        "swpc_gradient": (i, [vp, _FP, i, C.POINTER(C.c_double)]),
        "swpc_gradient_set_slot_memory": (i, [vp, C.c_longlong]),
        "swpc_gradient_memory": (i, [vp, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]),
        "swpc_gradient_segment_bytes": (i, [vp, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong), i]),
        "swpc_gradient_fetch": (i, [vp, i, C.POINTER(C.c_double), i, i]),
        "swpc_gradient_model": (i, [vp, _FP, _FP, _FP, i, i, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                    C.POINTER(C.c_double)]),
        "swpc_gradient_model_device": (i, [vp, vp, vp, vp, i, i, vp, vp, vp]),
        "swpc_device_bytes": (C.c_longlong, [vp]),
        "swpc_set_launch": (i, [vp, i, i, i, i]),
        "swpc_x2i": (i, [f, f, f]),
        "swpc_i2x": (f, [i, f, f]),
        "swpc_momentrate": (f, [f, i, f, f]),
        "swpc_sdr2moment": (None, [f, f, f, _FP]),
        "swpc_visco_setup": (None, [i, f, f, _FP, _FP]),
        "swpc_kbeg_a": (None, [C.POINTER(Grid), _IP]),
        "swpc_vmodel_lhm": (i, [C.POINTER(Grid), i, _FP, _FP, _FP, _FP, _FP, _FP, f, _FP, f, _FP, _FP, _FP,
                                _FP, _FP]),
        "swpc_vmodel_lhm_opt": (i, [C.POINTER(Grid), i, _FP, _FP, _FP, _FP, _FP, _FP, f, _FP, f, _FP, _FP, _FP,
                                    _FP, _FP, i]),
        "swpc_seawater_vel": (f, [f, i]),
        "swpc_setup_medium": (i, [C.POINTER(Grid), f, f, f, _FP, _FP, _FP, _FP, _FP, _FP, _FP, _FP, _FP, _FP,
                                  _FP, _FP, _FP, _IP, _IP, _IP, _IP, _IP, _IP, _FP, _FP]),
        "swpc_setup_medium_opt": (i, [C.POINTER(Grid), f, f, f, _FP, _FP, _FP, _FP, _FP, _FP, _FP, _FP, _FP, _FP,
                                      _FP, _FP, _FP, _IP, _IP, _IP, _IP, _IP, _IP, _FP, _FP, i]),
        "swpc_damping_profiles": (None, [C.POINTER(Grid), f, _FP, _FP, _FP, _FP, _FP, _FP]),
        "swpc_setup_medium_2d": (i, [C.POINTER(Grid), f, f, f, _FP, _FP, _FP, _FP, _FP, _FP, _FP, _IP, _IP, _IP,
                                     _IP, _IP, _IP, _FP, _FP]),
        "swpc_setup_medium_2d_opt": (i, [C.POINTER(Grid), f, f, f, _FP, _FP, _FP, _FP, _FP, _FP, _FP, _IP, _IP, _IP,
                                     _IP, _IP, _IP, _FP, _FP, i]),
        "swpc_rmedia_generate": (i, [C.POINTER(RmediaDesc), _FP, i, i, vp]),
        "swpc_pw_setup": (i, [C.POINTER(Grid), _FP, _FP, _FP, f, f, i, f, f, f, i] + [_FP] * 9 + [_FP]),
        "swpc_set_pw_mode": (i, [vp, i]),
        "swpc_set_subdomain": (i, [vp, i, i, i, i]),
        "swpc_step_half": (i, [vp, i, i]),
        "swpc_halo_count": (i, [vp, i, i, C.POINTER(C.c_longlong)]),
        "swpc_halo_pack": (i, [vp, i, i, vp]),
        "swpc_halo_unpack": (i, [vp, i, i, vp]),
        "swpc_enable_peer_access": (i, [i, i]),
        "swpc_clear_error": (i, [vp]),
        "swpc_raise_copy_error": (i, [vp]),
        "swpc_batch_create": (i, [C.POINTER(vp), i, C.POINTER(vp)]),
        "swpc_batch_step": (i, [vp, i]),
        "swpc_batch_run": (i, [vp, i, i]),
        "swpc_batch_sync": (i, [vp]),
        "swpc_batch_time_steps": (i, [vp, i, i, _FP]),
        "swpc_batch_autotune": (i, [vp, i, i, _IP, _IP, _IP, _IP]),
        "swpc_batch_set_shape": (i, [vp, i, i, i]),
        "swpc_batch_set_staged": (i, [vp, i, i]),
        "swpc_batch_get_launch": (i, [vp, _IP]),
        "swpc_batch_last_error": (C.c_char_p, [vp]),
        "swpc_batch_destroy": (i, [vp]),
        "swpc_fbatch_create": (i, [vp, i, C.POINTER(vp)]),
        "swpc_fbatch_destroy": (i, [vp]),
        "swpc_fbatch_green_source": (i, [vp, i, i, i, i, C.c_char, f, f, i]),
        "swpc_fbatch_set_strip": (i, [vp, i]),
        "swpc_fbatch_autotune": (i, [vp, i, i, _IP, _IP]),
        "swpc_fbatch_step": (i, [vp, i]),
        "swpc_fbatch_run": (i, [vp, i, i]),
        "swpc_fbatch_time_steps": (i, [vp, i, i, _FP]),
        "swpc_fbatch_sync": (i, [vp]),
        "swpc_fbatch_wav_fetch": (i, [vp, i, i, _FP]),
        "swpc_fbatch_download_field": (i, [vp, i, i, _FP, i, i]),
        "swpc_fbatch_device_bytes": (C.c_longlong, [vp]),
        "swpc_fbatch_set_launch": (i, [vp, i, i, i, i]),
        "swpc_fbatch_get_launch": (i, [vp, _IP]),
    }
    for name in ("swpc_kernel_update_stress", "swpc_absorb_update_stress", "swpc_kernel_update_vel",
                 "swpc_absorb_update_vel", "swpc_update_stress", "swpc_update_vel", "swpc_comm_stress",
                 "swpc_comm_vel"):
        sig[name] = (i, [vp])
    for name in ("swpc_source_stressglut", "swpc_source_bodyforce", "swpc_green_source", "swpc_wav_store"):
        sig[name] = (i, [vp, i])
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(ctx, rc: int) -> None:
    if rc != SWPC_OK:
        msg = load().swpc_last_error(ctx)
        raise SwpcError(rc, msg.decode() if msg else "")
