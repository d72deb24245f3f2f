"""ctypes binding of libfgpe.so (the C ABI declared in include/fgpe.h).

The shared library is built in-tree by ``fortress_b200.build.build()``.  There
is no CPU fallback: if the library is missing or no sm_100 device is present,
every call that needs the GPU raises :class:`FgpeError`.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
# FGPE_LIB_PATH selects an alternative build of the same library (for example
# a diagnostic build); the default is the in-tree libfgpe.so.
LIB_PATH = os.environ.get("FGPE_LIB_PATH") or os.path.join(_HERE, "libfgpe.so")

FGPE_OK = 0
FGPE_E_ARG = -1
FGPE_E_CUDA = -2
FGPE_E_STATE = -3
FGPE_E_NONFINITE = -4
FGPE_E_NEWTON = -5
FGPE_E_TIMEOUT = -6

FGPE_FP64 = 0
FGPE_FP32 = 1
FGPE_STEP_DEFAULT = 0
FGPE_STEP_NO_SNAPSHOT = 1
FGPE_BATCH_BRANCHES = 0
FGPE_BATCH_GROUPED = 1
FGPE_BATCH_PERSISTENT = 2

OPS = {"FFT": 1, "KE": 2, "SOC": 3, "BFT": 4, "SE": 5, "SP": 6}

# Every symbol include/fgpe.h declares.
EXPORTS = (
    "fgpe_create", "fgpe_destroy", "fgpe_last_error", "fgpe_set_stream",
    "fgpe_set_state", "fgpe_get_state", "fgpe_set_state_device", "fgpe_get_state_device",
    "fgpe_step", "fgpe_step_ex", "fgpe_normalize", "fgpe_norms", "fgpe_observables",
    "fgpe_conv", "fgpe_center", "fgpe_apply_op", "fgpe_version", "fgpe_device_ok",
    "fgpe_kernel_launches", "fgpe_norms_async", "fgpe_profile_enable", "fgpe_profile_read",
    "fgpe_batch_create", "fgpe_batch_destroy", "fgpe_batch_size", "fgpe_batch_instance",
    "fgpe_batch_last_error", "fgpe_batch_config", "fgpe_batch_step", "fgpe_batch_observables",
    "fgpe_batch_autotune", "fgpe_batch_tuning", "fgpe_set_kernels", "fgpe_normc_noalloc",
    "fgpe_checkpoint_save", "fgpe_checkpoint_load", "fgpe_batch_step_timed", "fgpe_norms_sink",
    "fgpe_fp64_fma_rate", "fgpe_batch_mode", "fgpe_batch_variant", "fgpe_batch_variant_shape",
    "fgpe_batch_variants", "fgpe_batch_wait_bound",
)


class FgpeError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"fgpe error {code}: {msg}")
        self.code = code


class Params(ctypes.Structure):
    _fields_ = [("dim", ctypes.c_int), ("spin", ctypes.c_int),
                ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("dz", ctypes.c_double),
                ("dt", ctypes.c_double), ("imag_time", ctypes.c_int),
                ("tau", ctypes.c_double * 3), ("gamma", ctypes.c_double * 3),
                ("alpha", ctypes.c_double * 3), ("precision", ctypes.c_int),
                ("kernels", ctypes.c_int), ("mag", ctypes.c_double), ("reserved", ctypes.c_int * 4)]


_LIB = None


def load():
    """Load libfgpe.so (raises if it was not built)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise FgpeError(FGPE_E_CUDA, f"{LIB_PATH} not built; run fortress_b200.build.build()")
    L = ctypes.CDLL(LIB_PATH)
    vp, dp, ip = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_int
    sig = {
        "fgpe_create": ([ctypes.POINTER(Params), ctypes.POINTER(vp)], ip),
        "fgpe_destroy": ([vp], ip),
        "fgpe_last_error": ([vp], ctypes.c_char_p),
        "fgpe_set_stream": ([vp, vp], ip),
        "fgpe_set_state": ([vp, vp], ip),
        "fgpe_get_state": ([vp, vp], ip),
        "fgpe_set_state_device": ([vp, vp], ip),
        "fgpe_get_state_device": ([vp, vp], ip),
        "fgpe_step": ([vp, ip], ip),
        "fgpe_step_ex": ([vp, ip, ip], ip),
        "fgpe_normalize": ([vp, dp], ip),
        "fgpe_norms": ([vp, dp], ip),
        "fgpe_observables": ([vp, dp, dp, dp, dp], ip),
        "fgpe_conv": ([vp, dp], ip),
        "fgpe_center": ([vp, dp], ip),
        "fgpe_apply_op": ([vp, ip], ip),
        "fgpe_version": ([], ip),
        "fgpe_device_ok": ([], ip),
        "fgpe_kernel_launches": ([vp, ctypes.POINTER(ctypes.c_longlong)], ip),
        "fgpe_norms_async": ([vp, vp], ip),
        "fgpe_norms_sink": ([vp, vp, ip], ip),
        "fgpe_profile_enable": ([vp, ip], ip),
        "fgpe_profile_read": ([vp, dp, ctypes.POINTER(ctypes.c_longlong), ip], ip),
        "fgpe_batch_create": ([ctypes.POINTER(Params), ip, ctypes.POINTER(vp)], ip),
        "fgpe_batch_destroy": ([vp], ip),
        "fgpe_batch_size": ([vp], ip),
        "fgpe_batch_instance": ([vp, ip, ctypes.POINTER(vp)], ip),
        "fgpe_batch_last_error": ([vp], ctypes.c_char_p),
        "fgpe_batch_config": ([vp, ip, ip], ip),
        "fgpe_batch_step": ([vp, ip], ip),
        "fgpe_batch_step_timed": ([vp, ip, dp], ip),
        "fgpe_batch_observables": ([vp, dp, ip], ip),
        "fgpe_batch_autotune": ([vp, ip, ctypes.c_char_p], ip),
        "fgpe_batch_tuning": ([vp, ctypes.POINTER(ip), ctypes.POINTER(ip)], ip),
        "fgpe_set_kernels": ([vp, ip], ip),
        "fgpe_normc_noalloc": ([ip, ip, ip, ip, ip, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                vp, vp, vp], ip),
        "fgpe_checkpoint_save": ([vp, ctypes.c_char_p, ctypes.c_longlong, dp], ip),
        "fgpe_checkpoint_load": ([vp, ctypes.c_char_p, ctypes.POINTER(ctypes.c_longlong), dp], ip),
        "fgpe_fp64_fma_rate": ([ip, dp], ip),
        "fgpe_batch_mode": ([vp, ip], ip),
        "fgpe_batch_variant": ([vp, ip, ctypes.POINTER(ip)], ip),
        "fgpe_batch_variant_shape": ([ip, ctypes.POINTER(ip)], ip),
        "fgpe_batch_variants": ([], ip),
        "fgpe_batch_wait_bound": ([vp, ctypes.c_double, ip], ip),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _LIB = L
    return L


def check(rc, handle=None):
    if rc != FGPE_OK:
        msg = load().fgpe_last_error(handle)
        raise FgpeError(rc, msg.decode() if msg else "")
    return rc


def check_batch(rc, batch=None):
    if rc != FGPE_OK:
        msg = load().fgpe_batch_last_error(batch)
        raise FgpeError(rc, msg.decode() if msg else "")
    return rc
