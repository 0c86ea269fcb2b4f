"""ctypes binding of libimaging2d_wlsq_b200.so (the C ABI in include/imaging2d_wlsq_b200.h).

The library is loaded from this package directory.  There is no fallback: if the shared library
is missing or fails to load, importing a module that needs it raises ImportError with the reason,
and every wrapped call raises LibraryError when the C function reports a failure.
"""
import ctypes
import os
from ctypes import POINTER, c_char_p, c_double, c_int, c_longlong, c_size_t, c_void_p

import numpy as np
from numpy.ctypeslib import ndpointer

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, "libimaging2d_wlsq_b200.so")
DROPIN_DIR = os.path.join(PKG_DIR, "dropin")

IMG2D_OK = 0
IMG2D_EINVAL = 1
IMG2D_ENOMEM = 2
IMG2D_ECUDA = 3
IMG2D_ENODEV = 4
FLAG_TWO_TABLES = 1
FLAG_GENERIC = 2
FLAG_NO_CLUSTER = 4
FLAG_CLUSTER_V1 = 8
FLAG_VARIANT_SHIFT = 8
SOURCE_RECOMPUTE, SOURCE_KEEP, SOURCE_REUSE = 0, 1, 2
FLAG_TABLE_FP16 = 16
FLAG_TABLE_BF16 = 32
FLAG_DEMIG_NO_RING = 64
FLAG_WIDE = 128
FLAG_WIDE_SCALAR = 1 << 16
FLAG_CLUSTER2 = 1 << 17
FLAG_WIDE_BULK = 1 << 18
FLAG_LINE_PACKING = 1 << 19
NOALLOC_SCRATCH_BYTES = 64 << 20

ERROR_NAMES = {1: "EINVAL", 2: "ENOMEM", 3: "ECUDA", 4: "ENODEV"}


class LibraryError(RuntimeError):
    """A C entry point returned a non-zero status."""

    def __init__(self, code, message):
        super().__init__(f"imaging2d_wlsq_b200 {ERROR_NAMES.get(code, code)}: {message}")
        self.code = code


def _c64(flags=("C", "A")):
    return ndpointer(dtype=np.complex64, flags=flags)


def _f32():
    return ndpointer(dtype=np.float32, flags=("C", "A"))


def _f64():
    return ndpointer(dtype=np.float64, flags=("C", "A"))


def load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m imaging2d_wlsq_b200.build` "
            "(CUDA toolkit with sm_100a support required)")
    lib = ctypes.CDLL(LIB_PATH)
    lib.img2d_last_error.restype = c_char_p
    lib.img2d_last_error.argtypes = []
    lib.img2d_version.restype = c_int
    lib.img2d_version.argtypes = []
    lib.img2d_extrapolate_host_order.restype = c_int
    lib.img2d_extrapolate_host_order.argtypes = [c_int] * 7 + [_c64(), _c64(), _c64(), _c64(), _f32()]
    lib.img2d_extrapolate_device_order.restype = c_int
    lib.img2d_extrapolate_device_order.argtypes = [c_int] * 7 + [_c64(), _c64(), _c64(), _c64(), _f32(), c_int]
    lib.img2d_migrate_compact.restype = c_int
    lib.img2d_migrate_compact.argtypes = [c_int] * 8 + [c_double, c_void_p, c_void_p, c_void_p, c_void_p,
                                                        c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                                        c_void_p, c_int]
    lib.img2d_plan_create.restype = c_int
    lib.img2d_plan_create.argtypes = [POINTER(c_void_p)] + [c_int] * 8 + [c_void_p, c_void_p, c_int]
    lib.img2d_plan_set_model.restype = c_int
    lib.img2d_plan_set_model.argtypes = [c_void_p, c_void_p, c_void_p, c_double, c_void_p, c_void_p, c_void_p]
    lib.img2d_plan_execute.restype = c_int
    lib.img2d_plan_execute.argtypes = [c_void_p] * 6
    lib.img2d_plan_execute_naive.restype = c_int
    lib.img2d_plan_execute_naive.argtypes = [c_void_p] * 5
    lib.img2d_plan_dense_table.restype = c_int
    lib.img2d_plan_dense_table.argtypes = [c_void_p, c_int, c_void_p, c_void_p]
    lib.img2d_plan_shot_offset.restype = c_longlong
    lib.img2d_plan_shot_offset.argtypes = [c_void_p, c_int]
    lib.img2d_plan_wavefield_elems.restype = c_longlong
    lib.img2d_plan_wavefield_elems.argtypes = [c_void_p]
    lib.img2d_plan_workspace_bytes.restype = c_size_t
    lib.img2d_plan_workspace_bytes.argtypes = [c_void_p]
    lib.img2d_plan_describe.restype = c_int
    lib.img2d_plan_describe.argtypes = [c_void_p, c_char_p, c_int]
    lib.img2d_plan_kernel_ms.restype = c_int
    lib.img2d_plan_kernel_ms.argtypes = [c_void_p, POINTER(ctypes.c_float)]
    lib.img2d_plan_status.restype = c_int
    lib.img2d_plan_status.argtypes = [c_void_p, c_void_p]
    lib.img2d_pack_shots.restype = c_int
    lib.img2d_pack_shots.argtypes = [c_int, c_int, c_int, c_void_p, c_void_p, c_int, c_int, c_void_p, c_void_p,
                                     c_void_p, c_void_p, POINTER(c_int), POINTER(c_double)]
    lib.img2d_measure_fp32_peak.restype = c_int
    lib.img2d_measure_fp32_peak.argtypes = [POINTER(c_double)]
    lib.img2d_ricker_sources.restype = c_int
    lib.img2d_ricker_sources.argtypes = [c_int] * 3 + [c_double] * 6 + [c_void_p] * 3
    lib.img2d_records_to_spectra.restype = c_int
    lib.img2d_records_to_spectra.argtypes = [c_int] * 5 + [c_void_p] * 5
    lib.img2d_measure_l2_bandwidth.restype = c_int
    lib.img2d_measure_l2_bandwidth.argtypes = [POINTER(c_double)]
    lib.img2d_migrate_compact_noalloc.restype = c_int
    lib.img2d_migrate_compact_noalloc.argtypes = [c_int] * 8 + [c_double] + [c_void_p] * 9
    lib.img2d_plan_demigrate.restype = c_int
    lib.img2d_plan_demigrate.argtypes = [c_void_p] * 4 + [c_int, c_int, c_void_p]
    lib.img2d_plan_describe_demigration.restype = c_int
    lib.img2d_plan_describe_demigration.argtypes = [c_void_p, c_char_p, c_int]
    lib.img2d_release_host_cache.restype = None
    lib.img2d_release_host_cache.argtypes = []
    lib.img2d_host_cache_device_count.restype = c_int
    lib.img2d_host_cache_device_count.argtypes = []
    lib.img2d_set_alloc_limit.restype = None
    lib.img2d_set_alloc_limit.argtypes = [c_size_t]
    lib.img2d_plan_destroy.restype = None
    lib.img2d_plan_destroy.argtypes = [c_void_p]
    return lib


_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        _LIB = load()
    return _LIB


def check(rc):
    if rc != IMG2D_OK:
        msg = lib().img2d_last_error()
        raise LibraryError(rc, msg.decode() if msg else "")
    return rc


def ptr(a):
    """Raw address of a numpy array, a torch tensor, or None."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return a.data_ptr()
