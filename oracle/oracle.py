"""ctypes binding of oracle/liboracle.so and oracle/_ref/extrapolation_cpu.so.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
legs as the checker / reference timing.  The product (imaging2d_wlsq_b200) never imports it.

  liboracle.so               CPU restatement of the reference path (oracle/wlsq_oracle.c)
  _ref/extrapolation_cpu.so  the reference's own CPU library built from its sources by
                             oracle/build_ref.sh (present when the reference sources were
                             available at build time)
"""
import ctypes
import os
from ctypes import c_double, c_int, c_void_p

import numpy as np
from numpy.ctypeslib import ndpointer

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "extrapolation_cpu.so")

_c64 = ndpointer(dtype=np.complex64, flags=("C", "A"))
_c128 = ndpointer(dtype=np.complex128, flags=("C", "A"))
_f32 = ndpointer(dtype=np.float32, flags=("C", "A"))
_f64 = ndpointer(dtype=np.float64, flags=("C", "A"))

_O = None
_R = None


def _load_oracle():
    global _O
    if _O is None:
        if not os.path.exists(ORACLE_LIB):
            raise FileNotFoundError(f"{ORACLE_LIB} missing; run `python -m imaging2d_wlsq_b200.build`")
        o = ctypes.CDLL(ORACLE_LIB)
        o.oracle_nearest_kappa.restype = c_int
        o.oracle_nearest_kappa.argtypes = [c_double, c_double, c_int]
        o.oracle_extrapolate_dense_f32.restype = None
        o.oracle_extrapolate_dense_f32.argtypes = [c_int] * 7 + [_c64, _c64, _c64, _c64, _f32]
        o.oracle_extrapolate_dense_f64.restype = None
        o.oracle_extrapolate_dense_f64.argtypes = [c_int] * 7 + [_c64, _c64, _c128, _c128, _f64]
        o.oracle_migrate_compact_f64.restype = None
        o.oracle_migrate_compact_f64.argtypes = [c_int] * 8 + [c_double, _f64, _f64, _c64, c_void_p,
                                                               c_void_p, c_void_p, c_void_p, _c128, _c128,
                                                               c_void_p, c_void_p]
        o.oracle_demigrate_compact_f64.restype = None
        o.oracle_demigrate_compact_f64.argtypes = [c_int] * 7 + [c_double, _f64, _f64, _c64, c_void_p, c_void_p,
                                                                 c_void_p, _c128, _f64, _c128]
        o.oracle_gather_dense_slab.restype = None
        o.oracle_gather_dense_slab.argtypes = [c_int] * 8 + [c_double, _f64, _f64, _c64, c_int, _c64]
        o.oracle_index_table.restype = None
        o.oracle_index_table.argtypes = [c_int] * 4 + [c_double, _f64, _f64, ndpointer(dtype=np.int32)]
        _O = o
    return _O


def have_ref():
    return os.path.exists(REF_LIB)


def _load_ref():
    global _R
    if _R is None:
        r = ctypes.CDLL(REF_LIB)
        for name in ("extrapolate", "extrapolate_v0"):
            f = getattr(r, name)
            f.restype = None
            f.argtypes = [c_int] * 7 + [_c64, _c64, _c64, _c64, _f32]
        _R = r
    return _R


def nearest_kappa(value, dk, nk):
    return _load_oracle().oracle_nearest_kappa(float(value), float(dk), int(nk))


def extrapolate_f32(ns, nextrap, nz, nx, nf, nt, M, opF, opB, wave, shot, image):
    """Host-order dense extrapolation in FP32 (in place, like the reference)."""
    _load_oracle().oracle_extrapolate_dense_f32(ns, nextrap, nz, nx, nf, nt, M, opF, opB, wave, shot, image)


def extrapolate_f64(ns, nextrap, nz, nx, nf, nt, M, opF, opB, wave, shot):
    """FP64 dense extrapolation; returns (image (ns, nz, nx) float64, wave, shot complex128)."""
    w = np.ascontiguousarray(wave, dtype=np.complex128).copy()
    s = np.ascontiguousarray(shot, dtype=np.complex128).copy()
    img = np.zeros((ns, nz, nx), dtype=np.float64)
    _load_oracle().oracle_extrapolate_dense_f64(ns, nextrap, nz, nx, nf, nt, M, opF, opB, w, s, img)
    return img, w, s


def ref_extrapolate(ns, nextrap, nz, nx, nf, nt, M, opF, opB, wave, shot, image, v0=False):
    """The reference's own extrapolation_cpu.so (host order, in place)."""
    f = _load_ref().extrapolate_v0 if v0 else _load_ref().extrapolate
    f(ns, nextrap, nz, nx, nf, nt, M, opF, opB, wave, shot, image)


def migrate_compact_f64(ns, nextrap, nz, nx, nf, nt, M, nk, dk, omega, velocity, tab_forw, wave, shot,
                        tab_back=None, shot_x0=None, shot_nx=None, offsets=None):
    """FP64 compact-table migration.  Returns (stack (nz, nx), per-shot (ns, nz, nx), wave, shot)."""
    o = _load_oracle()
    w = np.ascontiguousarray(wave, dtype=np.complex128).copy()
    s = np.ascontiguousarray(shot, dtype=np.complex128).copy()
    stack = np.zeros((nz, nx), dtype=np.float64)
    shots = np.zeros((ns, nz, nx), dtype=np.float64)
    x0 = None if shot_x0 is None else np.ascontiguousarray(shot_x0, dtype=np.int32)
    wn = None if shot_nx is None else np.ascontiguousarray(shot_nx, dtype=np.int32)
    off = None if offsets is None else np.ascontiguousarray(offsets, dtype=np.int64)
    tb = None if tab_back is None else np.ascontiguousarray(tab_back, dtype=np.complex64)

    def p(a):
        return None if a is None else a.ctypes.data

    o.oracle_migrate_compact_f64(ns, nextrap, nz, nx, nf, nt, M, nk, float(dk),
                                 np.ascontiguousarray(omega, dtype=np.float64),
                                 np.ascontiguousarray(velocity, dtype=np.float64),
                                 np.ascontiguousarray(tab_forw, dtype=np.complex64), p(tb), p(x0), p(wn), p(off),
                                 w, s, shots.ctypes.data, stack.ctypes.data)
    return stack, shots, w, s


def migrate_workload_f64(wl, nextrap=None, tab_back=None):
    n = nextrap or wl.nextrap
    return migrate_compact_f64(wl.ns, n, wl.nz, wl.nx, wl.nf, wl.nt, wl.M, wl.nk, wl.dk, wl.omega, wl.velocity,
                               wl.table, wl.wave, wl.shot, tab_back=tab_back, shot_x0=wl.shot_x0,
                               shot_nx=wl.shot_nx, offsets=wl.offsets())


def demigrate_compact_f64(ns, nextrap, nx, nf, nt, M, nk, dk, omega, velocity, tab_forw, wave, refl,
                          shot_x0=None, shot_nx=None, offsets=None):
    """FP64 demigration (adjoint of migrate_compact_f64 with respect to the receiver spectra,
    single-table mode).  refl: (>= nextrap, nx) reflectivity.  Returns the packed data array
    (complex128, same layout as wave; rows >= nf of each shot block are zero)."""
    o = _load_oracle()
    w = np.ascontiguousarray(wave, dtype=np.complex128)
    data = np.zeros_like(w)
    r = np.ascontiguousarray(np.asarray(refl, dtype=np.float64)[:nextrap])
    x0 = None if shot_x0 is None else np.ascontiguousarray(shot_x0, dtype=np.int32)
    wn = None if shot_nx is None else np.ascontiguousarray(shot_nx, dtype=np.int32)
    off = None if offsets is None else np.ascontiguousarray(offsets, dtype=np.int64)

    def p(a):
        return None if a is None else a.ctypes.data

    o.oracle_demigrate_compact_f64(ns, nextrap, nx, nf, nt, M, nk, float(dk),
                                   np.ascontiguousarray(omega, dtype=np.float64),
                                   np.ascontiguousarray(velocity, dtype=np.float64),
                                   np.ascontiguousarray(tab_forw, dtype=np.complex64), p(x0), p(wn), p(off),
                                   w, r, data)
    return data


def demigrate_workload_f64(wl, refl, nextrap=None):
    n = nextrap or wl.nextrap
    return demigrate_compact_f64(wl.ns, n, wl.nx, wl.nf, wl.nt, wl.M, wl.nk, wl.dk, wl.omega, wl.velocity,
                                 wl.table, wl.wave, refl, shot_x0=wl.shot_x0, shot_nx=wl.shot_nx,
                                 offsets=wl.offsets())


def gather_dense_slab(l0, nl, nx, x0, w, nf, M, nk, dk, omega, velocity, tab, conj_rows=False):
    out = np.empty((nl, nf, w, 2 * M + 1), dtype=np.complex64)
    _load_oracle().oracle_gather_dense_slab(l0, nl, nx, x0, w, nf, M, nk, float(dk),
                                            np.ascontiguousarray(omega, dtype=np.float64),
                                            np.ascontiguousarray(velocity, dtype=np.float64),
                                            np.ascontiguousarray(tab, dtype=np.complex64), int(conj_rows), out)
    return out


def index_table(nextrap, nx, nf, nk, dk, omega, velocity):
    out = np.empty((nf, nextrap, nx), dtype=np.int32)
    _load_oracle().oracle_index_table(nextrap, nx, nf, nk, float(dk), np.ascontiguousarray(omega, dtype=np.float64),
                                      np.ascontiguousarray(velocity, dtype=np.float64), out)
    return out
